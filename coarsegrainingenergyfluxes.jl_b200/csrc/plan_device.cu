// Device part of the spherical footprint build (Filtering.jl:675-731) for large footprints.
//
// The host decides every entry: for each (band j, row offset dj) it finds, with the host's libm, the
// last column offset a whose great-circle distance is within the radius (the distance grows with |di|,
// so the entries of a row are exactly |di| <= a; rows where rounding breaks that order are built on the
// host instead).  What remains is the bulk arithmetic of the weights, one per (row, |di| <= a), and the
// ZeroFill denominators, which this file computes on the device from the host's own row constants:
//     h = sin^2((phi' - phi)/2) + cos(phi) cos(phi') sin^2(|di| dlambda / 2),
//     d = 2 R asin(sqrt(min(h, 1))),   w = exp(-alpha (d / l)^2) * A(row),
// with the same operations in the same order as the host builder; only asin and exp are CUDA's, so a
// weight may differ from the host's by an ulp or two.  Compiled with --fmad=false like the rest.
#include <cstdint>

#include "cgef_internal.h"

namespace cgef {

namespace {

// One warp per band row: its half-row weights at woff[r] + |di| for |di| <= a[r].
__global__ void band_weights_kernel(const BandRow* rows, int64_t nrows, const double* sdp, const double* cc,
                                    const double* area, const double* sdl, double two_r, double alpha, double ell,
                                    int tophat, double* w) {
  const int lane = threadIdx.x & 31;
  const int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (r >= nrows) return;
  const BandRow br = rows[r];
  if (br.a < 0) return;
  const double s = sdp[r], c = cc[r], A = area[r];
  for (int k = lane; k <= br.a; k += 32) {
    double wk;
    if (tophat) {
      wk = 1.0 * A;  // Kernels.jl:318-320: every included offset weighs 1
    } else {
      const double sl = sdl[k];
      double h = s * s + c * sl * sl;
      if (h > 1.0) h = 1.0;
      const double d = two_r * asin(sqrt(h));
      const double q = d / ell;
      wk = exp(-alpha * (q * q)) * A;  // Kernels.jl:322-324
    }
    w[br.woff + k] = wk;
  }
}

// One block per band: the ZeroFill denominator, every in-domain entry's weight (a row's |di| = k > 0
// counts twice when +k is visited too, k <= hi).  Block-wide sums in a fixed order.
__global__ void band_den_kernel(const BandRow* rows, int W, int D, int ny, int periodic_y, const double* w,
                                double* den) {
  __shared__ double part[256];
  const int j = blockIdx.x;
  double s = 0.0;
  for (int rr = 0; rr < W; ++rr) {
    const int jj = j + rr - D;
    if (!periodic_y && (jj < 0 || jj >= ny)) continue;
    const BandRow br = rows[static_cast<int64_t>(j) * W + rr];
    if (br.a < 0) continue;
    for (int k = threadIdx.x; k <= br.a; k += blockDim.x) {
      const double wk = w[br.woff + k];
      s += (k == 0 || k > br.hi) ? wk : 2.0 * wk;
    }
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (static_cast<int>(threadIdx.x) < h) part[threadIdx.x] += part[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) den[j] = part[0];
}

}  // namespace

int device_band_tables(cgef_plan* p, const std::vector<double>& sdp, const std::vector<double>& cc,
                       const std::vector<double>& area, const std::vector<double>& sdl, size_t nweights,
                       const std::vector<std::pair<int64_t, std::vector<double>>>& host_rows) {
  DeviceGuard dg(p->device);
  const int64_t nrows = static_cast<int64_t>(p->h_rows.size());
  double *d_sdp = nullptr, *d_cc = nullptr, *d_area = nullptr, *d_sdl = nullptr;
  auto put = [](double** dst, const std::vector<double>& v) {
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(dst), std::max<size_t>(v.size(), 1) * sizeof(double));
    if (e == cudaSuccess && !v.empty())
      e = cudaMemcpy(*dst, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice);
    return e;
  };
  cudaError_t e = put(&d_sdp, sdp);
  if (e == cudaSuccess) e = put(&d_cc, cc);
  if (e == cudaSuccess) e = put(&d_area, area);
  if (e == cudaSuccess) e = put(&d_sdl, sdl);
  if (e == cudaSuccess)
    e = cudaMalloc(reinterpret_cast<void**>(&p->d_w), std::max<size_t>(nweights, 1) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&p->d_den_zf), sizeof(double) * p->ny);
  if (e == cudaSuccess) {
    const int64_t warps_per_block = 8;
    band_weights_kernel<<<static_cast<unsigned>((nrows + warps_per_block - 1) / warps_per_block),
                          32 * warps_per_block>>>(p->d_rows, nrows, d_sdp, d_cc, d_area, d_sdl, 2.0 * p->R, p->alpha,
                                                   p->scale, p->kernel == CGEF_TOPHAT ? 1 : 0, p->d_w);
    e = cudaGetLastError();
  }
  // rows the host built itself (rounding broke the monotone order there): their weights, zeros included
  for (size_t q = 0; q < host_rows.size() && e == cudaSuccess; ++q)
    e = cudaMemcpy(p->d_w + host_rows[q].first, host_rows[q].second.data(), host_rows[q].second.size() * sizeof(double),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess && p->periodic_x) {
    band_den_kernel<<<p->ny, 256>>>(p->d_rows, 2 * p->D + 1, p->D, p->ny, p->periodic_y, p->d_w, p->d_den_zf);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaFree(d_sdp);
  cudaFree(d_cc);
  cudaFree(d_area);
  cudaFree(d_sdl);
  if (e != cudaSuccess) return cuda_fail(e, "device footprint weights");
  count_launch(p->periodic_x ? 2 : 1);
  return CGEF_OK;
}

}  // namespace cgef
