// Decompositions of the subfilter stress and of the flux (Diagnostics.jl):
//  - tau_decomposition: tau = Leonard + Cross + Reynolds with generalized central moments
//    (Diagnostics.jl:1350-1527, Germano 1992), on the plane and -- in planetary Cartesian
//    components, rotated back to east/north -- on the sphere;
//  - compute_Pi_strain_convergence: Pi = Pi_alpha - Pi_delta (Diagnostics.jl:1724-1852,
//    Srinivasan, Barkan & McWilliams 2023, eq. 10), the strain kernel's epilogue on the plane.
// The filter passes are the plan's own engine over FP64 device planes (up to four fields a pass);
// residuals, products and the final moments are elementwise kernels.
#include <algorithm>
#include <vector>

#include "cgef_internal.h"

namespace cgef {
namespace {

struct DecompK {
  const void* u;
  const void* v;
  int dtype;
  const uint8_t* mask;
  int nx, ny;
  int nv;  // 2 (plane) or 3 (sphere, planetary components)
  const double* sinlam;
  const double* coslam;
  const double* sinphi;
  const double* cosphi;
};

__device__ __forceinline__ double ldv(const void* p, int dtype, int64_t k) {
  return dtype == CGEF_F32 ? static_cast<double>(static_cast<const float*>(p)[k]) : static_cast<const double*>(p)[k];
}

// base[c][q]: the velocity components (planetary X, Y, Z on the sphere; zero on masked cells, as the
// reference converts only active cells, Diagnostics.jl:1475-1482).
__global__ void decomp_base_kernel(DecompK a, double* base) {
  const int64_t N = static_cast<int64_t>(a.nx) * a.ny;
  const int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= N) return;
  const bool act = a.mask == nullptr || a.mask[q] != 0;
  const double u = act ? ldv(a.u, a.dtype, q) : 0.0, v = act ? ldv(a.v, a.dtype, q) : 0.0;
  if (a.nv == 2) {
    base[q] = u;
    base[N + q] = v;
    return;
  }
  const int i = static_cast<int>(q % a.nx), j = static_cast<int>(q / a.nx);
  const double sl = a.sinlam[i], cl = a.coslam[i], sp = a.sinphi[j], cp = a.cosphi[j];
  base[q] = -sl * u - sp * cl * v;
  base[N + q] = cl * u - sp * sl * v;
  base[2 * N + q] = cp * v;
}

// residual u' = u - ubar
__global__ void decomp_residual_kernel(const double* base, const double* bar, double* res, int64_t n) {
  const int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q < n) res[q] = base[q] - bar[q];
}

// products[k][q] = A[ia[k]][q] * B[ib[k]][q] for the k-th product of the list
struct ProdK {
  const double* A;
  const double* B;
  int ia[4], ib[4];
  int nprod;
  double* out;
};

__global__ void decomp_products_kernel(ProdK a, int64_t N) {
  const int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= N) return;
  for (int k = 0; k < a.nprod; ++k) a.out[k * N + q] = a.A[a.ia[k] * N + q] * a.B[a.ib[k] * N + q];
}

// dst[q] += factor * (Fab[q] - Fa[ia][q] * Fb[ib][q])   (one generalized second moment)
struct MomentK {
  const double* Fab;
  const double* Fa;
  const double* Fb;
  int ia, ib;
  double* dst;
  double factor;
};

__global__ void decomp_moment_kernel(MomentK a, int64_t N) {
  const int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= N) return;
  a.dst[q] += a.factor * (a.Fab[q] - a.Fa[a.ia * N + q] * a.Fb[a.ib * N + q]);
}

// L, C, R (symmetric, nv x nv, upper triangle in row-major order) -> local xx, xy, yy outputs.
struct FinishK {
  const double* T;  // [3 parts][ncomp][N]
  int nv, ncomp;
  const uint8_t* mask;
  int nx, ny;
  const double* sinlam;
  const double* coslam;
  const double* sinphi;
  const double* cosphi;
  void* out[9];
  int dtype;
};

__device__ __forceinline__ void st_any(void* p, int dtype, int64_t k, double v) {
  if (dtype == CGEF_F32)
    static_cast<float*>(p)[k] = static_cast<float>(v);
  else
    static_cast<double*>(p)[k] = v;
}

__global__ void decomp_finish_kernel(FinishK a) {
  const int64_t N = static_cast<int64_t>(a.nx) * a.ny;
  const int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= N) return;
  const bool act = a.mask == nullptr || a.mask[q] != 0;
  for (int part = 0; part < 3; ++part) {
    const double* t = a.T + static_cast<int64_t>(part) * a.ncomp * N + q;
    double xx = 0.0, xy = 0.0, yy = 0.0;
    if (act) {
      if (a.nv == 2) {
        xx = t[0];
        xy = t[N];
        yy = t[2 * N];
      } else {
        // planetary tensor -> east/north (the same rotation as the flux's, Diagnostics.jl:449-466)
        const int i = static_cast<int>(q % a.nx), j = static_cast<int>(q / a.nx);
        const double sl = a.sinlam[i], cl = a.coslam[i], sp = a.sinphi[j], cp = a.cosphi[j];
        const double e0 = -sl, e1 = cl, e2 = 0.0;
        const double n0 = -sp * cl, n1 = -sp * sl, n2 = cp;
        const double t00 = t[0], t01 = t[N], t02 = t[2 * N], t11 = t[3 * N], t12 = t[4 * N], t22 = t[5 * N];
        const double te0 = t00 * e0 + t01 * e1 + t02 * e2;
        const double te1 = t01 * e0 + t11 * e1 + t12 * e2;
        const double te2 = t02 * e0 + t12 * e1 + t22 * e2;
        const double tn0 = t00 * n0 + t01 * n1 + t02 * n2;
        const double tn1 = t01 * n0 + t11 * n1 + t12 * n2;
        const double tn2 = t02 * n0 + t12 * n1 + t22 * n2;
        xx = e0 * te0 + e1 * te1 + e2 * te2;
        xy = e0 * tn0 + e1 * tn1 + e2 * tn2;
        yy = n0 * tn0 + n1 * tn1 + n2 * tn2;
      }
    }
    if (a.out[3 * part]) st_any(a.out[3 * part], a.dtype, q, xx);
    if (a.out[3 * part + 1]) st_any(a.out[3 * part + 1], a.dtype, q, xy);
    if (a.out[3 * part + 2]) st_any(a.out[3 * part + 2], a.dtype, q, yy);
  }
}

int check(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, what);
  count_launch();
  return CGEF_OK;
}

// Filters `n` FP64 planes (contiguous, stride N) into `out`, four per pass.
int filter_planes(cgef_plan* p, const double* in, double* out, int n, cudaStream_t st) {
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  for (int k0 = 0; k0 < n; k0 += 4) {
    const int nf = std::min(4, n - k0);
    const void* f[4];
    double* o[4];
    for (int m = 0; m < nf; ++m) {
      f[m] = in + (k0 + m) * N;
      o[m] = out + (k0 + m) * N;
    }
    int rc = filter_fields_device(p, CGEF_F64, f, nf, o, N, 1, p->d_mask, 0, st);
    if (rc) return rc;
  }
  return CGEF_OK;
}

int tau_decomposition_device(cgef_plan* p, int dtype, const void* u, const void* v, const cgef_tau_parts* out,
                             cudaStream_t st) {
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (!u || !v || !out) return fail(CGEF_EINVAL, "u, v and out must be non-NULL");
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const bool sph = p->geometry == CGEF_SPHERICAL;
  const int nv = sph ? 3 : 2;
  const int nsym = nv * (nv + 1) / 2;
  // planes: base, bar, res, Fbar, Fres (nv each), 4 products, 4 filtered products, 3 parts x nsym
  const int64_t planes = 5 * nv + 8 + 3 * nsym;
  void* ws = nullptr;
  if ((rc = ensure_ws(p, kSlotDecomp, sizeof(double) * planes * N, &ws))) return rc;
  double* base = static_cast<double*>(ws);
  double* bar = base + nv * N;
  double* res = bar + nv * N;
  double* Fbar = res + nv * N;
  double* Fres = Fbar + nv * N;
  double* prod = Fres + nv * N;
  double* fprod = prod + 4 * N;
  double* parts = fprod + 4 * N;  // L, C, R
  const unsigned blocks = static_cast<unsigned>((N + 255) / 256);
  cudaError_t e = cudaMemsetAsync(parts, 0, sizeof(double) * 3 * nsym * N, st);
  if (e != cudaSuccess) return cuda_fail(e, "decomposition accumulators");
  DecompK dk{u, v, dtype, p->d_mask, p->nx, p->ny, nv, p->d_sinlam, p->d_coslam, p->d_sinphi, p->d_cosphi};
  decomp_base_kernel<<<blocks, 256, 0, st>>>(dk, base);
  if ((rc = check("decomp_base_kernel"))) return rc;
  // ubar, u' = u - ubar, then the filtered ubar and u' (Diagnostics.jl:1432-1437, 1484-1487)
  if ((rc = filter_planes(p, base, bar, nv, st))) return rc;
  decomp_residual_kernel<<<static_cast<unsigned>((nv * N + 255) / 256), 256, 0, st>>>(base, bar, res, nv * N);
  if ((rc = check("decomp_residual_kernel"))) return rc;
  if ((rc = filter_planes(p, bar, Fbar, nv, st))) return rc;
  if ((rc = filter_planes(p, res, Fres, nv, st))) return rc;
  // the moments: each entry is (A, a, B, b, part, component, factor) with
  // part += factor * M(A_a, B_b), M(f, g) = (fg)bar - fbar gbar
  struct Term {
    int A, a, B, b, part, comp;
    double factor;
  };
  std::vector<Term> terms;
  auto sym = [&](int i, int j) {  // index of (i, j), i <= j, in the upper triangle
    int k = 0;
    for (int m = 0; m < nv; ++m)
      for (int n = m; n < nv; ++n) {
        if (m == i && n == j) return k;
        ++k;
      }
    return -1;
  };
  for (int i = 0; i < nv; ++i)
    for (int j = i; j < nv; ++j) {
      terms.push_back(Term{0, i, 0, j, 0, sym(i, j), 1.0});                      // Leonard M(ubar_i, ubar_j)
      if (i == j) {
        terms.push_back(Term{0, i, 1, i, 1, sym(i, i), 2.0});                    // Cross 2 M(ubar_i, u'_i)
      } else {
        terms.push_back(Term{0, i, 1, j, 1, sym(i, j), 1.0});                    // Cross M(ubar_i, u'_j)
        terms.push_back(Term{1, i, 0, j, 1, sym(i, j), 1.0});                    //     + M(u'_i, ubar_j)
      }
      terms.push_back(Term{1, i, 1, j, 2, sym(i, j), 1.0});                      // Reynolds M(u'_i, u'_j)
    }
  const double* fld[2] = {bar, res};
  const double* flt[2] = {Fbar, Fres};
  for (size_t t0 = 0; t0 < terms.size(); t0 += 4) {
    const int nt = static_cast<int>(std::min<size_t>(4, terms.size() - t0));
    // products of up to four terms share one filter pass
    for (int k = 0; k < nt; ++k) {
      const Term& T = terms[t0 + k];
      ProdK pk{};
      pk.A = fld[T.A];
      pk.B = fld[T.B];
      pk.ia[0] = T.a;
      pk.ib[0] = T.b;
      pk.nprod = 1;
      pk.out = prod + k * N;
      decomp_products_kernel<<<blocks, 256, 0, st>>>(pk, N);
      if ((rc = check("decomp_products_kernel"))) return rc;
    }
    if ((rc = filter_planes(p, prod, fprod, nt, st))) return rc;
    for (int k = 0; k < nt; ++k) {
      const Term& T = terms[t0 + k];
      MomentK mk{fprod + k * N, flt[T.A], flt[T.B], T.a, T.b, parts + (static_cast<int64_t>(T.part) * nsym + T.comp) * N,
                 T.factor};
      decomp_moment_kernel<<<blocks, 256, 0, st>>>(mk, N);
      if ((rc = check("decomp_moment_kernel"))) return rc;
    }
  }
  FinishK fk{};
  fk.T = parts;
  fk.nv = nv;
  fk.ncomp = nsym;
  fk.mask = p->d_mask;
  fk.nx = p->nx;
  fk.ny = p->ny;
  fk.sinlam = p->d_sinlam;
  fk.coslam = p->d_coslam;
  fk.sinphi = p->d_sinphi;
  fk.cosphi = p->d_cosphi;
  for (int k = 0; k < 3; ++k) {
    fk.out[k] = out->leonard[k];
    fk.out[3 + k] = out->cross[k];
    fk.out[6 + k] = out->reynolds[k];
  }
  fk.dtype = dtype;
  decomp_finish_kernel<<<blocks, 256, 0, st>>>(fk);
  return check("decomp_finish_kernel");
}

int strain_convergence_device(cgef_plan* p, int dtype, const void* u, const void* v, int64_t nbatch64,
                              const uint8_t* slice_masks, const cgef_strain_conv_outputs* out, cudaStream_t st) {
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (p->geometry != CGEF_CARTESIAN)
    return fail(CGEF_EUNSUPPORTED, "compute_Pi_strain_convergence is defined on Cartesian grids only");
  if (!u || !v || !out) return fail(CGEF_EINVAL, "u, v and out must be non-NULL");
  if (nbatch64 < 1 || nbatch64 > 65535) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  const int nbatch = static_cast<int>(nbatch64);
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const uint8_t* mask = slice_masks ? slice_masks : p->d_mask;
  const int64_t mstride = slice_masks ? N : 0;
  double* planes = nullptr;
  int pitch = 0, np = 0;
  if ((rc = stage_pi(p, dtype, u, v, nbatch, mask, mstride, p->H, &planes, &pitch, &np, st))) return rc;
  void* gather = nullptr;
  if ((rc = ensure_ws(p, kSlotGather, sizeof(double) * 5 * N * nbatch, &gather))) return rc;
  double* g = static_cast<double*>(gather);
  if ((rc = pi_gather(p, planes, pitch, p->H, np, nbatch, mask, mstride, g, st))) return rc;
  StrainArgs sa{};
  sa.ubar = g;
  sa.vbar = g + N;
  sa.txx = g + 2 * N;
  sa.txy = g + 3 * N;
  sa.tyy = g + 4 * N;
  sa.in_slice_stride = 5 * N;
  sa.mask = mask;
  sa.mask_slice_stride = mstride;
  sa.nbatch = nbatch;
  sa.dtype = dtype;
  sa.out_slice_stride = N;
  sa.sc[0] = out->total;
  sa.sc[1] = out->strain;
  sa.sc[2] = out->convergence;
  sa.sc[3] = out->divergence;
  sa.sc[4] = out->strain_magnitude;
  return launch_strain(p, sa, st);
}

// Host entry points: copy in, run, copy out (synchronous).
int host_buffers(cgef_plan* p, int slot, size_t bytes, void** out) { return ensure_ws(p, slot, bytes, out); }

}  // namespace
}  // namespace cgef

using namespace cgef;

extern "C" {

int32_t cgef_tau_decomposition_device(cgef_plan* p, int32_t dtype, const void* u, const void* v,
                                      const cgef_tau_parts* out, void* stream) {
  int rc = check_plan(p);
  if (rc) return rc;
  DeviceGuard dg(p->device);
  return tau_decomposition_device(p, dtype, u, v, out, static_cast<cudaStream_t>(stream));
}

int32_t cgef_tau_decomposition(cgef_plan* p, int32_t dtype, const void* u, const void* v, const cgef_tau_parts* out) {
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (!u || !v || !out) return fail(CGEF_EINVAL, "u, v and out must be non-NULL");
  DeviceGuard dg(p->device);
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const size_t fb = dsize(dtype) * N;
  void* din = nullptr;
  if ((rc = host_buffers(p, kSlotIn, 2 * fb, &din))) return rc;
  void* dout = nullptr;
  if ((rc = host_buffers(p, kSlotOut, 9 * fb, &dout))) return rc;
  cudaStream_t st = p->stream;
  cudaError_t e = cudaMemcpyAsync(din, u, fb, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(static_cast<char*>(din) + fb, v, fb, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(H2D)");
  cgef_tau_parts dev{};
  void* const* hosts[3] = {out->leonard, out->cross, out->reynolds};
  void** devs[3] = {dev.leonard, dev.cross, dev.reynolds};
  for (int part = 0; part < 3; ++part)
    for (int k = 0; k < 3; ++k)
      devs[part][k] = hosts[part][k] ? static_cast<char*>(dout) + fb * (3 * part + k) : nullptr;
  if ((rc = tau_decomposition_device(p, dtype, din, static_cast<char*>(din) + fb, &dev, st))) return rc;
  for (int part = 0; part < 3; ++part)
    for (int k = 0; k < 3; ++k)
      if (hosts[part][k] &&
          (e = cudaMemcpyAsync(hosts[part][k], devs[part][k], fb, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync(D2H)");
  e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? CGEF_OK : cuda_fail(e, "tau decomposition");
}

int32_t cgef_pi_strain_convergence_device(cgef_plan* p, int32_t dtype, const void* u, const void* v, int64_t nbatch,
                                          const uint8_t* slice_masks, const cgef_strain_conv_outputs* out,
                                          void* stream) {
  int rc = check_plan(p);
  if (rc) return rc;
  DeviceGuard dg(p->device);
  return strain_convergence_device(p, dtype, u, v, nbatch, slice_masks, out, static_cast<cudaStream_t>(stream));
}

int32_t cgef_pi_strain_convergence(cgef_plan* p, int32_t dtype, const void* u, const void* v, int64_t nbatch,
                                   const cgef_strain_conv_outputs* out) {
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (!u || !v || !out) return fail(CGEF_EINVAL, "u, v and out must be non-NULL");
  if (nbatch < 1 || nbatch > 65535) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  DeviceGuard dg(p->device);
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const size_t fb = dsize(dtype) * N * nbatch;
  void* din = nullptr;
  if ((rc = host_buffers(p, kSlotIn, 2 * fb, &din))) return rc;
  void* dout = nullptr;
  if ((rc = host_buffers(p, kSlotOut, 5 * fb, &dout))) return rc;
  cudaStream_t st = p->stream;
  cudaError_t e = cudaMemcpyAsync(din, u, fb, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(static_cast<char*>(din) + fb, v, fb, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(H2D)");
  void* const hosts[5] = {out->total, out->strain, out->convergence, out->divergence, out->strain_magnitude};
  cgef_strain_conv_outputs dev{};
  void** devs[5] = {&dev.total, &dev.strain, &dev.convergence, &dev.divergence, &dev.strain_magnitude};
  for (int k = 0; k < 5; ++k) *devs[k] = hosts[k] ? static_cast<char*>(dout) + fb * k : nullptr;
  if ((rc = strain_convergence_device(p, dtype, din, static_cast<char*>(din) + fb, nbatch, nullptr, &dev, st)))
    return rc;
  for (int k = 0; k < 5; ++k)
    if (hosts[k] && (e = cudaMemcpyAsync(hosts[k], *devs[k], fb, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return cuda_fail(e, "cudaMemcpyAsync(D2H)");
  e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? CGEF_OK : cuda_fail(e, "strain convergence");
}

}  // extern "C"
