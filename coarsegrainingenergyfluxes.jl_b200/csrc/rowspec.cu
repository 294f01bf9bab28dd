// Row-spectral evaluation of the banded footprint sums (Filtering.jl:1569-1744, 2536-2598).
//
// For a target row j and a row offset dj, the footprint's weights depend only on the column offset
// di (the band row's half weights by |di|, over [-a, hi]), so that term of the direct sum,
//     out_j(i) += sum_di w_{j,dj}(di) q_{j+dj}(i + di),
// is a correlation along x of the source row with a fixed kernel.  On a periodic ring of length L
// (or a zero-padded line with L >= nx + a) it is exactly the inverse DFT of conj(K) * Q, where K and
// Q are the DFTs of the kernel row and the source row; every band kernel here is symmetric on the
// ring (the ring-closing rows' extra column -a is the column +a), so K is real.  The sum over dj is
// linear, so it is taken on the spectra:
//     S_j = sum_dj K_{j,dj} Q_{j+dj},   out_j = IDFT(S_j),
// which costs O(L log L) per quantity and row for the transforms plus (2D+1) multiply-adds per
// spectrum bin, instead of the direct sum's (entries per point) per cell.  The result equals the
// direct sum up to FP64 rounding of the transforms (about 1e-15 of a row's magnitude); the epilogue
// (normalisation, tau, rotation, mask) is the direct gather's own finish_target.
//
// Kernels: rs_forward (stage planes -> the NA accumulated quantities -> real DFT of each row as a
// half-length complex Stockham FFT in shared memory -> Q), rs_accumulate (S = banded product over
// rows, per bin), rs_inverse (S -> real inverse DFT of each row, the same way -> F), rs_finish
// (F -> outputs).  Each quantity is transformed on its own, so a quantity's result does not depend on
// which other quantities share the launch (a batch of fields equals the fields filtered one by one,
// bit for bit, as the reference requires of batched applies).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <set>
#include <utility>
#include <vector>

#include "banded_common.cuh"
#include "cgef_internal.h"

namespace cgef {

namespace {

constexpr int kRsThreads = 256;  // threads of the FFT kernels
constexpr int kRsMaxL = 4096;    // longest row: two buffers of kRsSeq half-length rows in shared memory
constexpr int kRsSeq = 2;        // quantities (rows) transformed together by one FFT block
constexpr int kRsAccThreads = 128;
constexpr int kRsRows = 4;  // target rows per thread of the spectral accumulation

struct Fft {
  int L;   // real row length (even)
  int M;   // complex FFT length, L / 2
  int nk;  // bins kept, L / 2 + 1
  int nrad;
  int rad[16];
  const double2* tw;  // exp(-2 pi i n / L), n < L; the length-M roots are every second entry
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -(a.y * b.y)), fma(a.x, b.y, a.y * b.x));
}

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 conj2(double2 a) { return make_double2(a.x, -a.y); }

// In-register R-point forward DFT, X_q = sum_r v_r exp(-2 pi i q r / R).
template <int R>
__device__ __forceinline__ void dft(double2 (&v)[R], const double2* tw, int M) {
  if constexpr (R == 2) {
    const double2 t = v[0];
    v[0] = cadd(t, v[1]);
    v[1] = csub(t, v[1]);
  } else if constexpr (R == 4) {
    const double2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    const double2 a2 = cadd(v[1], v[3]), a3 = csub(v[1], v[3]);
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    v[1] = make_double2(a1.x + a3.y, a1.y - a3.x);  // a1 - i a3
    v[3] = make_double2(a1.x - a3.y, a1.y + a3.x);  // a1 + i a3
  } else {
    // radix 3 and 5: the roots of unity come from the row's own twiddle table
    double2 x[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
      double2 s = v[0];
#pragma unroll
      for (int r = 1; r < R; ++r) s = cadd(s, cmul(v[r], __ldg(tw + 2 * (((q * r) % R) * (M / R)))));
      x[q] = s;
    }
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = x[q];
  }
}

// One Stockham autosort pass of radix R over `nseq` independent length-M sequences stored one after
// another: butterfly j of a sequence reads a[j + r M/R], twiddles by exp(-2 pi i (j mod Ns) r /
// (Ns R)), and writes b[(j / Ns) Ns R + j mod Ns + r Ns].
template <int R>
__device__ __forceinline__ void stockham_pass(const double2* a, double2* b, int M, int Ns, int nseq,
                                              const double2* tw) {
  const int nb = M / R;
  const int tstride = M / (Ns * R);
  for (int t = threadIdx.x; t < nseq * nb; t += blockDim.x) {
    const int sq = t / nb;
    const int j = t - sq * nb;
    const int jm = j % Ns;
    const double2* as = a + sq * M;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      v[r] = as[j + r * nb];
      if (r > 0) v[r] = cmul(v[r], __ldg(tw + 2 * (jm * tstride * r)));
    }
    dft<R>(v, tw, M);
    double2* bs = b + sq * M + (j - jm) * R + jm;
#pragma unroll
    for (int r = 0; r < R; ++r) bs[r * Ns] = v[r];
  }
}

// Forward DFTs of the `nseq` length-M sequences in `a` (shared memory), `b` as scratch; returns the
// buffer holding the transforms in natural order.  Every thread of the block must call it.
__device__ double2* fft_block(double2* a, double2* b, int nseq, const Fft& f) {
  int Ns = 1;
  for (int p = 0; p < f.nrad; ++p) {
    const int R = f.rad[p];
    switch (R) {
      case 2: stockham_pass<2>(a, b, f.M, Ns, nseq, f.tw); break;
      case 3: stockham_pass<3>(a, b, f.M, Ns, nseq, f.tw); break;
      case 4: stockham_pass<4>(a, b, f.M, Ns, nseq, f.tw); break;
      default: stockham_pass<5>(a, b, f.M, Ns, nseq, f.tw); break;
    }
    __syncthreads();
    double2* t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

struct RsK {
  Fft f;
  const double* planes;
  int64_t plane_stride, slice_stride;
  int pitch, halo, nx, ny, D, band_stride, periodic_y, nslices;
  const double* kspec;  // [band][dj + D][bin]
  double2* Q;           // [slice][row][m][bin]
  double2* S;           // [slice][row][m][bin]
  double* F;            // [slice][m][row][nx] (aliases Q once the sums are formed)
};

// Real DFTs of up to kRsSeq of the NA accumulated quantities of one source row (slice, row): each
// row's even and odd samples form one half-length complex sequence z, and with Z = FFT(z) the row's
// spectrum is X_k = E_k + exp(-2 pi i k / L) O_k, E_k = (Z_k + conj Z_{M-k}) / 2,
// O_k = (Z_k - conj Z_{M-k}) / 2i, for k = 0 .. M (Z_M = Z_0).
template <int MODE, int NF, bool DEF>
__global__ void __launch_bounds__(kRsThreads) rs_forward_kernel(RsK k) {
  using C = Cfg<MODE, NF, DEF>;
  extern __shared__ double2 rs_smem[];
  const int M = k.f.M;
  double2* a = rs_smem;
  double2* b = rs_smem + kRsSeq * M;
  const int m0 = blockIdx.x * kRsSeq, jr = blockIdx.y, s = blockIdx.z;
  const int nseq = min(kRsSeq, C::NA - m0);
  const double* row = k.planes + s * k.slice_stride + static_cast<int64_t>(jr) * k.pitch + k.halo;
  double* ad = reinterpret_cast<double*>(a);
  for (int i = threadIdx.x; i < k.f.L; i += blockDim.x) {
    double x[kRsSeq] = {};
    if (i < k.nx) {
      double v[C::NP];
#pragma unroll
      for (int pl = 0; pl < C::NP; ++pl) v[pl] = row[pl * k.plane_stride + i];
      double q[C::NA];
      expand<MODE, NF, DEF>(v, q);
#pragma unroll
      for (int m = 0; m < C::NA; ++m)
#pragma unroll
        for (int e = 0; e < kRsSeq; ++e)
          if (m == m0 + e) x[e] = q[m];
    }
#pragma unroll
    for (int e = 0; e < kRsSeq; ++e)
      if (e < nseq) ad[e * k.f.L + i] = x[e];  // sample i of sequence e: z[i/2].x (even i) or .y (odd)
  }
  __syncthreads();
  const double2* z = fft_block(a, b, nseq, k.f);
  for (int t = threadIdx.x; t < nseq * k.f.nk; t += blockDim.x) {
    const int e = t / k.f.nk;
    const int q = t - e * k.f.nk;
    const double2* ze = z + e * M;
    const double2 zq = ze[q == M ? 0 : q], zc = conj2(ze[q == 0 ? 0 : M - q]);
    const double2 E = make_double2(0.5 * (zq.x + zc.x), 0.5 * (zq.y + zc.y));
    const double2 O = make_double2(0.5 * (zq.y - zc.y), -0.5 * (zq.x - zc.x));  // (zq - zc) / 2i
    k.Q[((static_cast<int64_t>(s) * k.ny + jr) * C::NA + m0 + e) * k.f.nk + q] = cadd(E, cmul(__ldg(k.f.tw + q), O));
  }
}

// S_j = sum_dj K_{j,dj} Q_{j+dj} per bin: one thread per (bin, kRsRows target rows, group of NQ
// quantities of one slice).  Source rows outside a bounded y axis are skipped, as the direct sum
// skips them; on a periodic y axis they wrap.
template <int NQ>
__global__ void __launch_bounds__(kRsAccThreads) rs_accumulate_kernel(RsK k, int na, int ngroups) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int j0 = blockIdx.y * kRsRows;
  const int s = blockIdx.z / ngroups;
  const int mb = (blockIdx.z - s * ngroups) * NQ;
  if (q >= k.f.nk) return;
  const int nq = min(NQ, na - mb);
  const int nk = k.f.nk;
  const int W = 2 * k.D + 1;
  double2 acc[kRsRows][NQ];
#pragma unroll
  for (int t = 0; t < kRsRows; ++t)
#pragma unroll
    for (int m = 0; m < NQ; ++m) acc[t][m] = make_double2(0.0, 0.0);
  const double2* Qs = k.Q + static_cast<int64_t>(s) * k.ny * na * nk;
  for (int jr = j0 - k.D; jr < j0 + kRsRows + k.D; ++jr) {
    int jj = jr;
    if (jr < 0 || jr >= k.ny) {
      if (!k.periodic_y) continue;
      jj = jr % k.ny;
      if (jj < 0) jj += k.ny;
    }
    double2 qv[NQ];
    const double2* qrow = Qs + (static_cast<int64_t>(jj) * na + mb) * nk + q;
#pragma unroll
    for (int m = 0; m < NQ; ++m) qv[m] = m < nq ? qrow[m * nk] : make_double2(0.0, 0.0);
#pragma unroll
    for (int t = 0; t < kRsRows; ++t) {
      const int j = j0 + t;
      const int dj = jr - j;
      if (j < k.ny && dj >= -k.D && dj <= k.D) {
        const double kv = __ldg(k.kspec + (static_cast<int64_t>(k.band_stride ? j : 0) * W + dj + k.D) * nk + q);
#pragma unroll
        for (int m = 0; m < NQ; ++m) {
          acc[t][m].x = fma(kv, qv[m].x, acc[t][m].x);
          acc[t][m].y = fma(kv, qv[m].y, acc[t][m].y);
        }
      }
    }
  }
#pragma unroll
  for (int t = 0; t < kRsRows; ++t) {
    const int j = j0 + t;
    if (j >= k.ny) break;
    double2* srow = k.S + ((static_cast<int64_t>(s) * k.ny + j) * na + mb) * nk + q;
#pragma unroll
    for (int m = 0; m < NQ; ++m)
      if (m < nq) srow[m * nk] = acc[t][m];
  }
}

// Real inverse DFTs of up to kRsSeq summed spectra of one target row: with E'_k = S_k + conj S_{M-k}
// and O'_k = (S_k - conj S_{M-k}) exp(2 pi i k / L), z = IDFT_M(E' + i O') (unnormalised, taken as
// the conjugate of the forward FFT of the conjugate) holds the row's even samples in its real parts
// and its odd samples in its imaginary parts (the kernel spectra carry the 1/L).
template <int NA>
__global__ void __launch_bounds__(kRsThreads) rs_inverse_kernel(RsK k) {
  extern __shared__ double2 rs_smem[];
  const int M = k.f.M;
  double2* a = rs_smem;
  double2* b = rs_smem + kRsSeq * M;
  const int m0 = blockIdx.x * kRsSeq, j = blockIdx.y, s = blockIdx.z;
  const int nseq = min(kRsSeq, NA - m0);
  const double2* S = k.S + ((static_cast<int64_t>(s) * k.ny + j) * NA + m0) * k.f.nk;
  for (int t = threadIdx.x; t < nseq * M; t += blockDim.x) {
    const int e = t / M;
    const int q = t - e * M;
    const double2 sq = S[e * k.f.nk + q], sc = conj2(S[e * k.f.nk + M - q]);
    const double2 Ep = cadd(sq, sc);
    const double2 Op = cmul(csub(sq, sc), conj2(__ldg(k.f.tw + q)));
    // conj(E' + i O')
    a[e * M + q] = make_double2(Ep.x - Op.y, -(Ep.y + Op.x));
  }
  __syncthreads();
  const double2* z = fft_block(a, b, nseq, k.f);
  for (int t = threadIdx.x; t < nseq * k.nx; t += blockDim.x) {
    const int e = t / k.nx;
    const int i = t - e * k.nx;
    const double2 w = z[e * M + (i >> 1)];
    k.F[((static_cast<int64_t>(s) * NA + m0 + e) * k.ny + j) * k.nx + i] = (i & 1) ? -w.y : w.x;
  }
}

template <int MODE, int NF, bool DEF>
__global__ void __launch_bounds__(128) rs_finish_kernel(BandedK a, const double* F) {
  using C = Cfg<MODE, NF, DEF>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, s = blockIdx.z;
  if (i >= a.nx) return;
  const int64_t plane = static_cast<int64_t>(a.ny) * a.nx;
  const double* f = F + static_cast<int64_t>(s) * C::NA * plane + static_cast<int64_t>(j) * a.nx + i;
  double acc[C::NA];
#pragma unroll
  for (int m = 0; m < C::NA; ++m) acc[m] = f[m * plane];
  finish_target<MODE, NF, DEF>(a, acc, s, j, i);
}

// K_{row}(q) / L for every band row: w_0 + 2 sum_{d=1..min(a,hi)} w_d cos(2 pi q d / L), plus
// w_a cos(2 pi q a / L) for a ring-closing row (its column -a), with the cosines read from the
// twiddle table at (q d) mod L.
__global__ void rs_kspec_kernel(const BandRow* rows, int64_t nrows, const double* w, const double2* tw, int L, int nk,
                                double* kspec) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t r = blockIdx.y + static_cast<int64_t>(blockIdx.z) * gridDim.y;
  if (q >= nk || r >= nrows) return;
  const BandRow br = rows[r];
  double sum = 0.0;
  if (br.a >= 0) {
    const double* wr = w + br.woff;
    const int sym = min(br.a, br.hi);
    sum = wr[0];
    for (int d = 1; d <= sym; ++d)
      sum = fma(2.0 * wr[d], __ldg(&tw[static_cast<int64_t>(q) * d % L].x), sum);
    if (br.hi < br.a) sum = fma(wr[br.a], __ldg(&tw[static_cast<int64_t>(q) * br.a % L].x), sum);
  }
  kspec[r * nk + q] = sum / L;
}

int rs_check(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, what);
  count_launch();
  return CGEF_OK;
}

// Opts an FFT kernel into the shared memory its two L-point buffers need (once per kernel and
// device).
int rs_smem_attr(const void* kernel) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({kernel, dev})) return CGEF_OK;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       2 * kRsSeq * static_cast<int>(sizeof(double2)) * (kRsMaxL / 2));
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(row-spectral FFT)");
  done.insert({kernel, dev});
  return CGEF_OK;
}

template <int MODE, int NF, bool DEF>
int run_rowspec(const cgef_plan* p, const BandedK& a, double* scratch, cudaStream_t st) {
  using C = Cfg<MODE, NF, DEF>;
  constexpr int NA = C::NA;
  constexpr int NC = (NA + kRsSeq - 1) / kRsSeq;
  constexpr int NQ = NA <= 5 ? NA : (NA + 1) / 2;
  constexpr int ngroups = (NA + NQ - 1) / NQ;
  RsK k{};
  k.f.L = p->rs_L;
  k.f.M = p->rs_L / 2;
  k.f.nk = p->rs_nk;
  k.f.nrad = p->rs_nrad;
  for (int i = 0; i < p->rs_nrad; ++i) k.f.rad[i] = p->rs_rad[i];
  k.f.tw = reinterpret_cast<const double2*>(p->d_rs_tw);
  k.planes = a.planes;
  k.plane_stride = a.plane_stride;
  k.slice_stride = a.slice_stride;
  k.pitch = a.pitch;
  k.halo = a.halo;
  k.nx = p->nx;
  k.ny = p->ny;
  k.D = p->D;
  k.band_stride = a.band_stride;
  k.periodic_y = p->periodic_y;
  k.nslices = a.nslices;
  k.kspec = p->d_rs_k;
  const size_t spec = static_cast<size_t>(a.nslices) * p->ny * NA * p->rs_nk;
  k.Q = reinterpret_cast<double2*>(scratch);
  k.S = k.Q + spec;
  k.F = scratch;  // Q is dead once S is formed
  const int smem = 2 * kRsSeq * static_cast<int>(sizeof(double2)) * (p->rs_L / 2);
  int rc;
  if ((rc = rs_smem_attr(reinterpret_cast<const void*>(rs_forward_kernel<MODE, NF, DEF>))) != CGEF_OK) return rc;
  if ((rc = rs_smem_attr(reinterpret_cast<const void*>(rs_inverse_kernel<NA>))) != CGEF_OK) return rc;
  prof_begin(CGEF_KERNEL_BANDED, st);
  const dim3 rows(NC, p->ny, a.nslices);
  rs_forward_kernel<MODE, NF, DEF><<<rows, kRsThreads, smem, st>>>(k);
  rc = rs_check("rs_forward_kernel");
  if (rc == CGEF_OK) {
    const dim3 g((p->rs_nk + kRsAccThreads - 1) / kRsAccThreads, (p->ny + kRsRows - 1) / kRsRows,
                 a.nslices * ngroups);
    rs_accumulate_kernel<NQ><<<g, kRsAccThreads, 0, st>>>(k, NA, ngroups);
    rc = rs_check("rs_accumulate_kernel");
  }
  if (rc == CGEF_OK) {
    rs_inverse_kernel<NA><<<rows, kRsThreads, smem, st>>>(k);
    rc = rs_check("rs_inverse_kernel");
  }
  if (rc == CGEF_OK) {
    rs_finish_kernel<MODE, NF, DEF><<<dim3((p->nx + 127) / 128, p->ny, a.nslices), 128, 0, st>>>(a, scratch);
    rc = rs_check("rs_finish_kernel");
  }
  prof_end(CGEF_KERNEL_BANDED, st);
  return rc;
}

template <int MODE, int NF>
int dispatch_rowspec(bool def, const cgef_plan* p, const BandedK& a, double* scratch, cudaStream_t st) {
  return def ? run_rowspec<MODE, NF, true>(p, a, scratch, st) : run_rowspec<MODE, NF, false>(p, a, scratch, st);
}

// Radices of a Stockham plan for L (fours first), or empty when L has a prime factor above 5.
std::vector<int> fft_radices(int L) {
  std::vector<int> rad;
  for (int r : {4, 2, 3, 5})
    while (L % r == 0) {
      rad.push_back(r);
      L /= r;
    }
  if (L != 1) rad.clear();
  return rad;
}

// Smallest L >= n whose prime factors are 2, 3 and 5.
int smooth_length(int n) {
  for (int L = std::max(n, 1);; ++L) {
    int m = L;
    for (int r : {2, 3, 5})
      while (m % r == 0) m /= r;
    if (m == 1) return L;
  }
}

}  // namespace

int launch_rowspec(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                   const uint8_t* mask, int64_t mask_slice_stride, double* scratch, const GatherOut& out,
                   cudaStream_t st) {
  if (!p->rs_on || p->d_rs_k == nullptr) return fail(CGEF_EINVAL, "row-spectral evaluation not built for this plan");
  if (scratch == nullptr) return fail(CGEF_EINVAL, "row-spectral evaluation needs its scratch buffer");
  const bool def = p->strategy == CGEF_DEFORMABLE;
  const BandedK a = make_banded_args(p, mode, planes, pitch, np, nbatch, mask, mask_slice_stride, out);
  if (mode == kModePiSphere) return dispatch_rowspec<kModePiSphere, 1>(def, p, a, scratch, st);
  if (mode == kModePiCart) return dispatch_rowspec<kModePiCart, 1>(def, p, a, scratch, st);
  switch (nf) {
    case 1: return dispatch_rowspec<kModeFields, 1>(def, p, a, scratch, st);
    case 2: return dispatch_rowspec<kModeFields, 2>(def, p, a, scratch, st);
    case 3: return dispatch_rowspec<kModeFields, 3>(def, p, a, scratch, st);
    case 4: return dispatch_rowspec<kModeFields, 4>(def, p, a, scratch, st);
    default: return fail(CGEF_EINVAL, "row-spectral: 1..4 fields per pass");
  }
}

int build_row_spectra(cgef_plan* p) {
  p->rs_L = 0;
  p->rs_on = false;
  if (p->device < 0 || p->engine != CGEF_ENGINE_BANDED || p->h_rows.empty()) return CGEF_OK;
  // A bounded x axis needs symmetric rows (a correlation with a symmetric kernel is the
  // convolution the real spectra describe) and room for the kernel's reach without wrapping.
  if (!p->periodic_x)
    for (const BandRow& r : p->h_rows)
      if (r.a >= 0 && r.hi != r.a) return CGEF_OK;
  // the real rows are transformed as half-length complex sequences, so L is even
  const int L = p->periodic_x ? p->nx : 2 * smooth_length((p->nx + p->Amax + 1) / 2);
  if (L % 2 != 0 || L > kRsMaxL) return CGEF_OK;
  const std::vector<int> rad = fft_radices(L / 2);
  if (rad.empty() || rad.size() > 16) return CGEF_OK;
  const int nk = L / 2 + 1;
  const int64_t nrows = static_cast<int64_t>(p->h_rows.size());
  const size_t kbytes = sizeof(double) * static_cast<size_t>(nrows) * nk;
  if (kbytes > (size_t(8) << 30)) return CGEF_OK;

  std::vector<double> tw(2 * static_cast<size_t>(L));
  for (int n = 0; n < L; ++n) {
    const double ang = 2.0 * 3.14159265358979323846 * (static_cast<double>(n) / L);
    tw[2 * n] = std::cos(ang);
    tw[2 * n + 1] = -std::sin(ang);
  }
  DeviceGuard dg(p->device);
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p->d_rs_tw), tw.size() * sizeof(double));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(row-spectral twiddles)");
  e = cudaMemcpy(p->d_rs_tw, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(row-spectral twiddles)");
  e = cudaMalloc(reinterpret_cast<void**>(&p->d_rs_k), kbytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(row-spectral kernel spectra)");
  const int64_t zchunks = (nrows + 65534) / 65535;
  const dim3 g((nk + 127) / 128, static_cast<unsigned>(std::min<int64_t>(nrows, 65535)), static_cast<unsigned>(zchunks));
  rs_kspec_kernel<<<g, 128>>>(p->d_rows, nrows, p->d_w, reinterpret_cast<const double2*>(p->d_rs_tw), L, nk,
                               p->d_rs_k);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "rs_kspec_kernel");
  if ((e = cudaDeviceSynchronize()) != cudaSuccess) return cuda_fail(e, "rs_kspec_kernel");
  p->rs_L = L;
  p->rs_nk = nk;
  p->rs_nrad = static_cast<int>(rad.size());
  for (size_t i = 0; i < rad.size(); ++i) p->rs_rad[i] = rad[i];
  p->rs_on = true;
  return CGEF_OK;
}

}  // namespace cgef
