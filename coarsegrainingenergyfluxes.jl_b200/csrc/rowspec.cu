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
#include <string>
#include <utility>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "banded_common.cuh"
#include "cgef_internal.h"

namespace cgef {

namespace {

// FFT block shape: 192 threads cover every butterfly of a pass over two 720-point sequences (144, 160
// and 180 for radices 10, 9 and 8) in one round, and 4 such blocks fit an SM at 80 registers a thread
// (46 KB of shared memory each).  On the 0.25 degree sphere this is 9% faster than 128 threads with
// 126 registers; the result is the same bit for bit, as every butterfly's arithmetic is unchanged.
#ifndef CGEF_RS_THREADS
#define CGEF_RS_THREADS 192
#endif
#ifndef CGEF_RS_SEQ
#define CGEF_RS_SEQ 2
#endif
#ifndef CGEF_RS_MINB
#define CGEF_RS_MINB 4
#endif
constexpr int kRsThreads = CGEF_RS_THREADS;  // threads of the FFT kernels
constexpr int kRsMinBlocks = CGEF_RS_MINB;   // resident FFT blocks per SM the kernels are compiled for
constexpr int kRsCols = 8;                   // input columns a thread of the forward FFT loads at once
constexpr int kRsSeq = CGEF_RS_SEQ;          // quantities (rows) transformed together by one FFT block
constexpr int kRsBatch = 4;                  // spectrum bins a thread loads before it uses any of them
// longest row: two buffers of kRsSeq half-length rows (16 bytes a point) within 227 KB of shared memory
constexpr int kRsMaxL = 4096 < (227 * 1024) / (16 * kRsSeq) ? 4096 : (227 * 1024) / (16 * kRsSeq);
constexpr int kRsFftSmem = 2 * kRsSeq * 16 * (kRsMaxL / 2);  // the FFT kernels' shared-memory limit

struct Fft {
  int L;   // real row length (even)
  int M;   // complex FFT length, L / 2
  int nk;  // bins kept, L / 2 + 1
  int nkp; // row stride of the spectra in bins: nk rounded up to 32
  int nrad;
  int rad[16];
  unsigned magic[16];  // ceil(2^32 / Ns) of each pass, Ns = the product of the earlier radices
  const double2* tw;   // exp(-2 pi i n / L), n < L; the length-M roots are every second entry
  // per-pass twiddles, pass p at ptw + poff[p], laid out [r - 1][jm] (r < R, jm < Ns): the entry of tw
  // that the pass multiplies element r of butterfly jm by, so a warp's loads are contiguous
  const double2* ptw;
  int poff[16];
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -(a.y * b.y)), fma(a.x, b.y, a.y * b.x));
}

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 conj2(double2 a) { return make_double2(a.x, -a.y); }

// Forward root of unity W_R^e = exp(-2 pi i e / R) = (cos, -sin) of 2 pi e / R, for the radices whose
// in-register DFTs are composite.  The values are the roots to FP64 precision (computed from their
// series to 50 digits); with the loops unrolled the index is a constant and the table folds away.
template <int R>
__device__ __forceinline__ double2 root(int e) {
  e %= R;
  if constexpr (R == 8) {
    constexpr double c[8] = {1.0, 7.07106781186547573e-01, 0.0, -7.07106781186547573e-01,
                             -1.0, -7.07106781186547573e-01, 0.0, 7.07106781186547573e-01};
    constexpr double sn[8] = {0.0, 7.07106781186547573e-01, 1.0, 7.07106781186547573e-01,
                              0.0, -7.07106781186547573e-01, -1.0, -7.07106781186547573e-01};
    return make_double2(c[e], -sn[e]);
  } else if constexpr (R == 9) {
    constexpr double c[9] = {1.0, 7.66044443118978013e-01, 1.73648177666930359e-01, -0.5, -9.39692620785908428e-01,
                             -9.39692620785908428e-01, -0.5, 1.73648177666930359e-01, 7.66044443118978013e-01};
    constexpr double sn[9] = {0.0, 6.42787609686539363e-01, 9.84807753012208020e-01, 8.66025403784438597e-01,
                              3.42020143325668713e-01, -3.42020143325668713e-01, -8.66025403784438597e-01,
                              -9.84807753012208020e-01, -6.42787609686539363e-01};
    return make_double2(c[e], -sn[e]);
  } else if constexpr (R == 10) {
    constexpr double c[10] = {1.0, 8.09016994374947451e-01, 3.09016994374947451e-01, -3.09016994374947451e-01,
                              -8.09016994374947451e-01, -1.0, -8.09016994374947451e-01, -3.09016994374947451e-01,
                              3.09016994374947451e-01, 8.09016994374947451e-01};
    constexpr double sn[10] = {0.0, 5.87785252292473137e-01, 9.51056516295153531e-01, 9.51056516295153531e-01,
                               5.87785252292473137e-01, 0.0, -5.87785252292473137e-01, -9.51056516295153531e-01,
                               -9.51056516295153531e-01, -5.87785252292473137e-01};
    return make_double2(c[e], -sn[e]);
  } else {
    static_assert(R == 16, "composite radices: 8, 9, 10, 16");
    constexpr double c[16] = {1.0, 9.23879532511286738e-01, 7.07106781186547573e-01, 3.82683432365089782e-01,
                              0.0, -3.82683432365089782e-01, -7.07106781186547573e-01, -9.23879532511286738e-01,
                              -1.0, -9.23879532511286738e-01, -7.07106781186547573e-01, -3.82683432365089782e-01,
                              0.0, 3.82683432365089782e-01, 7.07106781186547573e-01, 9.23879532511286738e-01};
    constexpr double sn[16] = {0.0, 3.82683432365089782e-01, 7.07106781186547573e-01, 9.23879532511286738e-01,
                               1.0, 9.23879532511286738e-01, 7.07106781186547573e-01, 3.82683432365089782e-01,
                               0.0, -3.82683432365089782e-01, -7.07106781186547573e-01, -9.23879532511286738e-01,
                               -1.0, -9.23879532511286738e-01, -7.07106781186547573e-01, -3.82683432365089782e-01};
    return make_double2(c[e], -sn[e]);
  }
}

// v * W_R^e; the quarter turns are exact swaps.
template <int R>
__device__ __forceinline__ double2 rotate(double2 v, int e) {
  e %= R;
  if (e == 0) return v;
  if (4 * e == R) return make_double2(v.y, -v.x);      // -i
  if (2 * e == R) return make_double2(-v.x, -v.y);     // -1
  if (4 * e == 3 * R) return make_double2(-v.y, v.x);  // +i
  return cmul(v, root<R>(e));
}

template <int R>
__device__ __forceinline__ void dft(double2 (&v)[R]);

// R = R1 R2 in registers: R2 DFTs of size R1 over the stride-R2 elements, twiddles W_R^(n2 k1), then
// R1 DFTs of size R2; X[k1 + R1 k2] comes out in natural order.
template <int R1, int R2>
__device__ __forceinline__ void dft_split(double2 (&v)[R1 * R2]) {
  constexpr int R = R1 * R2;
  double2 t[R];
#pragma unroll
  for (int n2 = 0; n2 < R2; ++n2) {
    double2 u[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) u[n1] = v[n2 + R2 * n1];
    dft<R1>(u);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) t[k1 * R2 + n2] = rotate<R>(u[k1], n2 * k1);
  }
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) {
    double2 w[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) w[n2] = t[k1 * R2 + n2];
    dft<R2>(w);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = w[k2];
  }
}

// In-register R-point forward DFT, X_q = sum_r v_r exp(-2 pi i q r / R).
template <int R>
__device__ __forceinline__ void dft(double2 (&v)[R]) {
  if constexpr (R == 2) {
    const double2 t = v[0];
    v[0] = cadd(t, v[1]);
    v[1] = csub(t, v[1]);
  } else if constexpr (R == 3) {
    constexpr double s3 = 8.66025403784438597e-01;  // sin(2 pi / 3)
    const double2 t1 = cadd(v[1], v[2]);
    const double2 t2 = make_double2(v[0].x - 0.5 * t1.x, v[0].y - 0.5 * t1.y);
    const double2 t3 = make_double2(s3 * (v[1].x - v[2].x), s3 * (v[1].y - v[2].y));
    v[0] = cadd(v[0], t1);
    v[1] = make_double2(t2.x + t3.y, t2.y - t3.x);  // t2 - i t3
    v[2] = make_double2(t2.x - t3.y, t2.y + t3.x);  // t2 + i t3
  } else if constexpr (R == 4) {
    const double2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    const double2 a2 = cadd(v[1], v[3]), a3 = csub(v[1], v[3]);
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    v[1] = make_double2(a1.x + a3.y, a1.y - a3.x);  // a1 - i a3
    v[3] = make_double2(a1.x - a3.y, a1.y + a3.x);  // a1 + i a3
  } else if constexpr (R == 5) {
    constexpr double c1 = 3.09016994374947451e-01, c2 = -8.09016994374947451e-01;  // cos(2 pi / 5), cos(4 pi / 5)
    constexpr double s1 = 9.51056516295153531e-01, s2 = 5.87785252292473137e-01;   // sin(2 pi / 5), sin(4 pi / 5)
    const double2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    const double2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    const double2 a1 = make_double2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    const double2 a2 = make_double2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    const double2 b1 = make_double2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
    const double2 b2 = make_double2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = make_double2(a1.x + b1.y, a1.y - b1.x);  // a1 - i b1
    v[4] = make_double2(a1.x - b1.y, a1.y + b1.x);  // a1 + i b1
    v[2] = make_double2(a2.x + b2.y, a2.y - b2.x);  // a2 - i b2
    v[3] = make_double2(a2.x - b2.y, a2.y + b2.x);  // a2 + i b2
  } else if constexpr (R == 8) {
    dft_split<2, 4>(v);
  } else if constexpr (R == 9) {
    dft_split<3, 3>(v);
  } else if constexpr (R == 10) {
    dft_split<2, 5>(v);
  } else {
    static_assert(R == 16, "radices 2, 3, 4, 5, 8, 9, 10, 16");
    dft_split<4, 4>(v);
  }
}

// One Stockham autosort pass of radix R over `nseq` independent length-M sequences stored one after
// another: butterfly j of a sequence reads a[j + r M/R], twiddles by exp(-2 pi i (j mod Ns) r /
// (Ns R)), and writes b[(j / Ns) Ns R + j mod Ns + r Ns].  j / Ns is __umulhi(j, ns_magic) with
// ns_magic = ceil(2^32 / Ns) (Ns > 1), exact for j, Ns < 2^16.  The butterflies of all the sequences
// are one range over the block's threads (t = sq * M/R + j), so a block of nseq * M/R threads or more
// does a pass in one round.  TW false: the first pass (Ns = 1), whose twiddles are all 1, applies none
// (2-4% faster FFT kernels at L = 1440).
template <int R, bool TW>
__device__ __forceinline__ void stockham_pass(const double2* a, double2* b, int M, int Ns, unsigned ns_magic,
                                              int nseq, const double2* ptw) {
  const int nb = M / R;
  for (int t = threadIdx.x; t < nseq * nb; t += blockDim.x) {
    int sq = 0, j = t;
#pragma unroll
    for (int e = 1; e < kRsSeq; ++e)  // nseq <= kRsSeq
      if (j >= nb) j -= nb, ++sq;
    const double2* as = a + sq * M;
    const int jq = Ns == 1 ? j : static_cast<int>(__umulhi(static_cast<unsigned>(j), ns_magic));
    const int jm = j - jq * Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = as[j + r * nb];
    if constexpr (TW) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], __ldg(ptw + (r - 1) * Ns + jm));
    }
    dft<R>(v);
    double2* bs = b + sq * M + jq * Ns * R + jm;
#pragma unroll
    for (int r = 0; r < R; ++r) bs[r * Ns] = v[r];
  }
}

// The same pass with its input and output through functors: src(sq, n) gives element n of sequence sq,
// sink(sq, n, v) takes element n of the pass's output.  The inverse transform writes its last pass
// straight out as real samples, so that pass needs no shared-memory round trip and no barrier after it.
template <int R, bool TW, typename Src, typename Sink>
__device__ __forceinline__ void stockham_pass_io(Src src, Sink sink, int M, int Ns, unsigned ns_magic, int nseq,
                                                 const double2* ptw) {
  const int nb = M / R;
  for (int t = threadIdx.x; t < nseq * nb; t += blockDim.x) {
    int sq = 0, j = t;
#pragma unroll
    for (int e = 1; e < kRsSeq; ++e)
      if (j >= nb) j -= nb, ++sq;
    const int jq = Ns == 1 ? j : static_cast<int>(__umulhi(static_cast<unsigned>(j), ns_magic));
    const int jm = j - jq * Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src(sq, j + r * nb);
    if constexpr (TW) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], __ldg(ptw + (r - 1) * Ns + jm));
    }
    dft<R>(v);
#pragma unroll
    for (int r = 0; r < R; ++r) sink(sq, jq * Ns * R + jm + r * Ns, v[r]);
  }
}

template <bool TW, typename Src, typename Sink>
__device__ __forceinline__ void pass_io(int R, Src src, Sink sink, int M, int Ns, unsigned mg, int nseq,
                                        const double2* ptw) {
  switch (R) {
    case 2: stockham_pass_io<2, TW>(src, sink, M, Ns, mg, nseq, ptw); break;
    case 3: stockham_pass_io<3, TW>(src, sink, M, Ns, mg, nseq, ptw); break;
    case 4: stockham_pass_io<4, TW>(src, sink, M, Ns, mg, nseq, ptw); break;
    case 5: stockham_pass_io<5, TW>(src, sink, M, Ns, mg, nseq, ptw); break;
    case 8: stockham_pass_io<8, TW>(src, sink, M, Ns, mg, nseq, ptw); break;
    case 9: stockham_pass_io<9, TW>(src, sink, M, Ns, mg, nseq, ptw); break;
    case 10: stockham_pass_io<10, TW>(src, sink, M, Ns, mg, nseq, ptw); break;
    default:  // radix 16; callers pass TW false only for the others (a third inlined copy spills)
      if constexpr (TW) stockham_pass_io<16, true>(src, sink, M, Ns, mg, nseq, ptw);
      break;
  }
}

// Forward DFTs of the `nseq` length-M sequences in `a` (shared memory), `b` as scratch; returns the
// buffer holding the transforms in natural order.  Every thread of the block must call it.
__device__ __forceinline__ double2* fft_block(double2* a, double2* b, int nseq, const Fft& f) {
  int Ns = 1;
  for (int p = 0; p < f.nrad; ++p) {
    const int R = f.rad[p];
    const unsigned mg = f.magic[p];
    const double2* tp = f.ptw + f.poff[p];
    if (p == 0 && R != 16) {  // the first pass's twiddles are all 1: none are applied (radix 16 below)
      switch (R) {
        case 2: stockham_pass<2, false>(a, b, f.M, Ns, mg, nseq, tp); break;
        case 3: stockham_pass<3, false>(a, b, f.M, Ns, mg, nseq, tp); break;
        case 4: stockham_pass<4, false>(a, b, f.M, Ns, mg, nseq, tp); break;
        case 5: stockham_pass<5, false>(a, b, f.M, Ns, mg, nseq, tp); break;
        case 8: stockham_pass<8, false>(a, b, f.M, Ns, mg, nseq, tp); break;
        case 9: stockham_pass<9, false>(a, b, f.M, Ns, mg, nseq, tp); break;
        case 10: stockham_pass<10, false>(a, b, f.M, Ns, mg, nseq, tp); break;
        default: break;
      }
    } else {
      switch (R) {
        case 2: stockham_pass<2, true>(a, b, f.M, Ns, mg, nseq, tp); break;
        case 3: stockham_pass<3, true>(a, b, f.M, Ns, mg, nseq, tp); break;
        case 4: stockham_pass<4, true>(a, b, f.M, Ns, mg, nseq, tp); break;
        case 5: stockham_pass<5, true>(a, b, f.M, Ns, mg, nseq, tp); break;
        case 8: stockham_pass<8, true>(a, b, f.M, Ns, mg, nseq, tp); break;
        case 9: stockham_pass<9, true>(a, b, f.M, Ns, mg, nseq, tp); break;
        case 10: stockham_pass<10, true>(a, b, f.M, Ns, mg, nseq, tp); break;
        default: stockham_pass<16, true>(a, b, f.M, Ns, mg, nseq, tp); break;
      }
    }
    __syncthreads();
    double2* t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

// The same passes with every size known at compile time, for the transform length the 0.25 degree
// sphere uses (M = 720 = 10 x 9 x 8): no radix dispatch, the butterfly range and Ns fixed, the
// division by Ns a constant one.  Same arithmetic, same results.
#ifndef CGEF_RS_CT720
#define CGEF_RS_CT720 1
#endif

template <int R, int NS, int M, bool TW, typename Src, typename Sink>
__device__ __forceinline__ void stockham_pass_ct(Src src, Sink sink, int nseq, const double2* ptw) {
  constexpr int nb = M / R;
  for (int t = threadIdx.x; t < nseq * nb; t += kRsThreads) {
    int sq = 0, j = t;
#pragma unroll
    for (int e = 1; e < kRsSeq; ++e)
      if (j >= nb) j -= nb, ++sq;
    const int jq = j / NS, jm = j - jq * NS;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src(sq, j + r * nb);
    if constexpr (TW) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], __ldg(ptw + (r - 1) * NS + jm));
    }
    dft<R>(v);
#pragma unroll
    for (int r = 0; r < R; ++r) sink(sq, jq * NS * R + jm + r * NS, v[r]);
  }
}

// The three passes of a 720-point transform through shared memory (a, then b as scratch); the last
// pass's output goes to `last` (a sink); returns after the passes (no barrier after the last).
template <typename Last>
__device__ __forceinline__ void fft720(double2* a, double2* b, int nseq, const Fft& f, Last last) {
  constexpr int M = 720;
  auto from = [](const double2* s) { return [s](int e, int n) { return s[e * M + n]; }; };
  auto to = [](double2* d) { return [d](int e, int n, double2 v) { d[e * M + n] = v; }; };
  stockham_pass_ct<10, 1, M, false>(from(a), to(b), nseq, f.ptw + f.poff[0]);
  __syncthreads();
  stockham_pass_ct<9, 10, M, true>(from(b), to(a), nseq, f.ptw + f.poff[1]);
  __syncthreads();
  stockham_pass_ct<8, 90, M, true>(from(a), last, nseq, f.ptw + f.poff[2]);
}

__host__ __device__ inline bool is_fft720(const Fft& f) {
  return f.M == 720 && f.nrad == 3 && f.rad[0] == 10 && f.rad[1] == 9 && f.rad[2] == 8;
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
// LC: the real row length when known at compile time (1440 with the 720-point passes), else 0.
template <int MODE, int NF, bool DEF, int LC>
__device__ __forceinline__ void forward_body(const RsK& k) {
  using C = Cfg<MODE, NF, DEF>;
  extern __shared__ double2 rs_smem[];
  const int L = LC ? LC : k.f.L;
  const int M = LC ? LC / 2 : k.f.M;
  const int nkp = LC ? (LC / 2 + 1 + 31) / 32 * 32 : k.f.nkp;
  double2* a = rs_smem;
  double2* b = rs_smem + kRsSeq * M;
  const int m0 = blockIdx.x * kRsSeq, jr = blockIdx.y, s = blockIdx.z;
  const int nseq = min(kRsSeq, C::NA - m0);
  const double* row = k.planes + s * k.slice_stride + static_cast<int64_t>(jr) * k.pitch + k.halo;
  double* ad = reinterpret_cast<double*>(a);
  // kRsCols columns per thread at a time, their loads issued together
  for (int i0 = 0; i0 < L; i0 += kRsCols * kRsThreads) {
    double v[kRsCols][C::NP];
#pragma unroll
    for (int c = 0; c < kRsCols; ++c) {
      const int i = i0 + c * kRsThreads + threadIdx.x;
      const int ic = i < k.nx ? i : 0;
#pragma unroll
      for (int pl = 0; pl < C::NP; ++pl) v[c][pl] = row[pl * k.plane_stride + ic];
    }
#pragma unroll
    for (int c = 0; c < kRsCols; ++c) {
      const int i = i0 + c * kRsThreads + threadIdx.x;
      if (i >= L) break;
#pragma unroll
      for (int e = 0; e < kRsSeq; ++e)
        if (e < nseq)  // sample i of sequence e: z[i/2].x (even i) or .y (odd)
          ad[e * L + i] = i < k.nx ? quantity<MODE, NF, DEF>(v[c], m0 + e) : 0.0;
    }
  }
  __syncthreads();
  const double2* z;
  if constexpr (LC == 1440) {
    fft720(a, b, nseq, k.f, [b](int e, int n, double2 v) { b[e * 720 + n] = v; });
    __syncthreads();
    z = b;
  } else {
    z = fft_block(a, b, nseq, k.f);
  }
  // bin q of sequence e is item t = e * nk + q; a thread loads kRsBatch items' operands, then stores
  const int nk = LC ? LC / 2 + 1 : k.f.nk, items = nseq * nk;
  double2* Q0 = k.Q + ((static_cast<int64_t>(s) * k.ny + jr) * C::NA + m0) * nkp;
  for (int t0 = 0; t0 < items; t0 += kRsBatch * kRsThreads) {
    double2 w[kRsBatch], zq[kRsBatch], zc[kRsBatch];
#pragma unroll
    for (int u = 0; u < kRsBatch; ++u) {
      int q = min(t0 + u * kRsThreads + static_cast<int>(threadIdx.x), items - 1), e = 0;
#pragma unroll
      for (int i = 1; i < kRsSeq; ++i)
        if (q >= nk) q -= nk, ++e;
      w[u] = __ldg(k.f.tw + q);
      zq[u] = z[e * M + (q == M ? 0 : q)];
      zc[u] = conj2(z[e * M + (q == 0 ? 0 : M - q)]);
    }
#pragma unroll
    for (int u = 0; u < kRsBatch; ++u) {
      const int t = t0 + u * kRsThreads + threadIdx.x;
      if (t < items) {  // a guarded store, not a break: the break form measured 4% slower
        int q = t, e = 0;
#pragma unroll
        for (int i = 1; i < kRsSeq; ++i)
          if (q >= nk) q -= nk, ++e;
        const double2 E = make_double2(0.5 * (zq[u].x + zc[u].x), 0.5 * (zq[u].y + zc[u].y));
        const double2 O = make_double2(0.5 * (zq[u].y - zc[u].y), -0.5 * (zq[u].x - zc[u].x));  // (zq - zc) / 2i
        Q0[e * nkp + q] = cadd(E, cmul(w[u], O));
      }
    }
  }
}

template <int MODE, int NF, bool DEF>
__global__ void __launch_bounds__(kRsThreads, kRsMinBlocks) rs_forward_kernel(RsK k) {
  if (CGEF_RS_CT720 && is_fft720(k.f))
    forward_body<MODE, NF, DEF, 1440>(k);
  else
    forward_body<MODE, NF, DEF, 0>(k);
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc, bool fill) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  const int n = fill ? 16 : 0;  // 0: the 16 bytes are zero-filled and nothing is read
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gsrc), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// S_j = sum_dj K_{j,dj} Q_{j+dj} per bin.  A block owns 32 bins x TJ target rows x every quantity and
// walks the in-domain source rows its band touches; per source row it stages that row's spectra (all
// quantities) and the TJ kernel-spectrum slices that apply to it in shared memory through a
// kAccStages-deep cp.async pipeline of kAccRps rows a stage (one block barrier per stage), and each
// warp adds them into a register tile of RW target rows x every quantity, so one staged kernel value
// serves NA quantities and one staged source value RW rows (NA x RW complex multiply-adds per NA + RW
// shared-memory reads).  Rows off a bounded y axis are skipped (the direct sum skips them); on a
// periodic y axis they wrap.  Three rows a stage (104 KB of shared memory a block, two blocks an SM)
// made the 0.25 degree flux step 4% faster than one row a stage; six one-row stages or two-row
// stages gained less.  Banded spheres stage through tensor copies instead (rs_accumulate_tma_kernel).
#ifndef CGEF_ACC_STAGES
#define CGEF_ACC_STAGES 4
#endif
#ifndef CGEF_ACC_RPS
#define CGEF_ACC_RPS 3
#endif
constexpr int kAccStages = CGEF_ACC_STAGES;
constexpr int kAccRps = CGEF_ACC_RPS;  // source rows a pipeline stage holds (one block barrier each)
// target rows of an accumulation block: 16 at every band height (32-row blocks, one per SM, were 15%
// slower at 2000 km and 14% slower at 100 km: every stage's barrier then stalls the whole SM)
#ifndef CGEF_ACC_ROWS
#define CGEF_ACC_ROWS 16
#endif
constexpr int kAccRows = CGEF_ACC_ROWS;

template <int NA>
struct AccTile {
  static constexpr int RW = NA > 5 ? 4 : 8;  // target rows of a warp's register tile
};

template <int TJ, int NA>
__global__ void __launch_bounds__(32 * (TJ / AccTile<NA>::RW), 1) rs_accumulate_kernel(RsK k) {
  extern __shared__ __align__(16) unsigned char rs_acc_smem[];
  constexpr int RW = AccTile<NA>::RW;
  constexpr int kThreads = 32 * (TJ / RW);
  constexpr int kQChunks = (NA * 32 + kThreads - 1) / kThreads;  // 16-byte source-spectrum chunks per thread
  constexpr int kKChunks = (TJ * 16 + kThreads - 1) / kThreads;  // 16-byte kernel-spectrum chunks per thread
  constexpr int qbytes = NA * 32 * 16;
  constexpr int sbytes = qbytes + TJ * 32 * 8;
  const int lane = threadIdx.x & 31;
  const int rg = threadIdx.x >> 5;  // the warp's rows: rg * RW .. rg * RW + RW - 1
  const int q0 = blockIdx.x * 32;
  const int j0 = blockIdx.y * TJ;
  const int s = blockIdx.z;
  const int nkp = k.f.nkp;
  const int W = 2 * k.D + 1;
  // source rows jr = j0 - D + step; off a bounded y axis they are skipped
  int st0 = 0, st1 = TJ + 2 * k.D;
  if (!k.periodic_y) {
    st0 = max(0, k.D - j0);
    st1 = min(st1, k.ny - j0 + k.D);
  }
  // this thread's copies, their offsets fixed but for the source row
  const double2* q_base = k.Q + static_cast<int64_t>(s) * k.ny * NA * nkp + q0;
  int64_t q_off[kQChunks];
#pragma unroll
  for (int i = 0; i < kQChunks; ++i) {
    const int c = threadIdx.x + i * kThreads;
    q_off[i] = c < NA * 32 ? static_cast<int64_t>(c >> 5) * nkp + (c & 31) : 0;
  }
  int k_j[kKChunks];
  int64_t k_base[kKChunks];
#pragma unroll
  for (int i = 0; i < kKChunks; ++i) {
    const int c = threadIdx.x + i * kThreads;
    k_j[i] = c < TJ * 16 ? j0 + (c >> 4) : k.ny;  // k.ny: no copy
    k_base[i] = (static_cast<int64_t>(k.band_stride ? k_j[i] : 0) * W + k.D - k_j[i]) * nkp + q0 + 2 * (c & 15);
  }

  auto issue_row = [&](int step, unsigned char* b) {
    const int jraw = j0 - k.D + step;
    int jr = jraw;
    if (jr < 0 || jr >= k.ny) {  // only reached on a periodic y axis
      jr %= k.ny;
      if (jr < 0) jr += k.ny;
    }
    const double2* qrow = q_base + static_cast<int64_t>(jr) * NA * nkp;
#pragma unroll
    for (int i = 0; i < kQChunks; ++i) {
      const int c = threadIdx.x + i * kThreads;
      if (c < NA * 32) cp_async16(b + c * 16, qrow + q_off[i], true);
    }
#pragma unroll
    for (int i = 0; i < kKChunks; ++i) {
      const int c = threadIdx.x + i * kThreads;
      if (c < TJ * 16) {
        const int dj = jraw - k_j[i];
        const bool ok = k_j[i] < k.ny && dj >= -k.D && dj <= k.D;
        cp_async16(b + qbytes + c * 16, k.kspec + (ok ? k_base[i] + static_cast<int64_t>(jraw) * nkp : 0), ok);
      }
    }
  };
  auto issue = [&](int step, int buf) {
#pragma unroll
    for (int r = 0; r < kAccRps; ++r)
      if (step + r < st1) issue_row(step + r, rs_acc_smem + (buf * kAccRps + r) * sbytes);
  };

  double2 acc[RW][NA];
#pragma unroll
  for (int t = 0; t < RW; ++t)
#pragma unroll
    for (int m = 0; m < NA; ++m) acc[t][m] = make_double2(0.0, 0.0);
#pragma unroll
  for (int i = 0; i < kAccStages - 1; ++i) {
    if (st0 + i * kAccRps < st1) issue(st0 + i * kAccRps, i);
    cp_async_commit();
  }
  for (int sg = st0; sg < st1; sg += kAccRps) {
    cp_async_wait<kAccStages - 2>();
    __syncthreads();
    const int nxt = sg + (kAccStages - 1) * kAccRps;
    if (nxt < st1) issue(nxt, ((nxt - st0) / kAccRps) % kAccStages);
    cp_async_commit();
    const unsigned char* sb = rs_acc_smem + (((sg - st0) / kAccRps) % kAccStages) * kAccRps * sbytes;
#pragma unroll
    for (int r = 0; r < kAccRps; ++r) {
      if (sg + r >= st1) break;
      const unsigned char* b = sb + r * sbytes;
      const double2* qb = reinterpret_cast<const double2*>(b) + lane;
      const double* kb = reinterpret_cast<const double*>(b + qbytes) + rg * RW * 32 + lane;
      double kv[RW];
#pragma unroll
      for (int t = 0; t < RW; ++t) kv[t] = kb[t * 32];
#pragma unroll
      for (int m = 0; m < NA; ++m) {
        const double2 a = qb[m * 32];
#pragma unroll
        for (int t = 0; t < RW; ++t) {
          acc[t][m].x = fma(kv[t], a.x, acc[t][m].x);
          acc[t][m].y = fma(kv[t], a.y, acc[t][m].y);
        }
      }
    }
  }
  cp_async_wait<0>();
  double2* Ss = k.S + static_cast<int64_t>(s) * k.ny * NA * nkp + q0 + lane;
#pragma unroll
  for (int t = 0; t < RW; ++t) {
    const int j = j0 + rg * RW + t;
    if (j >= k.ny) break;
    double2* sr = Ss + static_cast<int64_t>(j) * NA * nkp;
#pragma unroll
    for (int m = 0; m < NA; ++m) sr[m * nkp] = acc[t][m];
  }
}

// The same sums with each source row staged by two tensor copies (TMA): one box of the row's spectra
// (32 bins x every quantity) and one of the TJ target rows' kernel-spectrum slices, the latter through a
// 3-D view of the kernel spectra whose axes are the bin, D + the source row and the target row (the
// entry of target j, source row jr is row j (2D) + D + jr of the table, so the target axis has stride
// 2D rows).  One thread issues both copies onto the stage's mbarrier; there is no per-thread copy
// arithmetic.  Slices of target rows out of the band are read (finite neighbours in the table) and
// ignored: their kernel values are taken as 0.  Banded spheres (one band per row, bounded y, D >= 1)
// only; every wait is bounded and a block whose barrier does not complete writes NaN sums.
#ifndef CGEF_ACC_TMA
#define CGEF_ACC_TMA 1
#endif
constexpr long long kAccWaitCycles = 200000000LL;  // about 0.1 s

__device__ __forceinline__ uint32_t tma_smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void tma_bar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tma_bar_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool tma_bar_wait(uint32_t bar, uint32_t parity, long long limit) {
  const long long start = clock64();
  for (int it = 1;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 63) == 0 && clock64() - start > limit) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

// Two source rows a stage and three blocks an SM (168 registers, 70 KB of shared memory a block) where
// the tile fits without spilling (NA <= 9): 2.8% faster on the 24-scale sweep than three rows a stage
// at two blocks an SM.
constexpr int kTmaRps = 2;
template <int NA>
constexpr int tma_min_blocks() {
  return NA <= 9 ? 3 : 1;
}
template <int TJ, int NA>
__global__ void __launch_bounds__(32 * (TJ / AccTile<NA>::RW), tma_min_blocks<NA>())
    rs_accumulate_tma_kernel(RsK k, const __grid_constant__ CUtensorMap qmap, const __grid_constant__ CUtensorMap kmap) {
  extern __shared__ __align__(128) unsigned char rs_tma_smem[];
  __shared__ __align__(8) uint64_t full[kAccStages];
  constexpr int RW = AccTile<NA>::RW;
  constexpr int qbytes = NA * 32 * 16;
  constexpr int sbytes = qbytes + TJ * 32 * 8;  // one source row's boxes, both multiples of 128 bytes
  static_assert(qbytes % 128 == 0 && sbytes % 128 == 0, "tensor-copy destinations 128-byte aligned");
  const int lane = threadIdx.x & 31;
  const int rg = threadIdx.x >> 5;  // the warp's rows: rg * RW .. rg * RW + RW - 1
  const int q0 = blockIdx.x * 32;
  const int j0 = blockIdx.y * TJ;
  const int s = blockIdx.z;
  const int nkp = k.f.nkp;
  const int D = k.D, ny = k.ny;
  const int st0 = max(0, D - j0), st1 = min(TJ + 2 * D, ny - j0 + D);  // in-domain source rows only
  if (threadIdx.x == 0) {
    for (int b = 0; b < kAccStages; ++b) tma_bar_init(tma_smem_u32(&full[b]));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // thread 0: the copies of the stage that starts at source step sg, into buffer buf
  auto issue = [&](int sg, int buf) {
    const uint32_t bar = tma_smem_u32(&full[buf]);
    const int nrows = min(kTmaRps, st1 - sg);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tma_bar_expect(bar, static_cast<uint32_t>(nrows * sbytes));
    for (int r = 0; r < nrows; ++r) {
      const int jraw = j0 - D + sg + r;
      const uint32_t dst = tma_smem_u32(rs_tma_smem + (buf * kTmaRps + r) * sbytes);
      tma_load_2d(dst, &qmap, 2 * q0, (s * ny + jraw) * NA, bar);
      tma_load_3d(dst + qbytes, &kmap, q0, D + jraw, j0, bar);
    }
  };
  double2 acc[RW][NA];
#pragma unroll
  for (int t = 0; t < RW; ++t)
#pragma unroll
    for (int m = 0; m < NA; ++m) acc[t][m] = make_double2(0.0, 0.0);
  const int ng = (st1 - st0 + kTmaRps - 1) / kTmaRps;  // stages of this block
  if (threadIdx.x == 0)
    for (int i = 0; i < kAccStages - 1 && i < ng; ++i) issue(st0 + i * kTmaRps, i);
  int failed = -1;
  for (int gi = 0; gi < ng; ++gi) {
    const int sg = st0 + gi * kTmaRps, buf = gi % kAccStages;
    const bool got = tma_bar_wait(tma_smem_u32(&full[buf]), (gi / kAccStages) & 1, kAccWaitCycles);
    if (__syncthreads_or(!got)) {
      failed = gi;
      break;
    }
    const int nx = gi + kAccStages - 1;
    if (threadIdx.x == 0 && nx < ng) issue(st0 + nx * kTmaRps, nx % kAccStages);
    const unsigned char* sb = rs_tma_smem + buf * kTmaRps * sbytes;
#pragma unroll
    for (int r = 0; r < kTmaRps; ++r) {
      const int st = sg + r;
      if (st >= st1) break;
      const unsigned char* b = sb + r * sbytes;
      const double2* qb = reinterpret_cast<const double2*>(b) + lane;
      const double* kb = reinterpret_cast<const double*>(b + qbytes) + rg * RW * 32 + lane;
      double kv[RW];
#pragma unroll
      for (int t = 0; t < RW; ++t)  // target row j0 + rg RW + t is in this source row's band
        kv[t] = static_cast<unsigned>(st - rg * RW - t) <= static_cast<unsigned>(2 * D) ? kb[t * 32] : 0.0;
#pragma unroll
      for (int m = 0; m < NA; ++m) {
        const double2 a = qb[m * 32];
#pragma unroll
        for (int t = 0; t < RW; ++t) {
          acc[t][m].x = fma(kv[t], a.x, acc[t][m].x);
          acc[t][m].y = fma(kv[t], a.y, acc[t][m].y);
        }
      }
    }
  }
  if (failed >= 0) {
    // a barrier did not complete: let the copies still in flight land (bounded again), then give NaN
    // sums so the result cannot pass for a valid one
    const int issued = min(ng, failed + kAccStages - 1);
    for (int gi = failed; gi < issued; ++gi)
      tma_bar_wait(tma_smem_u32(&full[gi % kAccStages]), (gi / kAccStages) & 1, kAccWaitCycles / 8);
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
    for (int t = 0; t < RW; ++t)
#pragma unroll
      for (int m = 0; m < NA; ++m) acc[t][m] = make_double2(nan, nan);
  }
  double2* Ss = k.S + static_cast<int64_t>(s) * ny * NA * nkp + q0 + lane;
#pragma unroll
  for (int t = 0; t < RW; ++t) {
    const int j = j0 + rg * RW + t;
    if (j >= ny) break;
    double2* sr = Ss + static_cast<int64_t>(j) * NA * nkp;
#pragma unroll
    for (int m = 0; m < NA; ++m) sr[m * nkp] = acc[t][m];
  }
}

// Real inverse DFTs of up to kRsSeq summed spectra of one target row: with E'_k = S_k + conj S_{M-k}
// and O'_k = (S_k - conj S_{M-k}) exp(2 pi i k / L), z = IDFT_M(E' + i O') (unnormalised, taken as
// the conjugate of the forward FFT of the conjugate) holds the row's even samples in its real parts
// and its odd samples in its imaginary parts (the kernel spectra carry the 1/L).
template <int NA, int LC>
__device__ __forceinline__ void inverse_body(const RsK& k) {
  extern __shared__ double2 rs_smem[];
  const int M = LC ? LC / 2 : k.f.M;
  const int nkp = LC ? (LC / 2 + 1 + 31) / 32 * 32 : k.f.nkp;
  double2* a = rs_smem;
  double2* b = rs_smem + kRsSeq * M;
  const int m0 = blockIdx.x * kRsSeq, j = blockIdx.y, s = blockIdx.z;
  const int nseq = min(kRsSeq, NA - m0);
  const double2* S = k.S + ((static_cast<int64_t>(s) * k.ny + j) * NA + m0) * nkp;
  // bin q of sequence e is item t = e * M + q; a thread loads kRsBatch items' operands, then stores
  const int items = nseq * M;
  for (int t0 = 0; t0 < items; t0 += kRsBatch * kRsThreads) {
    double2 w[kRsBatch], sq[kRsBatch], sc[kRsBatch];
#pragma unroll
    for (int u = 0; u < kRsBatch; ++u) {
      int q = min(t0 + u * kRsThreads + static_cast<int>(threadIdx.x), items - 1), e = 0;
#pragma unroll
      for (int i = 1; i < kRsSeq; ++i)
        if (q >= M) q -= M, ++e;
      w[u] = __ldg(k.f.tw + q);
      sq[u] = S[e * nkp + q];
      sc[u] = conj2(S[e * nkp + M - q]);
    }
#pragma unroll
    for (int u = 0; u < kRsBatch; ++u) {
      const int t = t0 + u * kRsThreads + threadIdx.x;
      if (t < items) {
        const double2 Ep = cadd(sq[u], sc[u]);
        const double2 Op = cmul(csub(sq[u], sc[u]), conj2(w[u]));
        a[t] = make_double2(Ep.x - Op.y, -(Ep.y + Op.x));  // conj(E' + i O')
      }
    }
  }
  __syncthreads();
  // the passes; the last one writes the row's samples straight out: element n is samples 2n (real part)
  // and 2n + 1 (minus the imaginary part), with no shared-memory round trip or barrier after it
  double* Fb = k.F + ((static_cast<int64_t>(s) * NA + m0) * k.ny + j) * k.nx;
  const int64_t fstride = static_cast<int64_t>(k.ny) * k.nx;  // between quantities
  const int nx = k.nx;
  auto to_row = [Fb, fstride, nx](int e, int n, double2 z) {
    double* Fe = Fb + e * fstride;
    if (2 * n < nx) Fe[2 * n] = z.x;
    if (2 * n + 1 < nx) Fe[2 * n + 1] = -z.y;
  };
  if constexpr (LC == 1440) {
    fft720(a, b, nseq, k.f, to_row);
    return;
  }
  const int np = k.f.nrad;
  int Ns = 1;
  for (int pass = 0; pass < np; ++pass) {
    const int R = k.f.rad[pass];
    const unsigned mg = k.f.magic[pass];
    const double2* src = a;
    auto from_smem = [src, M](int e, int n) { return src[e * M + n]; };
    if (pass == np - 1) {
      pass_io<true>(R, from_smem, to_row, M, Ns, mg, nseq, k.f.ptw + k.f.poff[pass]);
    } else {
      double2* dst = b;
      auto to_smem = [dst, M](int e, int n, double2 v) { dst[e * M + n] = v; };
      if (pass == 0 && R != 16)  // the first pass's twiddles are all 1: none are applied
        pass_io<false>(R, from_smem, to_smem, M, Ns, mg, nseq, k.f.ptw + k.f.poff[pass]);
      else
        pass_io<true>(R, from_smem, to_smem, M, Ns, mg, nseq, k.f.ptw + k.f.poff[pass]);
      __syncthreads();
      double2* t = a;
      a = b;
      b = t;
    }
    Ns *= R;
  }
}

template <int NA>
__global__ void __launch_bounds__(kRsThreads, kRsMinBlocks) rs_inverse_kernel(RsK k) {
  if (CGEF_RS_CT720 && is_fft720(k.f))
    inverse_body<NA, 1440>(k);
  else
    inverse_body<NA, 0>(k);
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
// w_a cos(2 pi q a / L) for a ring-closing row (its column -a) -- the real DFT of the row's weights laid
// out on the ring (w_|d| at d mod L for every visited d in [-a, hi]), taken like a source row's (a
// half-length Stockham FFT in shared memory, then the real split), kRsSeq rows per block.  O(L log L) a
// row instead of a cosine sum over every offset for every bin.
__global__ void __launch_bounds__(kRsThreads, kRsMinBlocks)
    rs_kspec_kernel(Fft f, const BandRow* rows, int64_t nrows, const double* w, double* kspec) {
  extern __shared__ double2 rs_smem[];
  const int M = f.M, L = f.L;
  double2* a = rs_smem;
  double2* b = rs_smem + kRsSeq * M;
  const int64_t r0 = static_cast<int64_t>(blockIdx.x) * kRsSeq;
  const int nseq = static_cast<int>(min(static_cast<int64_t>(kRsSeq), nrows - r0));
  double* ad = reinterpret_cast<double*>(a);
  for (int e = 0; e < nseq; ++e) {
    const BandRow br = rows[r0 + e];
    const double* wr = w + (br.a >= 0 ? br.woff : 0);
    for (int n = threadIdx.x; n < L; n += blockDim.x) {
      // every visited offset d in [-a, hi] lands on ring position d mod L (a footprint wider than a
      // periodic domain wraps it more than once)
      double x = 0.0;
      if (br.a >= 0) {
        for (int d = n; d <= br.hi; d += L) x += wr[d];
        for (int d = L - n; d <= br.a; d += L) x += wr[d];
      }
      ad[e * L + n] = x;
    }
  }
  __syncthreads();
  const double2* z = fft_block(a, b, nseq, f);
  const double inv_l = 1.0 / static_cast<double>(L);
  for (int t = threadIdx.x; t < nseq * f.nkp; t += blockDim.x) {
    const int e = t / f.nkp, q = t - e * f.nkp;
    double v = 0.0;
    if (q < f.nk) {
      const double2 zq = z[e * M + (q == M ? 0 : q)];
      const double2 zc = conj2(z[e * M + (q == 0 ? 0 : M - q)]);
      const double2 E = make_double2(0.5 * (zq.x + zc.x), 0.5 * (zq.y + zc.y));
      const double2 O = make_double2(0.5 * (zq.y - zc.y), -0.5 * (zq.x - zc.x));  // (zq - zc) / 2i
      v = cadd(E, cmul(__ldg(f.tw + q), O)).x * inv_l;
    }
    kspec[(r0 + e) * f.nkp + q] = v;
  }
}

int rs_check(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, what);
  count_launch();
  return CGEF_OK;
}

// The driver's tensor-map encoder, through the runtime (no link against the driver library); null
// when the driver does not provide it.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    else
      cudaGetLastError();
  });
  return fn;
}

// The accumulation's two tensor maps: the source spectra as doubles [slice row quantity][2 nkp] with
// 64 x NA boxes, and the kernel spectra as [target row][D + source row][bin] with 32 x 1 x kAccRows
// boxes (the target axis strides 2D table rows).  False where a map cannot be encoded.
bool rs_tma_maps(const RsK& k, int na, CUtensorMap* qm, CUtensorMap* km) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t nkp = static_cast<cuuint64_t>(k.f.nkp);
  const cuuint32_t one[3] = {1, 1, 1};
  const cuuint64_t qdim[2] = {2 * nkp, static_cast<cuuint64_t>(k.nslices) * k.ny * na};
  const cuuint64_t qstr[1] = {2 * nkp * sizeof(double)};
  const cuuint32_t qbox[2] = {64, static_cast<cuuint32_t>(na)};
  if (enc(qm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, static_cast<void*>(k.Q), qdim, qstr, qbox, one,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  const cuuint64_t kdim[3] = {nkp, static_cast<cuuint64_t>(k.ny + 2 * k.D), static_cast<cuuint64_t>(k.ny)};
  const cuuint64_t kstr[2] = {nkp * sizeof(double), static_cast<cuuint64_t>(2 * k.D) * nkp * sizeof(double)};
  const cuuint32_t kbox[3] = {32, 1, static_cast<cuuint32_t>(kAccRows)};
  return enc(km, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(k.kspec), kdim, kstr, kbox, one,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Opts a row-spectral kernel into `bytes` of dynamic shared memory (once per kernel and device): the
// FFT kernels' two L-point buffers, or the accumulation's pipeline stages.
int rs_smem_attr(const void* kernel, int bytes) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({kernel, dev})) return CGEF_OK;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(row-spectral FFT)");
  done.insert({kernel, dev});
  return CGEF_OK;
}

// The plan's transform description for the kernels.
Fft make_fft(const cgef_plan* p) {
  Fft f{};
  f.L = p->rs_L;
  f.M = p->rs_L / 2;
  f.nk = p->rs_nk;
  f.nkp = p->rs_nkp;
  f.nrad = p->rs_nrad;
  for (int i = 0, ns = 1; i < p->rs_nrad; ++i) {
    f.rad[i] = p->rs_rad[i];
    f.magic[i] = ns == 1 ? 0u : static_cast<unsigned>(((uint64_t(1) << 32) + ns - 1) / ns);
    f.poff[i] = p->rs_poff[i];
    ns *= p->rs_rad[i];
  }
  f.tw = reinterpret_cast<const double2*>(p->d_rs_tw);
  f.ptw = reinterpret_cast<const double2*>(p->d_rs_ptw);
  return f;
}

template <int MODE, int NF, bool DEF>
int run_rowspec(const cgef_plan* p, const BandedK& a, double* scratch, const RsShare& share, bool leave_raw,
                cudaStream_t st) {
  using C = Cfg<MODE, NF, DEF>;
  constexpr int NA = C::NA;
  constexpr int NC = (NA + kRsSeq - 1) / kRsSeq;
  RsK k{};
  k.f = make_fft(p);
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
  const size_t spec = static_cast<size_t>(a.nslices) * p->ny * NA * p->rs_nkp;
  // own scratch: [Q | S] with F over Q once S is formed; with shared source spectra: [F | S] and Q
  // outside, transformed here (keep) or by an earlier plan of the sweep (in)
  const bool shared = share.in != nullptr || share.keep != nullptr;
  k.Q = shared ? reinterpret_cast<double2*>(share.in ? const_cast<double*>(share.in) : share.keep)
               : reinterpret_cast<double2*>(scratch);
  k.S = reinterpret_cast<double2*>(scratch) + spec;
  k.F = scratch;
  const int smem = 2 * kRsSeq * static_cast<int>(sizeof(double2)) * (p->rs_L / 2);
  int rc;
  if ((rc = rs_smem_attr(reinterpret_cast<const void*>(rs_forward_kernel<MODE, NF, DEF>), kRsFftSmem)) != CGEF_OK)
    return rc;
  if ((rc = rs_smem_attr(reinterpret_cast<const void*>(rs_inverse_kernel<NA>), kRsFftSmem)) != CGEF_OK)
    return rc;
  prof_begin(CGEF_KERNEL_ROWSPEC, st);
  const dim3 rows(NC, p->ny, a.nslices);
  if (share.in == nullptr) {
    rs_forward_kernel<MODE, NF, DEF><<<rows, kRsThreads, smem, st>>>(k);
    rc = rs_check("rs_forward_kernel");
  }
  if (rc == CGEF_OK) {
    constexpr int RW = AccTile<NA>::RW;
    const int acc_smem = kAccStages * kAccRps * (NA * 32 * 16 + kAccRows * 32 * 8);
    const int tma_smem = kAccStages * kTmaRps * (NA * 32 * 16 + kAccRows * 32 * 8);
    const dim3 g(p->rs_nkp / 32, (p->ny + kAccRows - 1) / kAccRows, a.nslices);
    CUtensorMap qm, km;
    const bool tma = CGEF_ACC_TMA && k.band_stride != 0 && !k.periodic_y && k.D >= 1 && rs_tma_maps(k, NA, &qm, &km);
    if (tma) {
      rc = rs_smem_attr(reinterpret_cast<const void*>(rs_accumulate_tma_kernel<kAccRows, NA>), tma_smem);
      if (rc == CGEF_OK)
        rs_accumulate_tma_kernel<kAccRows, NA><<<g, 32 * (kAccRows / RW), tma_smem, st>>>(k, qm, km);
    } else {
      rc = rs_smem_attr(reinterpret_cast<const void*>(rs_accumulate_kernel<kAccRows, NA>), acc_smem);
      if (rc == CGEF_OK)
        rs_accumulate_kernel<kAccRows, NA><<<g, 32 * (kAccRows / RW), acc_smem, st>>>(k);
    }
    if (rc == CGEF_OK) rc = rs_check("rs_accumulate_kernel");
  }
  if (rc == CGEF_OK) {
    rs_inverse_kernel<NA><<<rows, kRsThreads, smem, st>>>(k);
    rc = rs_check("rs_inverse_kernel");
  }
  if (rc == CGEF_OK) {
    // A non-finite source value would reach every bin of its row's spectrum, so every target the row
    // feeds; the direct sum lets it reach only the targets whose footprint holds the cell.  The stage
    // flags such slices, and the direct gather sums them again here over the spectral sums (a launch
    // that finds no flag returns at once).
    double* partials = reinterpret_cast<double*>(reinterpret_cast<char*>(scratch) + rowspec_bytes(p, NA, a.nslices));
    GatherOut none{};
    none.slice_stride = a.out_stride;
    rc = launch_banded_nonfinite(p, MODE, NF, a.planes, a.pitch, static_cast<int>(a.slice_stride / a.plane_stride),
                                 a.nslices, a.mask, a.mask_stride, partials, none, st, scratch);
  }
  if (rc == CGEF_OK && !leave_raw) {
    rs_finish_kernel<MODE, NF, DEF><<<dim3((p->nx + 127) / 128, p->ny, a.nslices), 128, 0, st>>>(a, scratch);
    rc = rs_check("rs_finish_kernel");
  }
  prof_end(CGEF_KERNEL_ROWSPEC, st);
  return rc;
}

template <int MODE, int NF>
int dispatch_rowspec(bool def, const cgef_plan* p, const BandedK& a, double* scratch, const RsShare& share,
                     bool leave_raw, cudaStream_t st) {
  return def ? run_rowspec<MODE, NF, true>(p, a, scratch, share, leave_raw, st)
             : run_rowspec<MODE, NF, false>(p, a, scratch, share, leave_raw, st);
}

// Radices of a Stockham plan for M with few passes (tens, nines, then sixteens, eights, fours), or
// empty when M has a prime factor above 5.
std::vector<int> fft_radices(int M) {
  int e2 = 0, e3 = 0, e5 = 0;
  while (M % 2 == 0) M /= 2, ++e2;
  while (M % 3 == 0) M /= 3, ++e3;
  while (M % 5 == 0) M /= 5, ++e5;
  std::vector<int> rad;
  if (M != 1) return rad;
  for (; e5 > 0 && e2 > 0; --e5, --e2) rad.push_back(10);
  for (; e5 > 0; --e5) rad.push_back(5);
  for (; e3 >= 2; e3 -= 2) rad.push_back(9);
  if (e3 == 1) rad.push_back(3);
  for (; e2 >= 4; e2 -= 4) rad.push_back(16);
  if (e2 == 3) rad.push_back(8);
  if (e2 == 2) rad.push_back(4);
  if (e2 == 1) rad.push_back(2);
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

bool is_smooth(int n) { return n >= 1 && smooth_length(n) == n; }

// exp(-2 pi i n / L), n < L, as (re, im) pairs.
std::vector<double> roots_table(int L) {
  std::vector<double> tw(2 * static_cast<size_t>(L));
  for (int n = 0; n < L; ++n) {
    const double ang = 2.0 * 3.14159265358979323846 * (static_cast<double>(n) / L);
    tw[2 * n] = std::cos(ang);
    tw[2 * n + 1] = -std::sin(ang);
  }
  return tw;
}

// Per-pass twiddles of a Stockham plan with radices `rad` whose roots are those of `tw` (length L): pass
// p (Ns = the product of the earlier radices) multiplies element r of butterfly jm by exp(-2 pi i jm r /
// (Ns R)), entry jm r L / (Ns R) of tw; laid out [r - 1][jm] from poff[p].
std::vector<double> pass_twiddles(const std::vector<int>& rad, const std::vector<double>& tw, int L, int* poff) {
  std::vector<double> ptw;
  int ns = 1;
  for (size_t q = 0; q < rad.size(); ++q) {
    const int R = rad[q];
    poff[q] = static_cast<int>(ptw.size() / 2);
    for (int r = 1; r < R; ++r)
      for (int jm = 0; jm < ns; ++jm) {
        const int64_t n = static_cast<int64_t>(jm) * r * L / (static_cast<int64_t>(ns) * R);
        ptw.push_back(tw[2 * n]);
        ptw.push_back(tw[2 * n + 1]);
      }
    ns *= R;
  }
  return ptw;
}

// ---------------------------------------------------------------------------------------------------
// The spectral method (CGEF_ENGINE_SPECTRAL; ext/CoarseGrainingEnergyFluxesFFTWExt.jl:121-206): a
// 2-D real DFT as the row transforms above (L = nx), then per spectrum bin a complex DFT along y, the
// transfer function and the inverse along y (sp_column_kernel, in place), the inverse row transforms,
// and sp_finish_kernel.
// ---------------------------------------------------------------------------------------------------
constexpr int kSpThreads = 256;
constexpr int kSpMaxN = 4096;                 // longest y transform
constexpr int kSpSmemMax = 200 * 1024;        // shared memory the column kernel may use
constexpr int kSpSmemTarget = 96 * 1024;      // what it aims for (two blocks an SM)

struct SpK {
  double2* Q;       // [slice][row][m][bin]: the rows' spectra in, the filtered spectra out
  const double* T;  // transfer / (nx ny): [ky row][nkp]
  int ny, na, nk, nkp, cb;
  int nrad;
  int rad[16];
  unsigned magic[16];
  int poff[16];
  const double2* ptw;
};

// One Stockham pass (as stockham_pass) of a length-n complex FFT over nseq sequences `ss` elements apart.
template <int R>
__device__ __forceinline__ void col_pass(const double2* a, double2* b, int n, int ss, int Ns, unsigned ns_magic,
                                         int nseq, const double2* ptw) {
  const int nb = n / R;
  for (int t = threadIdx.x; t < nseq * nb; t += blockDim.x) {
    const int sq = t / nb, j = t - sq * nb;
    const double2* as = a + sq * ss;
    const int jq = Ns == 1 ? j : static_cast<int>(__umulhi(static_cast<unsigned>(j), ns_magic));
    const int jm = j - jq * Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = as[j + r * nb];
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], __ldg(ptw + (r - 1) * Ns + jm));
    dft<R>(v);
    double2* bs = b + sq * ss + jq * Ns * R + jm;
#pragma unroll
    for (int r = 0; r < R; ++r) bs[r * Ns] = v[r];
  }
}

// Forward DFTs of nseq length-ny sequences in `a` (shared memory, `ss` apart), `b` as scratch; returns
// the buffer holding them.  Every thread of the block must call it.
__device__ __forceinline__ double2* col_fft(double2* a, double2* b, int nseq, int ss, const SpK& k) {
  int Ns = 1;
  for (int p = 0; p < k.nrad; ++p) {
    const int R = k.rad[p];
    const unsigned mg = k.magic[p];
    const double2* tp = k.ptw + k.poff[p];
    switch (R) {
      case 2: col_pass<2>(a, b, k.ny, ss, Ns, mg, nseq, tp); break;
      case 3: col_pass<3>(a, b, k.ny, ss, Ns, mg, nseq, tp); break;
      case 4: col_pass<4>(a, b, k.ny, ss, Ns, mg, nseq, tp); break;
      case 5: col_pass<5>(a, b, k.ny, ss, Ns, mg, nseq, tp); break;
      case 8: col_pass<8>(a, b, k.ny, ss, Ns, mg, nseq, tp); break;
      case 9: col_pass<9>(a, b, k.ny, ss, Ns, mg, nseq, tp); break;
      case 10: col_pass<10>(a, b, k.ny, ss, Ns, mg, nseq, tp); break;
      default: col_pass<16>(a, b, k.ny, ss, Ns, mg, nseq, tp); break;
    }
    __syncthreads();
    double2* t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

// One block per (cb bins, quantity, slice): the bins' columns of row spectra (coalesced: a row's cb
// bins are adjacent), DFT along y, times Ghat(|k|) / (nx ny), inverse DFT along y as conj(DFT(conj)),
// stored back in place.  Sequences sit ny + 1 elements apart in shared memory (no bank aliasing of the
// transposing loads and stores).
__global__ void __launch_bounds__(kSpThreads) sp_column_kernel(SpK k) {
  extern __shared__ double2 rs_smem[];
  const int q0 = blockIdx.x * k.cb, m = blockIdx.y, s = blockIdx.z;
  const int nseq = min(k.cb, k.nk - q0);
  const int ny = k.ny, ss = ny + 1;
  double2* a = rs_smem;
  double2* b = rs_smem + k.cb * ss;
  const int64_t rstride = static_cast<int64_t>(k.na) * k.nkp;
  double2* base = k.Q + static_cast<int64_t>(s) * ny * rstride + static_cast<int64_t>(m) * k.nkp + q0;
  for (int t = threadIdx.x; t < nseq * ny; t += blockDim.x) {
    const int r = t / nseq, e = t - r * nseq;
    a[e * ss + r] = base[r * rstride + e];
  }
  __syncthreads();
  double2* x = col_fft(a, b, nseq, ss, k);
  for (int t = threadIdx.x; t < nseq * ny; t += blockDim.x) {
    const int e = t / ny, r = t - e * ny;
    const double g = __ldg(k.T + static_cast<int64_t>(r) * k.nkp + q0 + e);
    const double2 v = x[e * ss + r];
    x[e * ss + r] = make_double2(v.x * g, -(v.y * g));  // conj(X g)
  }
  __syncthreads();
  double2* y = col_fft(x, x == a ? b : a, nseq, ss, k);
  for (int t = threadIdx.x; t < nseq * ny; t += blockDim.x) {
    const int r = t / nseq, e = t - r * nseq;
    const double2 v = y[e * ss + r];
    base[r * rstride + e] = make_double2(v.x, -v.y);
  }
}

struct SpFin {
  const double* F;  // [slice][m][row][nx], the filtered quantities
  int nx, ny, renorm;
  GatherOut go;
};

// Per cell: Deformable's renormalisation, 1 / filter(mask) where |filter(mask)| >= 0.01 and 0 elsewhere
// (FFTWExt.jl:163-173, 201), applied to every filtered quantity; the flux mode then forms
// tau_ij = (u_i u_j)bar - ubar_i ubar_j (Diagnostics.jl:525-535).  Every cell is written.
template <int MODE, int NF, bool DEF>
__global__ void __launch_bounds__(128) sp_finish_kernel(SpFin f) {
  using C = Cfg<MODE, NF, DEF>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, s = blockIdx.z;
  if (i >= f.nx) return;
  const int64_t plane = static_cast<int64_t>(f.ny) * f.nx;
  const int64_t pix = static_cast<int64_t>(j) * f.nx + i;
  const double* src = f.F + static_cast<int64_t>(s) * C::NA * plane + pix;
  double v[C::NA];
#pragma unroll
  for (int m = 0; m < C::NA; ++m) v[m] = src[m * plane];
  double ir = 1.0;
  if (DEF && f.renorm) {
    const double r = v[C::NA - 1];
    ir = fabs(r) >= 0.01 ? 1.0 / r : 0.0;
  }
  const int64_t o = static_cast<int64_t>(s) * f.go.slice_stride + pix;
  if constexpr (MODE == kModePiCart) {
    const double ub = v[0] * ir, vb = v[1] * ir;
    f.go.o[0][o] = ub;
    f.go.o[1][o] = vb;
    f.go.o[2][o] = v[2] * ir - ub * ub;
    f.go.o[3][o] = v[3] * ir - ub * vb;
    f.go.o[4][o] = v[4] * ir - vb * vb;
  } else {
#pragma unroll
    for (int m = 0; m < NF; ++m) f.go.o[m][o] = v[m] * ir;
  }
}

int sp_smem_attr() {
  static std::mutex mu;
  static std::set<int> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  std::lock_guard<std::mutex> lock(mu);
  if (done.count(dev)) return CGEF_OK;
  cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(sp_column_kernel),
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSpSmemMax);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(spectral column kernel)");
  done.insert(dev);
  return CGEF_OK;
}

// Bins a column block takes: the most (16 at most) whose two buffers fit kSpSmemTarget, else one.
int spectral_cb(int ny) {
  for (int cb = 16; cb > 1; cb /= 2)
    if (2 * cb * (ny + 1) * static_cast<int>(sizeof(double2)) <= kSpSmemTarget) return cb;
  return 1;
}

template <int MODE, int NF, bool DEF>
int run_spectral(const cgef_plan* p, const double* planes, int pitch, int np, int nbatch, bool renorm, double* scratch,
                 const GatherOut& go, cudaStream_t st) {
  using C = Cfg<MODE, NF, DEF>;
  constexpr int NA = C::NA;
  constexpr int NC = (NA + kRsSeq - 1) / kRsSeq;
  RsK k{};
  k.f = make_fft(p);
  k.planes = planes;
  k.plane_stride = static_cast<int64_t>(p->ny) * pitch;
  k.slice_stride = np * k.plane_stride;
  k.pitch = pitch;
  k.halo = p->H;
  k.nx = p->nx;
  k.ny = p->ny;
  k.periodic_y = 1;
  k.nslices = nbatch;
  const size_t spec = static_cast<size_t>(nbatch) * p->ny * NA * p->rs_nkp;  // complex bins
  k.Q = reinterpret_cast<double2*>(scratch);
  k.S = k.Q;              // the column pass filters the row spectra in place
  k.F = scratch + 2 * spec;
  SpK c{};
  c.Q = k.Q;
  c.T = p->d_sp_T;
  c.ny = p->ny;
  c.na = NA;
  c.nk = p->rs_nk;
  c.nkp = p->rs_nkp;
  c.cb = spectral_cb(p->ny);
  c.nrad = p->sp_nrad;
  for (int i = 0, ns = 1; i < p->sp_nrad; ++i) {
    c.rad[i] = p->sp_rad[i];
    c.magic[i] = ns == 1 ? 0u : static_cast<unsigned>(((uint64_t(1) << 32) + ns - 1) / ns);
    c.poff[i] = p->sp_poff[i];
    ns *= p->sp_rad[i];
  }
  c.ptw = reinterpret_cast<const double2*>(p->d_sp_ptw);
  SpFin fin{};
  fin.F = k.F;
  fin.nx = p->nx;
  fin.ny = p->ny;
  fin.renorm = renorm ? 1 : 0;
  fin.go = go;
  const int smem = 2 * kRsSeq * static_cast<int>(sizeof(double2)) * (p->rs_L / 2);
  const int csmem = 2 * c.cb * (p->ny + 1) * static_cast<int>(sizeof(double2));
  int rc;
  if ((rc = rs_smem_attr(reinterpret_cast<const void*>(rs_forward_kernel<MODE, NF, DEF>), kRsFftSmem)) != CGEF_OK)
    return rc;
  if ((rc = rs_smem_attr(reinterpret_cast<const void*>(rs_inverse_kernel<NA>), kRsFftSmem)) != CGEF_OK)
    return rc;
  if ((rc = sp_smem_attr()) != CGEF_OK) return rc;
  prof_begin(CGEF_KERNEL_ROWSPEC, st);
  const dim3 rows(NC, p->ny, nbatch);
  rs_forward_kernel<MODE, NF, DEF><<<rows, kRsThreads, smem, st>>>(k);
  rc = rs_check("rs_forward_kernel");
  if (rc == CGEF_OK) {
    sp_column_kernel<<<dim3((c.nk + c.cb - 1) / c.cb, NA, nbatch), kSpThreads, csmem, st>>>(c);
    rc = rs_check("sp_column_kernel");
  }
  if (rc == CGEF_OK) {
    rs_inverse_kernel<NA><<<rows, kRsThreads, smem, st>>>(k);
    rc = rs_check("rs_inverse_kernel");
  }
  if (rc == CGEF_OK) {
    sp_finish_kernel<MODE, NF, DEF><<<dim3((p->nx + 127) / 128, p->ny, nbatch), 128, 0, st>>>(fin);
    rc = rs_check("sp_finish_kernel");
  }
  prof_end(CGEF_KERNEL_ROWSPEC, st);
  return rc;
}

}  // namespace

int launch_rowspec(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                   const uint8_t* mask, int64_t mask_slice_stride, double* scratch, const GatherOut& out,
                   cudaStream_t st, const RsShare& share, bool leave_raw) {
  if (!p->rs_on || p->d_rs_k == nullptr) return fail(CGEF_EINVAL, "row-spectral evaluation not built for this plan");
  if (scratch == nullptr) return fail(CGEF_EINVAL, "row-spectral evaluation needs its scratch buffer");
  const bool def = p->strategy == CGEF_DEFORMABLE;
  const BandedK a = make_banded_args(p, mode, planes, pitch, np, nbatch, mask, mask_slice_stride, out);
  const bool raw = leave_raw && mode != kModeFields;
  if (mode == kModePiSphere) return dispatch_rowspec<kModePiSphere, 1>(def, p, a, scratch, share, raw, st);
  if (mode == kModePiCart) return dispatch_rowspec<kModePiCart, 1>(def, p, a, scratch, share, raw, st);
  switch (nf) {
    case 1: return dispatch_rowspec<kModeFields, 1>(def, p, a, scratch, share, raw, st);
    case 2: return dispatch_rowspec<kModeFields, 2>(def, p, a, scratch, share, raw, st);
    case 3: return dispatch_rowspec<kModeFields, 3>(def, p, a, scratch, share, raw, st);
    case 4: return dispatch_rowspec<kModeFields, 4>(def, p, a, scratch, share, raw, st);
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
  const int nkp = (nk + 31) / 32 * 32;
  const int64_t nrows = static_cast<int64_t>(p->h_rows.size());
  const size_t kbytes = sizeof(double) * static_cast<size_t>(nrows) * nkp;
  if (kbytes > (size_t(8) << 30)) return CGEF_OK;

  const std::vector<double> tw = roots_table(L);
  // per-pass twiddles of the half-length transform
  int poff[16] = {};
  const std::vector<double> ptw = pass_twiddles(rad, tw, L, poff);
  DeviceGuard dg(p->device);
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p->d_rs_tw), tw.size() * sizeof(double));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(row-spectral twiddles)");
  e = cudaMemcpy(p->d_rs_tw, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(row-spectral twiddles)");
  e = cudaMalloc(reinterpret_cast<void**>(&p->d_rs_ptw), std::max<size_t>(ptw.size(), 2) * sizeof(double));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(row-spectral pass twiddles)");
  e = cudaMemcpy(p->d_rs_ptw, ptw.data(), ptw.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(row-spectral pass twiddles)");
  for (size_t q = 0; q < rad.size(); ++q) p->rs_poff[q] = poff[q];
  e = cudaMalloc(reinterpret_cast<void**>(&p->d_rs_k), kbytes);
  if (e == cudaErrorMemoryAllocation) {
    // no room for the kernel spectra: the plan keeps the direct gather only
    cudaGetLastError();
    p->d_rs_k = nullptr;
    cudaFree(p->d_rs_tw);
    p->d_rs_tw = nullptr;
    cudaFree(p->d_rs_ptw);
    p->d_rs_ptw = nullptr;
    return CGEF_OK;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(row-spectral kernel spectra)");
  p->rs_L = L;
  p->rs_nk = nk;
  p->rs_nkp = nkp;
  p->rs_nrad = static_cast<int>(rad.size());
  for (size_t i = 0; i < rad.size(); ++i) p->rs_rad[i] = rad[i];
  int rc = rs_smem_attr(reinterpret_cast<const void*>(rs_kspec_kernel), kRsFftSmem);
  if (rc == CGEF_OK) {
    const int smem = 2 * kRsSeq * static_cast<int>(sizeof(double2)) * (L / 2);
    rs_kspec_kernel<<<static_cast<unsigned>((nrows + kRsSeq - 1) / kRsSeq), kRsThreads, smem>>>(
        make_fft(p), p->d_rows, nrows, p->d_w, p->d_rs_k);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaDeviceSynchronize()) != cudaSuccess)
      rc = cuda_fail(e, "rs_kspec_kernel");
    else
      count_launch();
  }
  if (rc != CGEF_OK) {
    p->rs_L = 0;
    return rc;
  }
  p->rs_on = true;
  return CGEF_OK;
}

int launch_spectral(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                    bool renorm, double* scratch, const GatherOut& out, cudaStream_t st) {
  if (p->engine != CGEF_ENGINE_SPECTRAL || p->d_sp_T == nullptr)
    return fail(CGEF_EINVAL, "spectral method not built for this plan");
  if (scratch == nullptr) return fail(CGEF_EINVAL, "spectral method needs its scratch buffer");
  const bool def = p->strategy == CGEF_DEFORMABLE;
  if (mode == kModePiCart)
    return def ? run_spectral<kModePiCart, 1, true>(p, planes, pitch, np, nbatch, renorm, scratch, out, st)
               : run_spectral<kModePiCart, 1, false>(p, planes, pitch, np, nbatch, renorm, scratch, out, st);
  if (mode != kModeFields) return fail(CGEF_EUNSUPPORTED, "the spectral method is defined on the plane only");
  switch (nf) {
    case 1: return def ? run_spectral<kModeFields, 1, true>(p, planes, pitch, np, nbatch, renorm, scratch, out, st)
                       : run_spectral<kModeFields, 1, false>(p, planes, pitch, np, nbatch, renorm, scratch, out, st);
    case 2: return def ? run_spectral<kModeFields, 2, true>(p, planes, pitch, np, nbatch, renorm, scratch, out, st)
                       : run_spectral<kModeFields, 2, false>(p, planes, pitch, np, nbatch, renorm, scratch, out, st);
    case 3: return def ? run_spectral<kModeFields, 3, true>(p, planes, pitch, np, nbatch, renorm, scratch, out, st)
                       : run_spectral<kModeFields, 3, false>(p, planes, pitch, np, nbatch, renorm, scratch, out, st);
    case 4: return def ? run_spectral<kModeFields, 4, true>(p, planes, pitch, np, nbatch, renorm, scratch, out, st)
                       : run_spectral<kModeFields, 4, false>(p, planes, pitch, np, nbatch, renorm, scratch, out, st);
    default: return fail(CGEF_EINVAL, "spectral method: 1..4 fields per pass");
  }
}

// FFTWExt.jl:121-181: the transforms' tables and Ghat(|k|, l) on the rfft grid (Kernels.jl:394-406;
// the top-hat's Bessel form, SpecialFunctionsExt.jl:10-17, through std::cyl_bessel_j), divided by
// nx ny so the unnormalised transforms there and back give the filter.
int build_spectral(cgef_plan* p) {
  const int nx = p->nx, ny = p->ny;
  if (nx % 2 != 0 || nx > kRsMaxL || ny > kSpMaxN || !is_smooth(nx / 2) || !is_smooth(ny))
    return fail(CGEF_EUNSUPPORTED, "the spectral method needs an even nx with nx / 2 and ny free of prime factors "
                                   "above 5, both at most 4096 (got nx = " + std::to_string(nx) +
                                   ", ny = " + std::to_string(ny) + ")");
  const std::vector<int> radx = fft_radices(nx / 2), rady = fft_radices(ny);
  if (radx.size() > 16 || rady.size() > 16) return fail(CGEF_EUNSUPPORTED, "spectral method: too many FFT passes");
  const int nk = nx / 2 + 1;
  const int nkp = (nk + 31) / 32 * 32;
  std::vector<double> T(static_cast<size_t>(ny) * nkp, 0.0);
  p->h_sp_T.assign(static_cast<size_t>(ny) * nk, 0.0);
  const double pi2 = 2.0 * 3.14159265358979323846;
  const double norm = 1.0 / (static_cast<double>(nx) * ny);
  for (int r = 0; r < ny; ++r) {
    const int mr = r < (ny + 1) / 2 ? r : r - ny;  // fftfreq order
    const double ky = pi2 * (static_cast<double>(mr) / (ny * p->dy));
    for (int q = 0; q < nk; ++q) {
      const double kx = pi2 * (static_cast<double>(q) / (nx * p->dx));
      const double k = std::sqrt(kx * kx + ky * ky);
      double g;
      if (p->kernel == CGEF_GAUSSIAN) {
        g = std::exp(-(k * k) * (p->scale * p->scale) / (4.0 * p->alpha));
      } else {
        const double x = k * (p->scale / 2.0);
        g = x == 0.0 ? 1.0 : 2.0 * std::cyl_bessel_j(1.0, x) / x;
      }
      p->h_sp_T[static_cast<size_t>(r) * nk + q] = g;
      T[static_cast<size_t>(r) * nkp + q] = g * norm;
    }
  }
  p->rs_L = nx;
  p->rs_nk = nk;
  p->rs_nkp = nkp;
  p->rs_nrad = static_cast<int>(radx.size());
  for (size_t i = 0; i < radx.size(); ++i) p->rs_rad[i] = radx[i];
  p->sp_nrad = static_cast<int>(rady.size());
  for (size_t i = 0; i < rady.size(); ++i) p->sp_rad[i] = rady[i];
  p->rs_on = false;
  if (p->device < 0) return CGEF_OK;
  const std::vector<double> twx = roots_table(nx), twy = roots_table(ny);
  const std::vector<double> ptwx = pass_twiddles(radx, twx, nx, p->rs_poff);
  const std::vector<double> ptwy = pass_twiddles(rady, twy, ny, p->sp_poff);
  DeviceGuard dg(p->device);
  auto put = [](double** dst, const std::vector<double>& v, const char* what) {
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(dst), std::max<size_t>(v.size(), 2) * sizeof(double));
    if (e == cudaSuccess && !v.empty())
      e = cudaMemcpy(*dst, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice);
    return e == cudaSuccess ? CGEF_OK : cuda_fail(e, what);
  };
  int rc;
  if ((rc = put(&p->d_rs_tw, twx, "spectral method: x roots")) != CGEF_OK) return rc;
  if ((rc = put(&p->d_rs_ptw, ptwx, "spectral method: x pass twiddles")) != CGEF_OK) return rc;
  if ((rc = put(&p->d_sp_ptw, ptwy, "spectral method: y pass twiddles")) != CGEF_OK) return rc;
  if ((rc = put(&p->d_sp_T, T, "spectral method: transfer function")) != CGEF_OK) return rc;
  return CGEF_OK;
}

}  // namespace cgef
