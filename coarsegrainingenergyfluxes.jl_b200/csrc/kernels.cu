// Device kernels of the coarse-graining path (sm_100a).
//
// stage      : raw u, v (or K fields) -> padded FP64 planes with a wrapped/zero halo; masked
//              values; planetary-Cartesian components on the sphere (Diagnostics.jl:555-573).
// banded     : the footprint direct sum (Filtering.jl:2550-2598) -- every CTA walks the source
//              rows of its target rows once, applying per-band weights staged in shared memory
//              to all fields and their products (formed on the fly) with FP64 FMA; the epilogue
//              normalises, forms tau = (u_i u_j)bar - ubar_i ubar_j in FP64 and rotates to the
//              local frame (Diagnostics.jl:596-650).
// separable  : row pass + column pass of the square-truncated Gaussian (Filtering.jl:1211-1280,
//              1472-1524).
// prefix     : exact top-hat by per-row prefix sums and interval sweeps (Filtering.jl:894-1078).
// strain     : ReduceInRun 3-node derivatives of ubar, vbar, curvature terms, Pi = -S:tau and
//              the area-weighted energy partial sums (Diagnostics.jl:652-699, 1086-1134).
//
// This file is compiled with --fmad=false: every product and sum outside the explicit fma()
// accumulations is rounded separately, as in the reference's Julia code.
#include <algorithm>
#include <cstdint>

#include "banded_common.cuh"
#include "cgef_internal.h"
#include "stencil.cuh"

#ifndef CGEF_BANDED_MINB
#define CGEF_BANDED_MINB 4
#endif
#ifndef CGEF_BANDED_MINB_SPHERE_PI
#define CGEF_BANDED_MINB_SPHERE_PI 3
#endif
#ifndef CGEF_BANDED_UNROLL
#define CGEF_BANDED_UNROLL 2
#endif

namespace cgef {

namespace {

// Resident CTAs per SM the banded gather is compiled for, and the unroll of its inner loop.  The
// sphere flux gather (nine accumulated quantities per row) gets the registers of three CTAs per SM:
// at four it spills its accumulators.
constexpr int kBandedMinBlocks = CGEF_BANDED_MINB;
constexpr int banded_min_blocks(int mode) { return mode == kModePiSphere ? CGEF_BANDED_MINB_SPHERE_PI : kBandedMinBlocks; }
constexpr int kBandedUnroll = CGEF_BANDED_UNROLL;

__device__ __forceinline__ int wrap(int a, int n) {
  int r = a % n;
  return r < 0 ? r + n : r;
}

// Column c of a source row as the halo would hold it: itself inside the row, wrapped on a periodic axis,
// -1 (a zero value) off a bounded one.
__device__ __forceinline__ int source_col(int c, int nx, int periodic) {
  if (c >= 0 && c < nx) return c;
  return periodic ? wrap(c, nx) : -1;
}

template <typename T>
__device__ __forceinline__ double ld(const void* p, int64_t k) {
  return static_cast<double>(static_cast<const T*>(p)[k]);
}

__device__ __forceinline__ double load_any(const void* p, int dtype, int64_t k) {
  return dtype == CGEF_F32 ? ld<float>(p, k) : ld<double>(p, k);
}

__device__ __forceinline__ void store_any(void* p, int dtype, int64_t k, double v) {
  if (dtype == CGEF_F32)
    static_cast<float*>(p)[k] = static_cast<float>(v);
  else
    static_cast<double*>(p)[k] = v;
}

// ------------------------------------------------------------------------------------------
// stage
// ------------------------------------------------------------------------------------------
struct StageK {
  const void* f[4];
  int nf;
  int dtype;
  const uint8_t* mask;
  int64_t mask_stride;
  int nx, ny, pitch, halo, np, periodic_x, with_mask;
  int64_t in_slice_stride;  // nx*ny
  int64_t plane_stride;     // ny*pitch
  int64_t slice_stride;     // np*plane_stride
  const double* sinlam;
  const double* coslam;
  const double* sinphi;
  const double* cosphi;
  double* planes;
  int* flags;          // nslices + 1 non-finite flags (zeroed before the launch)
  int nslices;
  int check_products;  // flux modes: a product of two staged values must be finite too
};

template <int MODE>
__global__ void stage_kernel(StageK a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int s = blockIdx.z;
  if (p >= a.pitch) return;
  int i = p - a.halo;
  bool inside = true;
  if (i < 0 || i >= a.nx) {
    if (a.periodic_x)
      i = wrap(i, a.nx);
    else
      inside = false;
  }
  double vals[4] = {0.0, 0.0, 0.0, 0.0};
  double mval = 0.0;
  if (inside) {
    const int64_t k = s * a.in_slice_stride + static_cast<int64_t>(j) * a.nx + i;
    // the cell's values load with its mask (one round trip of latency); a masked cell stages zeros
    const bool act = a.mask == nullptr || a.mask[s * a.mask_stride + static_cast<int64_t>(j) * a.nx + i] != 0;
    double f[4] = {0.0, 0.0, 0.0, 0.0};
    const int nl = MODE == kModePiSphere ? 2 : a.nf;
#pragma unroll
    for (int m = 0; m < 4; ++m)
      if (m < nl) f[m] = load_any(a.f[m], a.dtype, k);
    double sl = 0.0, cl = 0.0, sp = 0.0, cp = 0.0;
    if (MODE == kModePiSphere) sl = a.sinlam[i], cl = a.coslam[i], sp = a.sinphi[j], cp = a.cosphi[j];
    mval = act ? 1.0 : 0.0;
    if (act) {
      if (MODE == kModePiSphere) {
        const double u = f[0], v = f[1];
        vals[0] = -sl * u - sp * cl * v;
        vals[1] = cl * u - sp * sl * v;
        vals[2] = cp * v;
      } else {
        for (int m = 0; m < a.nf; ++m) vals[m] = f[m];
      }
      // an active non-finite value (or product, which the flux accumulates) flags the slice
      const int nv = MODE == kModePiSphere ? 3 : a.nf;
      bool bad = false;
      for (int m = 0; m < nv; ++m) {
        bad |= !isfinite(vals[m]);
        if (a.check_products)
          for (int n = m; n < nv; ++n) bad |= !isfinite(vals[m] * vals[n]);
      }
      if (bad) {
        a.flags[s] = 1;
        a.flags[a.nslices] = 1;
      }
    }
  }
  double* out = a.planes + s * a.slice_stride + static_cast<int64_t>(j) * a.pitch + p;
  const int nv = MODE == kModePiSphere ? 3 : a.nf;
  for (int m = 0; m < nv; ++m) out[m * a.plane_stride] = vals[m];
  if (a.with_mask) out[nv * a.plane_stride] = mval;
}

// ------------------------------------------------------------------------------------------
// banded gather
// ------------------------------------------------------------------------------------------

// One warp = one work item: 32 consecutive target columns (one per lane) x kRows target rows,
// summed over the item's source rows.  For each source row the warp stages, 32 columns at a time,
// the kRows rows' weights (zero outside each row's own interval) in its own shared-memory slab,
// then every lane streams its three (or K) staged values along the row and applies the kRows
// weights to all accumulated quantities with FP64 FMA.  Warps never wait for one another.
//
// PAIR: the weights of every row are even in the longitude offset (w(-d) = w(d)), so each lane adds
// the quantities of the mirrored source columns c + d and c - d first and applies each row's weight
// once per pair: per pair of columns (sphere) 6 DMUL + 6 DFMA + 3 DADD + R*NA DFMA instead of
// 12 DMUL + 2*R*NA DFMA.
// The centre column (d = 0) is its own mirror and a ring-closing row's +a column is its -a column on a
// periodic ring (the reference visits [-a, a-1]); both carry half weight, which is exact in FP64.
//
// SAFE: the slice holds a non-finite source value (the stage's flag).  A zero weight (a column inside a
// row's window but outside its disk, or outside the row's own interval in the warp's shared column
// range) must not multiply it, so the warp skips zero weights -- the weight is the same for every
// lane, so the branch is uniform.  The fast gather skips flagged slices and the SAFE gather sums only
// them, so each slice is summed once.
template <int MODE, int NF, bool DEF, int R, bool PAIR, bool SAFE>
__device__ __forceinline__ void banded_unit(const BandedK& a, int64_t gid, double* wb, int (&ri)[3][R], int lane) {
  using C = Cfg<MODE, NF, DEF>;
  const int item_id = static_cast<int>(gid / a.nslices);
  const int slice = static_cast<int>(gid - static_cast<int64_t>(item_id) * a.nslices);
  if ((a.flags[slice] != 0) != SAFE) return;
  const WorkItem it = a.items[item_id];
  const int col = it.x0 + lane;
  const int j0 = it.j0;

  double acc[R][C::NA];
#pragma unroll
  for (int t = 0; t < R; ++t)
#pragma unroll
    for (int m = 0; m < C::NA; ++m) acc[t][m] = 0.0;

  // Inactive targets output 0 (Filtering.jl:2561): a warp with no active target skips the sums.
  bool any_act = false;
  if (col < a.nx) {
#pragma unroll
    for (int t = 0; t < R; ++t) {
      const int j = j0 + t;
      if (j < a.ny)
        any_act |= a.mask == nullptr || a.mask[slice * a.mask_stride + static_cast<int64_t>(j) * a.nx + col] != 0;
    }
  }
  const bool warp_act = __any_sync(0xffffffffu, any_act);

  const double* base = a.planes + slice * a.slice_stride + a.halo + col;
  for (int jr = it.jr0; warp_act && jr < it.jr1; ++jr) {
    int jj = jr;
    if (jr < 0 || jr >= a.ny) {
      if (!a.periodic_y) continue;
      jj = wrap(jr, a.ny);
    }
    // lanes 0..R-1 fetch the rows' intervals into the warp's slab
    if (lane < R) {
      int ra = -1, rhi = -1, roff = 0;
      const int j = j0 + lane;
      const int dj = jr - j;
      if (j < a.ny && dj >= -a.D && dj <= a.D) {
        const BandRow r = a.rows[static_cast<int64_t>(j) * a.band_stride + dj + a.D];
        ra = r.a;
        rhi = r.hi;
        roff = r.woff;
      }
      ri[0][lane] = ra;
      ri[1][lane] = rhi;
      ri[2][lane] = roff;
    }
    __syncwarp();
    int A = -1, HI = -1;
#pragma unroll
    for (int t = 0; t < R; ++t) {
      A = max(A, ri[0][t]);
      HI = max(HI, ri[1][t]);
    }
    if (A < 0) {
      __syncwarp();
      continue;
    }
    const double* src = base + static_cast<int64_t>(jj) * a.pitch;
    const double* rowp = src - col;  // column 0 of the source row (the SAFE gather indexes it itself)
    if constexpr (PAIR) {
      // offsets d = 0 .. A, the pair (c + d, c - d) per step
      for (int d0 = 0; d0 <= A; d0 += 32) {
        const int d = d0 + lane;
        double wv[R];
#pragma unroll
        for (int t = 0; t < R; ++t) {
          const int at = ri[0][t];
          double w = (at >= 0 && d <= at) ? __ldg(a.w + ri[2][t] + d) : 0.0;
          if (d == 0 || (d == at && ri[1][t] < at)) w *= 0.5;
          wv[t] = w;
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < R; ++t) wb[t * 32 + lane] = wv[t];
        __syncwarp();
        const int cn = min(32, A - d0 + 1);
        const double* sp = src + d0;
        const double* sm = src - d0;
#pragma unroll kBandedUnroll
        for (int kk = 0; kk < cn; ++kk) {
          double v1[C::NP], v2[C::NP];
          if constexpr (SAFE) {
            const int c1 = source_col(col + d0 + kk, a.nx, a.periodic_x);
            const int c2 = source_col(col - d0 - kk, a.nx, a.periodic_x);
#pragma unroll
            for (int pl = 0; pl < C::NP; ++pl) {
              v1[pl] = c1 >= 0 ? __ldg(rowp + pl * a.plane_stride + c1) : 0.0;
              v2[pl] = c2 >= 0 ? __ldg(rowp + pl * a.plane_stride + c2) : 0.0;
            }
          } else {
#pragma unroll
            for (int pl = 0; pl < C::NP; ++pl) {
              v1[pl] = __ldg(sp + pl * a.plane_stride + kk);
              v2[pl] = __ldg(sm + pl * a.plane_stride - kk);
            }
          }
          double q[C::NA];
          expand_pair<MODE, NF, DEF>(v1, v2, q);
#pragma unroll
          for (int t = 0; t < R; ++t) {
            const double wt = wb[t * 32 + kk];
            if (SAFE && wt == 0.0) continue;
#pragma unroll
            for (int m = 0; m < C::NA; ++m) acc[t][m] = fma(wt, q[m], acc[t][m]);
          }
        }
      }
    } else {
      for (int c0 = -A; c0 <= HI; c0 += 32) {
        const int k = c0 + lane;
        double wv[R];
#pragma unroll
        for (int t = 0; t < R; ++t) {
          const int at = ri[0][t];
          wv[t] = (at >= 0 && k >= -at && k <= ri[1][t]) ? __ldg(a.w + ri[2][t] + abs(k)) : 0.0;
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < R; ++t) wb[t * 32 + lane] = wv[t];
        __syncwarp();
        const int cn = min(32, HI - c0 + 1);
        const double* s = src + c0;
#pragma unroll kBandedUnroll
        for (int kk = 0; kk < cn; ++kk) {
          double v[C::NP];
          if constexpr (SAFE) {
            const int c = source_col(col + c0 + kk, a.nx, a.periodic_x);
#pragma unroll
            for (int pl = 0; pl < C::NP; ++pl) v[pl] = c >= 0 ? __ldg(rowp + pl * a.plane_stride + c) : 0.0;
          } else {
#pragma unroll
            for (int pl = 0; pl < C::NP; ++pl) v[pl] = __ldg(s + pl * a.plane_stride + kk);
          }
          double q[C::NA];
          expand<MODE, NF, DEF>(v, q);
#pragma unroll
          for (int t = 0; t < R; ++t) {
            const double wt = wb[t * 32 + kk];
            if (SAFE && wt == 0.0) continue;
#pragma unroll
            for (int m = 0; m < C::NA; ++m) acc[t][m] = fma(wt, q[m], acc[t][m]);
          }
        }
      }
    }
    __syncwarp();
  }

  if (it.slot >= 0) {
    // partial sums of a split tile: [slot][slice][t][m][lane]
    double* pp = a.partials + ((static_cast<int64_t>(it.slot) * a.nslices + slice) * R * C::NA) * 32 + lane;
#pragma unroll
    for (int t = 0; t < R; ++t)
#pragma unroll
      for (int m = 0; m < C::NA; ++m) pp[(t * C::NA + m) * 32] = acc[t][m];
    return;
  }
  if (col >= a.nx) return;
#pragma unroll
  for (int t = 0; t < R; ++t) {
    const int j = j0 + t;
    if (j >= a.ny) break;
    if (a.raw != nullptr)
      write_raw<MODE, NF, DEF>(a, acc[t], slice, j, col);
    else
      finish_target<MODE, NF, DEF>(a, acc[t], slice, j, col);
  }
}

// Takes the next unit of the launch's queue (one atomic per warp) and hands it to every lane.
__device__ __forceinline__ int64_t take_unit(unsigned long long* queue, int lane) {
  unsigned long long u = 0;
  if (lane == 0) u = atomicAdd(queue, 1ull);
  return static_cast<int64_t>(__shfl_sync(0xffffffffu, u, 0));
}

// A warp leaves after its last (empty) take; the last warp of the launch to leave zeroes the queue
// for the next launch.  Every warp's takes are fenced before its count, so none can follow the reset.
__device__ __forceinline__ void leave_queue(unsigned long long* queue, int lane) {
  if (lane != 0) return;
  const unsigned long long nwarps = static_cast<unsigned long long>(gridDim.x) * (blockDim.x >> 5);
  __threadfence();
  if (atomicAdd(queue + 1, 1ull) == nwarps - 1) {
    __threadfence();
    atomicExch(queue, 0ull);
    atomicExch(queue + 1, 0ull);
  }
}

// Persistent launch: at most as many warps as fit on the GPU at once, each taking (item, slice)
// units in the schedule's longest-first order until none is left, so no warp idles behind a slower
// sibling of its block while units remain.  Results do not depend on which warp takes a unit.
template <int MODE, int NF, bool DEF, int R, bool PAIR, bool SAFE>
__global__ void __launch_bounds__(32 * kWarps, banded_min_blocks(MODE)) banded_kernel(BandedK a) {
  __shared__ double wbuf[kWarps][R][32];
  __shared__ int rint[kWarps][3][R];  // per warp: a, hi, woff of the R rows for the current source row
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int64_t total = static_cast<int64_t>(a.nitems) * a.nslices;
  if (SAFE) {
    // the rare non-finite pass: a small grid striding over the units, no queue (no flagged slice: it
    // returns at once)
    if (a.flags[a.nslices] == 0) return;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kWarps;
    for (int64_t gid = static_cast<int64_t>(blockIdx.x) * kWarps + warp; gid < total; gid += stride) {
      banded_unit<MODE, NF, DEF, R, PAIR, SAFE>(a, gid, &wbuf[warp][0][0], rint[warp], lane);
      __syncwarp();
    }
    return;
  }
  for (int64_t gid = take_unit(a.queue, lane); gid < total; gid = take_unit(a.queue, lane)) {
    banded_unit<MODE, NF, DEF, R, PAIR, SAFE>(a, gid, &wbuf[warp][0][0], rint[warp], lane);
    __syncwarp();
  }
  leave_queue(a.queue, lane);
}

// One (split tile, slice, target row) of the combine pass: the slots added in slot order, then finished.
template <int MODE, int NF, bool DEF, int R, bool SAFE>
__device__ __forceinline__ void combine_group_row(const BandedK& a, int64_t gid, int lane) {
  using C = Cfg<MODE, NF, DEF>;
  constexpr int kAhead = 4;
  const int t = static_cast<int>(gid % R);
  const int64_t gs = gid / R;
  const int gi = static_cast<int>(gs / a.nslices);
  const int slice = static_cast<int>(gs - static_cast<int64_t>(gi) * a.nslices);
  if ((a.flags[slice] != 0) != SAFE) return;
  const SplitGroup g = a.groups[gi];
  const int col = g.x0 + lane;
  const int j = g.j0 + t;
  if (col >= a.nx || j >= a.ny) return;
  double acc[C::NA];
#pragma unroll
  for (int m = 0; m < C::NA; ++m) acc[m] = 0.0;
  const int64_t slot_stride = static_cast<int64_t>(a.nslices) * R * C::NA * 32;
  const double* p0 =
      a.partials + ((static_cast<int64_t>(g.slot0) * a.nslices + slice) * R * C::NA + t * C::NA) * 32 + lane;
  int q = 0;
  for (; q + kAhead <= g.nslots; q += kAhead) {
    double v[kAhead][C::NA];
#pragma unroll
    for (int u = 0; u < kAhead; ++u)
#pragma unroll
      for (int m = 0; m < C::NA; ++m) v[u][m] = p0[(q + u) * slot_stride + m * 32];
#pragma unroll
    for (int u = 0; u < kAhead; ++u)
#pragma unroll
      for (int m = 0; m < C::NA; ++m) acc[m] += v[u][m];
  }
  for (; q < g.nslots; ++q)
#pragma unroll
    for (int m = 0; m < C::NA; ++m) acc[m] += p0[q * slot_stride + m * 32];
  if (a.raw != nullptr)
    write_raw<MODE, NF, DEF>(a, acc, slice, j, col);
  else
    finish_target<MODE, NF, DEF>(a, acc, slice, j, col);
}

// Adds the partial slots of every split tile in slot order (deterministic) and finishes it: one warp
// per (tile, slice, target row).  The loads of four slots are in flight together; the additions stay
// in slot order.
template <int MODE, int NF, bool DEF, int R, bool SAFE>
__global__ void __launch_bounds__(128) banded_combine_kernel(BandedK a) {
  const int lane = threadIdx.x & 31;
  const int64_t total = static_cast<int64_t>(a.ngroups) * a.nslices * R;
  if (SAFE && a.flags[a.nslices] == 0) return;
  const int64_t stride = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t gid = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; gid < total; gid += stride)
    combine_group_row<MODE, NF, DEF, R, SAFE>(a, gid, lane);
}

// ------------------------------------------------------------------------------------------
// separable (Cartesian Gaussian)
// ------------------------------------------------------------------------------------------
struct SepK {
  const double* planes;
  int64_t plane_stride, slice_stride;
  int pitch, halo;
  const double* gx;
  const double* gy;
  const double* px;
  const double* py;
  int di_lim, dj_lim, periodic_y;
  int nx, ny;
  double* rowbuf;  // [slice][NA][ny][nx]
  int64_t rb_plane, rb_slice;
  const uint8_t* mask;
  int64_t mask_stride;
  double* out[9];
  int64_t out_stride;
};

template <int MODE, int NF, bool DEF>
__global__ void sep_row_kernel(SepK a) {
  using C = Cfg<MODE, NF, DEF>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int s = blockIdx.z;
  if (i >= a.nx) return;
  double acc[C::NA];
#pragma unroll
  for (int m = 0; m < C::NA; ++m) acc[m] = 0.0;
  const double* src = a.planes + s * a.slice_stride + static_cast<int64_t>(j) * a.pitch + a.halo + i;
  for (int k = -a.di_lim; k <= a.di_lim; ++k) {
    const double w = a.gx[k + a.di_lim];
    double v[C::NP];
#pragma unroll
    for (int pl = 0; pl < C::NP; ++pl) v[pl] = src[pl * a.plane_stride + k];
    double q[C::NA];
    expand<MODE, NF, DEF>(v, q);
#pragma unroll
    for (int m = 0; m < C::NA; ++m) acc[m] = fma(w, q[m], acc[m]);
  }
  double* o = a.rowbuf + s * a.rb_slice + static_cast<int64_t>(j) * a.nx + i;
#pragma unroll
  for (int m = 0; m < C::NA; ++m) o[m * a.rb_plane] = acc[m];
}

template <int MODE, int NF, bool DEF>
__global__ void sep_col_kernel(SepK a) {
  using C = Cfg<MODE, NF, DEF>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int s = blockIdx.z;
  if (i >= a.nx) return;
  double acc[C::NA];
#pragma unroll
  for (int m = 0; m < C::NA; ++m) acc[m] = 0.0;
  const double* rb = a.rowbuf + s * a.rb_slice + i;
  for (int k = -a.dj_lim; k <= a.dj_lim; ++k) {
    int jj = j + k;
    if (jj < 0 || jj >= a.ny) {
      if (!a.periodic_y) continue;
      jj = wrap(jj, a.ny);
    }
    const double w = a.gy[k + a.dj_lim];
#pragma unroll
    for (int m = 0; m < C::NA; ++m) acc[m] = fma(w, rb[m * a.rb_plane + static_cast<int64_t>(jj) * a.nx], acc[m]);
  }
  const int64_t pix = static_cast<int64_t>(j) * a.nx + i;
  const bool act = a.mask == nullptr || a.mask[s * a.mask_stride + pix] != 0;
  double F[C::NA0];
  bool zero = !act;
  if (DEF) {
    // invrenorm = 1/conv(mask), 0 where the local mass vanishes (Filtering.jl:1436-1445)
    const double den = acc[C::NA - 1];
    const double inv = den > kNormEps ? 1.0 / den : 0.0;
#pragma unroll
    for (int m = 0; m < C::NA0; ++m) F[m] = acc[m] * inv;
  } else {
    const double den = a.px[i] * a.py[j];
#pragma unroll
    for (int m = 0; m < C::NA0; ++m) F[m] = den > kNormEps ? acc[m] / den : 0.0;
  }
  if (zero) {
#pragma unroll
    for (int m = 0; m < C::NA0; ++m) F[m] = 0.0;
  }
  if (MODE == kModePiCart && !zero) {
    // masked cells output 0 before tau is formed (Filtering.jl:1521-1523), so tau there is 0
  }
  write_outputs<MODE, C::NA0>(a.out, s * a.out_stride + pix, F, MODE != kModeFields && zero, 0.0, 0.0, 0.0, 0.0);
}

// ------------------------------------------------------------------------------------------
// prefix-sum top-hat
// ------------------------------------------------------------------------------------------
struct PreK {
  const double* planes;
  int64_t plane_stride, slice_stride;
  int pitch, halo;
  int nx, ny, ne, nb, nslices;
  double wx;
  double* P;  // [slice][NA][ny][ne+1]
  int64_t P_plane, P_slice;
  const double* xe;
  const double* prefix_wx;
  const PrefixRow* rows;
  const double* x;
  double x0, dx;
  int nrep;
  const uint8_t* mask;
  int64_t mask_stride;
  double* out[9];
  int64_t out_stride;
  const double* sinlam;
  const double* coslam;
  const double* sinphi;
  const double* cosphi;
};

// One block per (slice, row) computes every quantity's running sum along the (tripled, for a periodic
// axis) row (prefixsum_fill_numerator_row!, Filtering.jl:894-907): the row's staged values are read into
// shared memory once (when they fit), and warp m scans quantity m -- each chunk of 32 columns forms the
// quantity of its cells (once per cell), takes a warp-wide inclusive scan of the terms (shuffles), adds the
// carried sum of the chunks before it and stores the 32 prefix values from consecutive lanes.  The terms
// and their order along the row are the reference's; only the grouping of the additions differs, so the
// sums agree with its sequential running sum to FP64 rounding.
template <int MODE, int NF, bool DEF>
__global__ void __launch_bounds__(320) prefix_scan_kernel(PreK a, int row_in_smem) {
  using C = Cfg<MODE, NF, DEF>;
  extern __shared__ double pre_row[];
  const int lane = threadIdx.x & 31;
  const int m = threadIdx.x >> 5;  // the warp's quantity
  const int j = blockIdx.x;
  const int s = blockIdx.y;
  const double* grow = a.planes + s * a.slice_stride + static_cast<int64_t>(j) * a.pitch + a.halo;
  const double* row = grow;
  int64_t pstride = a.plane_stride;
  if (row_in_smem) {
    for (int t = threadIdx.x; t < C::NP * a.nx; t += blockDim.x) {
      const int pl = t / a.nx, i = t - pl * a.nx;
      pre_row[t] = grow[pl * a.plane_stride + i];
    }
    __syncthreads();
    row = pre_row;
    pstride = a.nx;
  }
  if (m >= C::NA) return;
  double* P = a.P + s * a.P_slice + m * a.P_plane + static_cast<int64_t>(j) * (a.ne + 1);
  if (lane == 0) P[0] = 0.0;
  // kChunks chunks of 32 columns per iteration: their scans are independent, only the carry chains them
  constexpr int kChunks = 4;
  double carry = 0.0;
  for (int k0 = 0; k0 < a.ne; k0 += 32 * kChunks) {
    double x[kChunks];
#pragma unroll
    for (int c = 0; c < kChunks; ++c) {
      const int k = k0 + 32 * c + lane;
      x[c] = 0.0;
      if (k < a.ne) {
        const int i = k % a.nx;
        double v[C::NP];
#pragma unroll
        for (int pl = 0; pl < C::NP; ++pl) v[pl] = row[pl * pstride + i];
        x[c] = quantity<MODE, NF, DEF>(v, m) * a.wx;
      }
    }
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
#pragma unroll
      for (int c = 0; c < kChunks; ++c) {
        const double y = __shfl_up_sync(0xffffffffu, x[c], d);
        if (lane >= d) x[c] = x[c] + y;
      }
    }
#pragma unroll
    for (int c = 0; c < kChunks; ++c) {
      const int k = k0 + 32 * c + lane;
      x[c] = carry + x[c];
      if (k < a.ne) P[k + 1] = x[c];
      carry = __shfl_sync(0xffffffffu, x[c], 31);
    }
  }
}

__device__ __forceinline__ int lower_index(const double* xe, int ne, double xlo, int est) {
  int k = est < 0 ? 0 : (est > ne ? ne : est);
  while (k > 0 && xe[k - 1] >= xlo) --k;
  while (k < ne && xe[k] < xlo) ++k;
  return k;  // first k with xe[k] >= xlo (ne if none)
}

__device__ __forceinline__ int upper_index(const double* xe, int ne, double xhi, int est) {
  int h = est < -1 ? -1 : (est > ne - 1 ? ne - 1 : est);
  while (h + 1 < ne && xe[h + 1] <= xhi) ++h;
  while (h >= 0 && xe[h] > xhi) --h;
  return h;  // last h with xe[h] <= xhi (-1 if none)
}

template <int MODE, int NF, bool DEF>
__global__ void prefix_sweep_kernel(PreK a) {
  using C = Cfg<MODE, NF, DEF>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int s = blockIdx.z;
  if (i >= a.nx) return;
  double num[C::NA0];
#pragma unroll
  for (int m = 0; m < C::NA0; ++m) num[m] = 0.0;
  double den = 0.0;
  const double xc = a.x[i];
  const int off = a.nrep == 3 ? a.nx : 0;
  const int64_t pitchP = a.ne + 1;
  const double* Ps = a.P + s * a.P_slice;
  for (int b = 0; b < a.nb; ++b) {
    const PrefixRow pr = a.rows[static_cast<int64_t>(j) * a.nb + b];
    if (pr.mode == 0) continue;
    int lo, hi;
    if (pr.mode == 1) {
      lo = 0;
      hi = a.nx - 1;
    } else if (pr.mode == 2) {
      lo = i - pr.w < 0 ? 0 : i - pr.w;
      hi = i + pr.w > a.nx - 1 ? a.nx - 1 : i + pr.w;
    } else {
      const double xlo = xc - pr.hw, xhi = xc + pr.hw;
      const int est_lo = static_cast<int>(floor((xlo - a.x0) / a.dx)) + off;
      const int est_hi = static_cast<int>(floor((xhi - a.x0) / a.dx)) + off;
      lo = lower_index(a.xe, a.ne, xlo, est_lo);
      hi = upper_index(a.xe, a.ne, xhi, est_hi);
      if (hi < lo) continue;
    }
    const int64_t rbase = static_cast<int64_t>(pr.jj) * pitchP;
#pragma unroll
    for (int m = 0; m < C::NA0; ++m) {
      const double* Pr = Ps + m * a.P_plane + rbase;
      num[m] = num[m] + pr.wy * (Pr[hi + 1] - Pr[lo]);
    }
    double dd;
    if (DEF) {
      const double* Pd = Ps + (C::NA - 1) * a.P_plane + rbase;
      dd = Pd[hi + 1] - Pd[lo];
    } else {
      dd = a.prefix_wx[hi + 1] - a.prefix_wx[lo];
    }
    den = den + pr.wy * dd;
  }
  const int64_t pix = static_cast<int64_t>(j) * a.nx + i;
  const bool act = a.mask == nullptr || a.mask[s * a.mask_stride + pix] != 0;
  const bool zero = !act || !(den > kNormEps);
  double F[C::NA0];
#pragma unroll
  for (int m = 0; m < C::NA0; ++m) F[m] = zero ? 0.0 : num[m] / den;
  const double sl = a.sinlam ? a.sinlam[i] : 0.0, cl = a.coslam ? a.coslam[i] : 0.0;
  const double sp = a.sinphi ? a.sinphi[j] : 0.0, cp = a.cosphi ? a.cosphi[j] : 0.0;
  write_outputs<MODE, C::NA0>(a.out, s * a.out_stride + pix, F, zero, sl, cl, sp, cp);
}

// ------------------------------------------------------------------------------------------
// derivatives, strain, Pi, energy
// ------------------------------------------------------------------------------------------
__device__ double stencil(const Line& L, int p) {
  const int m1 = nb_index(p, -1, L.n, L.periodic), p1 = nb_index(p, 1, L.n, L.periodic);
  const bool am1 = act_at(L, m1), ap1 = act_at(L, p1);
  if (am1 && ap1) return (L.f[p1 * L.stride] - L.f[m1 * L.stride]) / (2.0 * L.h);
  if (ap1) {
    const int p2 = nb_index(p, 2, L.n, L.periodic);
    if (act_at(L, p2) && p2 != p)
      return (-3.0 * L.f[p * L.stride] + 4.0 * L.f[p1 * L.stride] - L.f[p2 * L.stride]) / (2.0 * L.h);
    return (L.f[p1 * L.stride] - L.f[p * L.stride]) / L.h;
  }
  if (am1) {
    const int m2 = nb_index(p, -2, L.n, L.periodic);
    if (act_at(L, m2) && m2 != p)
      return (3.0 * L.f[p * L.stride] - 4.0 * L.f[m1 * L.stride] + L.f[m2 * L.stride]) / (2.0 * L.h);
    return (L.f[p * L.stride] - L.f[m1 * L.stride]) / L.h;
  }
  return 0.0;
}

struct StrainK {
  const double* ub;
  const double* vb;
  const double* txx;
  const double* txy;
  const double* tyy;
  int64_t in_stride;
  const uint8_t* mask;
  int64_t mask_stride;
  int nx, ny, periodic_x, periodic_y, sphere, dtype;
  double dx, dy, yscale;
  const double* xscale;
  const double* tanfac;
  const double* area;
  void* pi;
  void* ub_o;
  void* vb_o;
  void* txx_o;
  void* txy_o;
  void* tyy_o;
  void* sxx_o;
  void* sxy_o;
  void* syy_o;
  int64_t out_stride;
  double* partials;  // [slice][block][2]
  // velocity-gradient planes (closure features): scale * (S_ee-form du/dx, du/dy, dv/dx + u t, dv/dy)
  float* grad;       // [slice][4][ny*nx] or nullptr
  int64_t grad_stride;
  double grad_scale;
  double* gpartials;  // [slice][block][2]: sum of |grad|^2 and active count
  // strain / convergence split of the flux (plane): total, strain, convergence, divergence, |strain|
  void* sc[5];
  // Row-spectral source (strain_kernel with RAW): the unnormalised footprint sums of the flux's
  // quantities, [slice][NA][ny][nx], finished here at each target and at its stencil neighbours with
  // the arithmetic of finish_target; ub, vb and the tau planes are then unused.
  const double* raw;
  const double* den_zf;  // ZeroFill denominator per row (periodic x) or per cell
  int den_zf_2d;
  const double* sinlam;
  const double* coslam;
  const double* sinphi;
  const double* cosphi;
};

#ifndef CGEF_STRAIN_BY
#define CGEF_STRAIN_BY 8
#endif
#ifndef CGEF_STRAIN_LEAN
#define CGEF_STRAIN_LEAN 1
#endif
constexpr int kStrainBX = 32, kStrainBY = CGEF_STRAIN_BY;

// Finishing of the raw sums: the normalisation of finish_target (inactive targets and denominators
// at or below kNormEps give 0), then the local-frame velocity of write_outputs.
template <int MODE, bool DEF>
struct RawFlux {
  static constexpr int NA0 = MODE == kModePiSphere ? 9 : 5;
  static constexpr int NA = NA0 + (DEF ? 1 : 0);
  static constexpr int NV = MODE == kModePiSphere ? 3 : 2;
};

// The raw sums one finished value needs at a cell, with its activity and denominator, loaded together:
// whether the cell is zero is decided after the loads, so a cell costs one round trip of memory latency
// (every cell of the raw planes is written, masked ones too).
template <int NQ>
struct RawCell {
  double F[NQ];
  double den;
  bool act;
};

template <int MODE, bool DEF, int NQ>
__device__ __forceinline__ void raw_load(const StrainK& a, const double* Fs, const uint8_t* mk, int j, int i,
                                         RawCell<NQ>& c) {
  const int64_t plane = static_cast<int64_t>(a.nx) * a.ny;
  const int64_t pix = static_cast<int64_t>(j) * a.nx + i;
  c.act = mk == nullptr || mk[pix] != 0;
  if (DEF)
    c.den = Fs[(RawFlux<MODE, DEF>::NA - 1) * plane + pix];
  else
    c.den = a.den_zf_2d ? a.den_zf[pix] : a.den_zf[j];
#pragma unroll
  for (int m = 0; m < NQ; ++m) c.F[m] = Fs[m * plane + pix];
}

// Finished local velocity at (j, i) from its loaded raw sums, and the reciprocal of its denominator
// (0 where the cell finishes to zero).
template <int MODE, bool DEF>
__device__ __forceinline__ void raw_velocity(const StrainK& a, const RawCell<RawFlux<MODE, DEF>::NV>& c, int j, int i,
                                             double& u, double& v, double& inv) {
  using R = RawFlux<MODE, DEF>;
  if (!c.act || !(c.den > kNormEps)) {
    u = 0.0;
    v = 0.0;
    inv = 0.0;
    return;
  }
  inv = 1.0 / c.den;
  double F[R::NV];
#pragma unroll
  for (int m = 0; m < R::NV; ++m) F[m] = c.F[m] * inv;
  if constexpr (MODE == kModePiSphere) {
    local_velocity(F[0], F[1], F[2], a.sinlam[i], a.coslam[i], a.sinphi[j], a.cosphi[j], u, v);
  } else {
    u = F[0];
    v = F[1];
  }
}

// Finished local stress at target (j, i) from its loaded raw sums and the reciprocal of its denominator
// that the tile's finishing computed (the same division of the same value); its velocity is the tile's.
template <int MODE, bool DEF>
__device__ __forceinline__ void raw_target(const StrainK& a, const RawCell<RawFlux<MODE, DEF>::NA0>& c, int j, int i,
                                           double inv, double& txx, double& txy, double& tyy) {
  using R = RawFlux<MODE, DEF>;
  if (!c.act || !(c.den > kNormEps)) {
    txx = txy = tyy = 0.0;
    return;
  }
  double F[R::NA0];
#pragma unroll
  for (int m = 0; m < R::NA0; ++m) F[m] = c.F[m] * inv;
  if constexpr (MODE == kModePiSphere) {
    local_tau_sphere(F, a.sinlam[i], a.coslam[i], a.sinphi[j], a.cosphi[j], txx, txy, tyy);
  } else {
    // Diagnostics.jl:525-527
    txx = F[2] - F[0] * F[0];
    txy = F[3] - F[0] * F[1];
    tyy = F[4] - F[1] * F[1];
  }
}

__device__ __forceinline__ void block_sum2(double& a, double& b, double* sh) {
  // deterministic: warp shuffles in a fixed tree, then warp results in order
  __syncthreads();  // sh may still be read by a previous call
  for (int off = 16; off > 0; off >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, off);
    b += __shfl_down_sync(0xffffffffu, b, off);
  }
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5, nw = (blockDim.x * blockDim.y) >> 5;
  if (lane == 0) {
    sh[2 * warp] = a;
    sh[2 * warp + 1] = b;
  }
  __syncthreads();
  if (tid == 0) {
    double sa = 0.0, sb = 0.0;
    for (int w = 0; w < nw; ++w) {
      sa += sh[2 * w];
      sb += sh[2 * w + 1];
    }
    a = sa;
    b = sb;
  }
}

// One block per 32 x 8 target tile: the filtered local velocity over the tile and a halo of kStrainHalo
// cells (the 3-node stencil's reach along either axis) is loaded once into shared memory -- from the
// finished planes of the direct engines (RAW false), or finished here from the row-spectral
// evaluation's raw sums (RAW true; MODE, DEF: the flux's quantities), the same values bit for bit, so
// that evaluation writes no finished planes.  The stencil cases come from the mask; the values they
// read come from the tile.
constexpr int kStrainHalo = 2;

// stencil_case() from the activity of the neighbours at -1, +1, -2 and +2 along the axis, as the tile
// holds them (0 off a bounded axis, the wrapped cell on a periodic one).  Equal to stencil_case() for
// axes of three or more cells (with two, a periodic cell's -1 and +1 neighbours are one cell, which
// makes the case centred or empty and never reads x2; with one, the derivative is 0 regardless).  Only
// the kind matters here: the values come from the tile by offset.
__device__ __forceinline__ StencilCase tile_case(unsigned char am1, unsigned char ap1, unsigned char am2,
                                                 unsigned char ap2) {
  StencilCase c{0, -1, -1, -1};
  if (am1 && ap1)
    c.kind = 1;
  else if (ap1)
    c.kind = ap2 ? 2 : 3;
  else if (am1)
    c.kind = am2 ? 4 : 5;
  return c;
}

template <bool RAW, int MODE, bool DEF, bool FULL = true>
__global__ void __launch_bounds__(kStrainBX * kStrainBY) strain_kernel(StrainK a) {
  constexpr int TW = kStrainBX + 2 * kStrainHalo, TH = kStrainBY + 2 * kStrainHalo;
  __shared__ double sh[2 * (kStrainBX * kStrainBY / 32)];
  __shared__ double tu[TH][TW];
  __shared__ double tv[TH][TW];
  __shared__ unsigned char tm[TH][TW];  // activity (0 off a bounded axis)
  __shared__ double ti[RAW ? TH : 1][RAW ? TW : 1];  // reciprocal denominators of the finished raw sums
  const int x0 = blockIdx.x * kStrainBX, y0 = blockIdx.y * kStrainBY;
  const int s = blockIdx.z;
  const uint8_t* mk = a.mask ? a.mask + s * a.mask_stride : nullptr;
  const double* ub = RAW ? nullptr : a.ub + s * a.in_stride;
  const double* vb = RAW ? nullptr : a.vb + s * a.in_stride;
  const double* Fs = RAW ? a.raw + s * static_cast<int64_t>(RawFlux<MODE, DEF>::NA) * a.nx * a.ny : nullptr;
  using R = RawFlux<MODE, DEF>;
  const int i = x0 + threadIdx.x;
  const int j = y0 + threadIdx.y;
  const bool target = i < a.nx && j < a.ny;
  const int64_t pix = static_cast<int64_t>(j) * a.nx + i;
  // the target's own loads first, so that they overlap the tile's
  RawCell<R::NA0> cen{};
  double ctxx = 0.0, ctxy = 0.0, ctyy = 0.0;
  if (target) {
    if (RAW) {
      raw_load<MODE, DEF, R::NA0>(a, Fs, mk, j, i, cen);
    } else {
      ctxx = a.txx ? a.txx[s * a.in_stride + pix] : 0.0;
      ctxy = a.txy ? a.txy[s * a.in_stride + pix] : 0.0;
      ctyy = a.tyy ? a.tyy[s * a.in_stride + pix] : 0.0;
    }
  }
  // the tile: every thread's cells are loaded before any of them is finished
  constexpr int kThreads = kStrainBX * kStrainBY, kPer = (TW * TH + kThreads - 1) / kThreads;
  const int tid = threadIdx.y * kStrainBX + threadIdx.x;
  RawCell<R::NV> rc[kPer];
  double lu[kPer], lv[kPer];
  int cj[kPer], ci[kPer];
  bool cin[kPer];
#pragma unroll
  for (int it = 0; it < kPer; ++it) {
    const int c = tid + it * kThreads;
    const int r = c / TW, q = c - r * TW;
    int jj = y0 - kStrainHalo + r, ii = x0 - kStrainHalo + q;
    bool inside = c < TW * TH;
    if (jj < 0 || jj >= a.ny) {
      if (a.periodic_y)
        jj = wrap(jj, a.ny);
      else
        inside = false;
    }
    if (ii < 0 || ii >= a.nx) {
      if (a.periodic_x)
        ii = wrap(ii, a.nx);
      else
        inside = false;
    }
    cj[it] = jj;
    ci[it] = ii;
    cin[it] = inside;
    rc[it].act = false;
    lu[it] = lv[it] = 0.0;
    if (inside) {
      if (RAW) {
        raw_load<MODE, DEF, R::NV>(a, Fs, mk, jj, ii, rc[it]);
      } else {
        const int64_t k = static_cast<int64_t>(jj) * a.nx + ii;
        rc[it].act = mk == nullptr || mk[k] != 0;
        lu[it] = ub[k];
        lv[it] = vb[k];
      }
    }
  }
#pragma unroll
  for (int it = 0; it < kPer; ++it) {
    const int c = tid + it * kThreads;
    if (c < TW * TH) {
      const int r = c / TW, q = c - r * TW;
      double u = lu[it], v = lv[it], inv = 0.0;
      if (RAW && cin[it]) raw_velocity<MODE, DEF>(a, rc[it], cj[it], ci[it], u, v, inv);
      if (RAW) ti[r][q] = inv;
      tu[r][q] = cin[it] ? u : 0.0;
      tv[r][q] = cin[it] ? v : 0.0;
      tm[r][q] = cin[it] && rc[it].act ? 1 : 0;
    }
  }
  __syncthreads();
  const int cx0 = threadIdx.x + kStrainHalo, cy0 = threadIdx.y + kStrainHalo;
  double e_num = 0.0, e_area = 0.0, g_sum = 0.0, g_cnt = 0.0;
  if (target) {
    const int64_t o = s * a.out_stride + pix;
    const bool act = mk == nullptr || mk[pix] != 0;
    double sxx = 0.0, sxy = 0.0, syy = 0.0, pi = 0.0;
    double g1 = 0.0, g2 = 0.0;  // du/dy and dv/dx + u t (the two halves of 2 S_en)
    const double u0 = tu[cy0][cx0], v0 = tv[cy0][cx0];
    double txx, txy, tyy;
    if (RAW) {
      raw_target<MODE, DEF>(a, cen, j, i, ti[cy0][cx0], txx, txy, tyy);
    } else {
      txx = ctxx;
      txy = ctxy;
      tyy = ctyy;
    }
    if (act) {
      const StencilCase cx = tile_case(tm[cy0][cx0 - 1], tm[cy0][cx0 + 1], tm[cy0][cx0 - 2], tm[cy0][cx0 + 2]);
      const StencilCase cy = tile_case(tm[cy0 - 1][cx0], tm[cy0 + 1][cx0], tm[cy0 - 2][cx0], tm[cy0 + 2][cx0]);
      const double xs = a.xscale[j];
      // the tile holds every neighbour a case reads: m1 and p1 at -1 and +1, x2 at +2 (forward) or -2
      const int dx2 = cx.kind == 2 ? 2 : -2, dy2 = cy.kind == 2 ? 2 : -2;
      const double dudx = a.nx < 2 ? 0.0
                                   : stencil_eval(cx, u0, tu[cy0][cx0 - 1], tu[cy0][cx0 + 1], tu[cy0][cx0 + dx2],
                                                  a.dx) * xs;
      const double dvdx = a.nx < 2 ? 0.0
                                   : stencil_eval(cx, v0, tv[cy0][cx0 - 1], tv[cy0][cx0 + 1], tv[cy0][cx0 + dx2],
                                                  a.dx) * xs;
      const double dudy = a.ny < 2 ? 0.0
                                   : stencil_eval(cy, u0, tu[cy0 - 1][cx0], tu[cy0 + 1][cx0], tu[cy0 + dy2][cx0],
                                                  a.dy) * a.yscale;
      const double dvdy = a.ny < 2 ? 0.0
                                   : stencil_eval(cy, v0, tv[cy0 - 1][cx0], tv[cy0 + 1][cx0], tv[cy0 + dy2][cx0],
                                                  a.dy) * a.yscale;
      sxx = dudx;
      syy = dvdy;
      if (a.sphere) {
        const double tf = a.tanfac[j];
        sxx -= v0 * tf;                          // S_ee = du/dx - v tan(phi)/R
        sxy = 0.5 * (dudy + dvdx + u0 * tf);     // S_en
        g1 = dudy;
        g2 = dvdx + u0 * tf;
      } else {
        sxy = 0.5 * (dudy + dvdx);
        g1 = dudy;
        g2 = dvdx;
      }
      pi = -(sxx * txx + 2.0 * sxy * txy + syy * tyy);
      const double ar = a.area[j];
      e_num = (u0 * u0 + v0 * v0) * ar;
      e_area = ar;
    }
    if (a.pi) store_any(a.pi, a.dtype, o, pi);
    if constexpr (FULL) {  // FULL false: Pi and E only (no intermediate fields, splits or closure features)
    if (a.ub_o) store_any(a.ub_o, a.dtype, o, u0);
    if (a.vb_o) store_any(a.vb_o, a.dtype, o, v0);
    if (a.txx_o) store_any(a.txx_o, a.dtype, o, txx);
    if (a.txy_o) store_any(a.txy_o, a.dtype, o, txy);
    if (a.tyy_o) store_any(a.tyy_o, a.dtype, o, tyy);
    if (a.sxx_o) store_any(a.sxx_o, a.dtype, o, sxx);
    if (a.sxy_o) store_any(a.sxy_o, a.dtype, o, sxy);
    if (a.syy_o) store_any(a.syy_o, a.dtype, o, syy);
    if (a.sc[0] || a.sc[1] || a.sc[2] || a.sc[3] || a.sc[4]) {
      // Diagnostics.jl:1757-1769 (Srinivasan, Barkan & McWilliams 2023, eq. 10)
      double d = 0.0, al = 0.0, pa = 0.0, pd = 0.0;
      if (act) {
        const double ux = sxx, vy = syy, uy = g1, vx = g2;
        d = ux + vy;
        al = sqrt((ux - vy) * (ux - vy) + (uy + vx) * (uy + vx));
        pa = (tyy - txx) * (ux - vy) / 2.0 - txy * (uy + vx);
        pd = (tyy + txx) * (ux + vy) / 2.0;
      }
      const double vals[5] = {pa - pd, pa, pd, d, al};
#pragma unroll
      for (int k = 0; k < 5; ++k)
        if (a.sc[k]) store_any(a.sc[k], a.dtype, o, vals[k]);
    }
    if (a.grad) {
      const double g[4] = {a.grad_scale * sxx, a.grad_scale * g1, a.grad_scale * g2, a.grad_scale * syy};
      float* gp = a.grad + s * a.grad_stride + pix;
      const int64_t N = static_cast<int64_t>(a.nx) * a.ny;
#pragma unroll
      for (int k = 0; k < 4; ++k) gp[k * N] = static_cast<float>(g[k]);
      if (act) {
        g_sum = g[0] * g[0] + g[1] * g[1] + g[2] * g[2] + g[3] * g[3];
        g_cnt = 1.0;
      }
    }
    }
  }
  if (FULL && a.gpartials) {
    block_sum2(g_sum, g_cnt, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      const int64_t nblk = static_cast<int64_t>(gridDim.x) * gridDim.y;
      const int64_t b = static_cast<int64_t>(blockIdx.y) * gridDim.x + blockIdx.x;
      a.gpartials[(s * nblk + b) * 2] = g_sum;
      a.gpartials[(s * nblk + b) * 2 + 1] = g_cnt;
    }
  }
  if (a.partials) {
    block_sum2(e_num, e_area, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      const int64_t nblk = static_cast<int64_t>(gridDim.x) * gridDim.y;
      const int64_t b = static_cast<int64_t>(blockIdx.y) * gridDim.x + blockIdx.x;
      a.partials[(s * nblk + b) * 2] = e_num;
      a.partials[(s * nblk + b) * 2 + 1] = e_area;
    }
  }
}

struct EnergyK {
  const double* ub;
  const double* vb;
  int64_t in_stride;
  const uint8_t* mask;
  int64_t mask_stride;
  int nx, ny;
  const double* area;
  double* partials;
};

__global__ void energy_partial_kernel(EnergyK a) {
  __shared__ double sh[2 * (kStrainBX * kStrainBY / 32)];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int s = blockIdx.z;
  double e_num = 0.0, e_area = 0.0;
  if (i < a.nx && j < a.ny) {
    const int64_t pix = static_cast<int64_t>(j) * a.nx + i;
    const bool act = a.mask == nullptr || a.mask[s * a.mask_stride + pix] != 0;
    if (act) {
      const double u0 = a.ub[s * a.in_stride + pix], v0 = a.vb[s * a.in_stride + pix];
      e_num = (u0 * u0 + v0 * v0) * a.area[j];
      e_area = a.area[j];
    }
  }
  block_sum2(e_num, e_area, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const int64_t nblk = static_cast<int64_t>(gridDim.x) * gridDim.y;
    const int64_t b = static_cast<int64_t>(blockIdx.y) * gridDim.x + blockIdx.x;
    a.partials[(s * nblk + b) * 2] = e_num;
    a.partials[(s * nblk + b) * 2 + 1] = e_area;
  }
}

// One block per slice: sums the block partials in a fixed order; out = factor * sum / weight
// (E = 1/2 sum / area with factor 1/2).  Thread t adds partials t, t + 256, ... in that order; its loads
// are issued eight at a time before any is added (a missing one adds an exact zero), so the sum costs a
// few round trips of memory latency instead of one per partial.
constexpr int kFinishThreads = 256, kFinishBatch = 8;
__global__ void __launch_bounds__(kFinishThreads) energy_finish_kernel(const double* partials, int64_t nblk,
                                                                       double* energy, int64_t estride, double factor) {
  __shared__ double sa[kFinishThreads], sb[kFinishThreads];
  const int s = blockIdx.x;
  double a = 0.0, b = 0.0;
  const double* ps = partials + s * nblk * 2;
  for (int64_t k0 = threadIdx.x; k0 < nblk; k0 += kFinishBatch * kFinishThreads) {
    double va[kFinishBatch], vb[kFinishBatch];
#pragma unroll
    for (int u = 0; u < kFinishBatch; ++u) {
      const int64_t k = k0 + static_cast<int64_t>(u) * kFinishThreads;
      va[u] = k < nblk ? ps[k * 2] : 0.0;
      vb[u] = k < nblk ? ps[k * 2 + 1] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kFinishBatch; ++u) {
      a += va[u];
      b += vb[u];
    }
  }
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (static_cast<int>(threadIdx.x) < w) {
      sa[threadIdx.x] += sa[threadIdx.x + w];
      sb[threadIdx.x] += sb[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) energy[s * estride] = sb[0] > 0.0 ? factor * sa[0] / sb[0] : 0.0;
}

struct DerivK {
  const void* f;
  void* out;
  int dtype;
  const uint8_t* mask;
  int nx, ny, periodic_x, periodic_y, axis;
  double dx, dy, yscale;
  const double* xscale;
  double* scratch;  // FP64 copy of f
};

__global__ void to_f64_kernel(const void* f, int dtype, double* out, int64_t n) {
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k < n) out[k] = load_any(f, dtype, k);
}

__global__ void derivative_kernel(DerivK a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.nx || j >= a.ny) return;
  const int64_t pix = static_cast<int64_t>(j) * a.nx + i;
  const bool act = a.mask == nullptr || a.mask[pix] != 0;
  double d = 0.0;
  if (act) {
    if (a.axis == 0) {
      Line L{a.scratch + static_cast<int64_t>(j) * a.nx, a.mask ? a.mask + static_cast<int64_t>(j) * a.nx : nullptr, 1,
             a.nx, a.periodic_x, a.dx};
      d = a.nx < 2 ? 0.0 : stencil(L, i) * a.xscale[j];
    } else {
      Line L{a.scratch + i, a.mask ? a.mask + i : nullptr, a.nx, a.ny, a.periodic_y, a.dy};
      d = a.ny < 2 ? 0.0 : stencil(L, j) * a.yscale;
    }
  }
  store_any(a.out, a.dtype, pix, d);
}

__global__ void convert_kernel(const double* src, int64_t src_stride, void* dst, int64_t dst_stride, int dtype,
                               int64_t n) {
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (k < n) store_any(dst, dtype, s * dst_stride + k, src[s * src_stride + k]);
}

inline int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, what);
  count_launch();
  return CGEF_OK;
}

}  // namespace

// ------------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------------
int launch_stage(const cgef_plan* p, int mode, const StageArgs& s, double* planes, int pitch, int halo, int np,
                 bool with_mask_plane, cudaStream_t st) {
  StageK a{};
  a.f[0] = s.a;
  a.f[1] = s.b;
  if (mode == kModeFields) {
    if (s.nf > 4) return fail(CGEF_EINVAL, "stage: at most 4 fields per pass");
    for (int m = 0; m < s.nf; ++m) a.f[m] = s.fields[m];
  }
  a.nf = mode == kModePiCart ? 2 : (mode == kModePiSphere ? 3 : s.nf);
  a.dtype = s.dtype;
  a.mask = s.mask;
  a.mask_stride = s.mask_slice_stride;
  a.nx = p->nx;
  a.ny = p->ny;
  a.pitch = pitch;
  a.halo = halo;
  a.np = np;
  a.periodic_x = p->periodic_x;
  a.with_mask = with_mask_plane ? 1 : 0;
  a.in_slice_stride = static_cast<int64_t>(p->nx) * p->ny;
  a.plane_stride = static_cast<int64_t>(p->ny) * pitch;
  a.slice_stride = np * a.plane_stride;
  a.sinlam = p->d_sinlam;
  a.coslam = p->d_coslam;
  a.sinphi = p->d_sinphi;
  a.cosphi = p->d_cosphi;
  a.planes = planes;
  a.flags = stage_flags(p, planes, np, pitch, s.nbatch);
  a.nslices = s.nbatch;
  a.check_products = mode != kModeFields;
  cudaError_t e = cudaMemsetAsync(a.flags, 0, sizeof(int) * (static_cast<size_t>(s.nbatch) + 1), st);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(stage flags)");
  dim3 block(256), grid((pitch + 255) / 256, p->ny, s.nbatch);
  prof_begin(CGEF_KERNEL_STAGE, st);
  if (mode == kModePiSphere)
    stage_kernel<kModePiSphere><<<grid, block, 0, st>>>(a);
  else
    stage_kernel<kModeFields><<<grid, block, 0, st>>>(a);
  prof_end(CGEF_KERNEL_STAGE, st);
  return check_launch("stage_kernel");
}

namespace {

// SMs of the current device (cached per device).
int sm_count() {
  static int cached[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  if (cached[dev] == 0) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) return 148;
    cached[dev] = sms;
  }
  return cached[dev];
}

// Blocks of one kernel instance that fit on the current device at once (cached per device).
template <typename K>
int64_t resident_blocks(K kernel) {
  static int64_t cached[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  if (cached[dev] == 0) {
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 32 * kWarps, 0) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || per_sm < 1 || sms < 1)
      return 1 << 20;
    cached[dev] = static_cast<int64_t>(per_sm) * sms;
  }
  return cached[dev];
}

// The gather (then the combine pass of split tiles) over the launch's slices: the fast gather over
// the unflagged ones (SAFE false, timed as the banded kind), or the zero-weight-skipping one over the
// slices the stage flagged as non-finite (SAFE true; returns at once when none is).
template <int MODE, int NF, bool DEF, int R, bool SAFE>
int run_banded(const BandedK& a, bool pair, cudaStream_t st) {
  const int64_t units = static_cast<int64_t>(a.nitems) * a.nslices;
  const int64_t need = (units + kWarps - 1) / kWarps;
  const int64_t cw = static_cast<int64_t>(a.ngroups) * a.nslices * R;
  int64_t cblocks = (cw + 3) / 4;
  if (SAFE) {
    // the non-finite pass strides over its units with two blocks per SM and no queue: launched on
    // every row-spectral evaluation, it mostly finds no flag and returns at once
    const int64_t small = 2 * static_cast<int64_t>(sm_count());
    if (pair) {
      banded_kernel<MODE, NF, DEF, R, true, true><<<static_cast<unsigned>(std::min(need, small)), 32 * kWarps, 0, st>>>(a);
    } else {
      banded_kernel<MODE, NF, DEF, R, false, true><<<static_cast<unsigned>(std::min(need, small)), 32 * kWarps, 0, st>>>(a);
    }
    cblocks = std::min(cblocks, small);
  } else {
    // the queue starts at zero even after a launch that stopped part-way (the kernel's last warp also
    // zeroes it on the way out)
    cudaError_t e = cudaMemsetAsync(a.queue, 0, 2 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(work queue)");
    prof_begin(CGEF_KERNEL_BANDED, st);
    if (pair) {
      const auto k = banded_kernel<MODE, NF, DEF, R, true, false>;
      k<<<static_cast<unsigned>(std::min(need, resident_blocks(k))), 32 * kWarps, 0, st>>>(a);
    } else {
      const auto k = banded_kernel<MODE, NF, DEF, R, false, false>;
      k<<<static_cast<unsigned>(std::min(need, resident_blocks(k))), 32 * kWarps, 0, st>>>(a);
    }
  }
  int rc = check_launch("banded_kernel");
  if (rc == CGEF_OK && a.ngroups > 0) {
    banded_combine_kernel<MODE, NF, DEF, R, SAFE><<<static_cast<unsigned>(cblocks), 128, 0, st>>>(a);
    rc = check_launch("banded_combine_kernel");
  }
  if (!SAFE) prof_end(CGEF_KERNEL_BANDED, st);
  return rc;
}

// The flux modes run kRows-row tiles only (taller tiles spill their accumulators); the filter
// passes also have kRowsTall-row tiles.
template <int MODE, int NF>
int dispatch_banded(bool def, int R, bool pair, const BandedK& a, cudaStream_t st) {
  if constexpr (MODE == kModeFields && NF + 1 <= kTallMaxQuantities) {
    if (R == kRowsTall)
      return def ? run_banded<MODE, NF, true, kRowsTall, false>(a, pair, st)
                 : run_banded<MODE, NF, false, kRowsTall, false>(a, pair, st);
  } else if constexpr (MODE == kModeFields && NF <= kTallMaxQuantities) {
    if (R == kRowsTall && !def) return run_banded<MODE, NF, false, kRowsTall, false>(a, pair, st);
  }
  return def ? run_banded<MODE, NF, true, kRows, false>(a, pair, st)
             : run_banded<MODE, NF, false, kRows, false>(a, pair, st);
}

// The zero-weight-skipping gather over the flagged slices: kRows-row tiles only.
template <int MODE, int NF>
int dispatch_banded_safe(bool def, bool pair, const BandedK& a, cudaStream_t st) {
  return def ? run_banded<MODE, NF, true, kRows, true>(a, pair, st)
             : run_banded<MODE, NF, false, kRows, true>(a, pair, st);
}

}  // namespace

int launch_banded(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                  const uint8_t* mask, int64_t mask_slice_stride, double* partials, const GatherOut& out,
                  cudaStream_t st, bool direct_only) {
  if (p->rs_on && !direct_only && nbatch <= 65535)  // grid z of the row-spectral kernels: one slice each
    return launch_rowspec(p, mode, nf, planes, pitch, np, nbatch, mask, mask_slice_stride, partials, out, st);
  return launch_banded_items(p, mode, nf, planes, pitch, np, nbatch, mask, mask_slice_stride, partials, nullptr, 0,
                             nullptr, 0, out, st);
}

namespace {

// Both gathers of a launch, or only the zero-weight-skipping one (safe_only, writing raw sums).
int banded_gathers(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                   const uint8_t* mask, int64_t mask_slice_stride, double* partials, const WorkItem* items, int nitems,
                   const SplitGroup* groups, int ngroups, const GatherOut& out, cudaStream_t st, bool safe_only,
                   double* raw) {
  const bool def = p->strategy == CGEF_DEFORMABLE;
  BandedK a = make_banded_args(p, mode, planes, pitch, np, nbatch, mask, mask_slice_stride, out);
  a.raw = raw;
  a.partials = partials;
  a.queue = p->d_queue;
  if (a.queue == nullptr) return fail(CGEF_EINVAL, "banded: the plan has no work queue");
  const int na = (mode == kModePiSphere ? 9 : (mode == kModePiCart ? 5 : nf)) + (def ? 1 : 0);
  const bool pair = p->paired;
  if (nf < 1 || nf > 4) return fail(CGEF_EINVAL, "banded: 1..4 fields per pass");
  int rc = CGEF_OK;
  if (!safe_only) {
    const Schedule& S = schedule_for(p, mode, na);
    const int R = items ? kRows : S.rows;
    a.items = items ? items : S.d_items;
    a.nitems = items ? nitems : static_cast<int>(S.h_items.size());
    a.groups = items ? groups : S.d_groups;
    a.ngroups = items ? ngroups : static_cast<int>(S.h_groups.size());
    if (a.nitems == 0) return CGEF_OK;
    if (a.ngroups > 0 && partials == nullptr) return fail(CGEF_EINVAL, "banded: split tiles need a partials buffer");
    if (mode == kModePiSphere) rc = dispatch_banded<kModePiSphere, 1>(def, R, pair, a, st);
    else if (mode == kModePiCart) rc = dispatch_banded<kModePiCart, 1>(def, R, pair, a, st);
    else if (nf == 1) rc = dispatch_banded<kModeFields, 1>(def, R, pair, a, st);
    else if (nf == 2) rc = dispatch_banded<kModeFields, 2>(def, R, pair, a, st);
    else if (nf == 3) rc = dispatch_banded<kModeFields, 3>(def, R, pair, a, st);
    else rc = dispatch_banded<kModeFields, 4>(def, R, pair, a, st);
    if (rc) return rc;
  }
  // the slices flagged as holding a non-finite value, with kRows-row tiles
  const Schedule& S0 = p->sched[0];
  a.items = items ? items : S0.d_items;
  a.nitems = items ? nitems : static_cast<int>(S0.h_items.size());
  a.groups = items ? groups : S0.d_groups;
  a.ngroups = items ? ngroups : static_cast<int>(S0.h_groups.size());
  if (a.nitems == 0) return CGEF_OK;
  if (a.ngroups > 0 && partials == nullptr) return fail(CGEF_EINVAL, "banded: split tiles need a partials buffer");
  if (mode == kModePiSphere) return dispatch_banded_safe<kModePiSphere, 1>(def, pair, a, st);
  if (mode == kModePiCart) return dispatch_banded_safe<kModePiCart, 1>(def, pair, a, st);
  switch (nf) {
    case 1: return dispatch_banded_safe<kModeFields, 1>(def, pair, a, st);
    case 2: return dispatch_banded_safe<kModeFields, 2>(def, pair, a, st);
    case 3: return dispatch_banded_safe<kModeFields, 3>(def, pair, a, st);
    default: return dispatch_banded_safe<kModeFields, 4>(def, pair, a, st);
  }
}

}  // namespace

int launch_banded_items(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                        const uint8_t* mask, int64_t mask_slice_stride, double* partials, const WorkItem* items,
                        int nitems, const SplitGroup* groups, int ngroups, const GatherOut& out, cudaStream_t st) {
  return banded_gathers(p, mode, mode == kModeFields ? nf : 1, planes, pitch, np, nbatch, mask, mask_slice_stride,
                        partials, items, nitems, groups, ngroups, out, st, false, nullptr);
}

int launch_banded_nonfinite(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                            const uint8_t* mask, int64_t mask_slice_stride, double* partials, const GatherOut& out,
                            cudaStream_t st, double* raw) {
  return banded_gathers(p, mode, mode == kModeFields ? nf : 1, planes, pitch, np, nbatch, mask, mask_slice_stride,
                        partials, nullptr, 0, nullptr, 0, out, st, true, raw);
}

namespace {

template <int MODE, int NF, bool DEF>
int run_sep(const SepK& a, int nbatch, int nx, int ny, cudaStream_t st) {
  dim3 block(128), grid((nx + 127) / 128, ny, nbatch);
  prof_begin(CGEF_KERNEL_SEPARABLE, st);
  sep_row_kernel<MODE, NF, DEF><<<grid, block, 0, st>>>(a);
  int rc = check_launch("sep_row_kernel");
  if (rc) return rc;
  sep_col_kernel<MODE, NF, DEF><<<grid, block, 0, st>>>(a);
  prof_end(CGEF_KERNEL_SEPARABLE, st);
  return check_launch("sep_col_kernel");
}

template <int MODE, int NF>
int dispatch_sep(bool def, const SepK& a, int nbatch, int nx, int ny, cudaStream_t st) {
  return def ? run_sep<MODE, NF, true>(a, nbatch, nx, ny, st) : run_sep<MODE, NF, false>(a, nbatch, nx, ny, st);
}

}  // namespace

int launch_separable(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                     const uint8_t* mask, int64_t mask_slice_stride, double* rowbuf, const GatherOut& out,
                     cudaStream_t st) {
  const bool def = p->strategy == CGEF_DEFORMABLE && (p->masked || mask_slice_stride != 0);
  SepK a{};
  a.planes = planes;
  a.plane_stride = static_cast<int64_t>(p->ny) * pitch;
  a.slice_stride = np * a.plane_stride;
  a.pitch = pitch;
  a.halo = p->H;
  a.gx = p->d_gx;
  a.gy = p->d_gy;
  a.px = p->d_px;
  a.py = p->d_py;
  a.di_lim = p->di_lim;
  a.dj_lim = p->sep_dj_lim;
  a.periodic_y = p->periodic_y;
  a.nx = p->nx;
  a.ny = p->ny;
  a.rowbuf = rowbuf;
  a.rb_plane = static_cast<int64_t>(p->nx) * p->ny;
  const int na = (mode == kModePiCart ? 5 : nf) + (def ? 1 : 0);
  a.rb_slice = na * a.rb_plane;
  a.mask = mask;
  a.mask_stride = mask_slice_stride;
  for (int m = 0; m < 9; ++m) a.out[m] = out.o[m];
  a.out_stride = out.slice_stride;
  if (mode == kModePiCart) return dispatch_sep<kModePiCart, 1>(def, a, nbatch, p->nx, p->ny, st);
  if (mode == kModePiSphere) return fail(CGEF_EUNSUPPORTED, "separable engine is Cartesian only (Filtering.jl:1149-1151)");
  switch (nf) {
    case 1: return dispatch_sep<kModeFields, 1>(def, a, nbatch, p->nx, p->ny, st);
    case 2: return dispatch_sep<kModeFields, 2>(def, a, nbatch, p->nx, p->ny, st);
    case 3: return dispatch_sep<kModeFields, 3>(def, a, nbatch, p->nx, p->ny, st);
    case 4: return dispatch_sep<kModeFields, 4>(def, a, nbatch, p->nx, p->ny, st);
    default: return fail(CGEF_EINVAL, "separable: 1..4 fields per pass");
  }
}

namespace {

template <int MODE, int NF, bool DEF>
int run_prefix(const PreK& a, int nbatch, int nx, int ny, cudaStream_t st) {
  using C = Cfg<MODE, NF, DEF>;
  // the row's staged values in shared memory when they fit (opted in once per device up to 200 KB)
  const size_t row_bytes = sizeof(double) * C::NP * static_cast<size_t>(nx);
  const bool in_smem = row_bytes <= (size_t(200) << 10);
  if (in_smem && row_bytes > (size_t(48) << 10)) {
    static int opted[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
    if (!opted[dev]) {
      cudaError_t e = cudaFuncSetAttribute(prefix_scan_kernel<MODE, NF, DEF>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, 200 << 10);
      if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(prefix_scan_kernel)");
      opted[dev] = 1;
    }
  }
  prof_begin(CGEF_KERNEL_PREFIX, st);
  prefix_scan_kernel<MODE, NF, DEF><<<dim3(ny, nbatch), 32 * C::NA, in_smem ? row_bytes : 0, st>>>(a, in_smem ? 1 : 0);
  int rc = check_launch("prefix_scan_kernel");
  if (rc) return rc;
  dim3 block(128), grid((nx + 127) / 128, ny, nbatch);
  prefix_sweep_kernel<MODE, NF, DEF><<<grid, block, 0, st>>>(a);
  prof_end(CGEF_KERNEL_PREFIX, st);
  return check_launch("prefix_sweep_kernel");
}

template <int MODE, int NF>
int dispatch_prefix(bool def, const PreK& a, int nbatch, int nx, int ny, cudaStream_t st) {
  return def ? run_prefix<MODE, NF, true>(a, nbatch, nx, ny, st) : run_prefix<MODE, NF, false>(a, nbatch, nx, ny, st);
}

}  // namespace

int launch_prefix(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                  const uint8_t* mask, int64_t mask_slice_stride, double* prefix, const GatherOut& out,
                  cudaStream_t st) {
  const bool def = p->strategy == CGEF_DEFORMABLE && (p->masked || mask_slice_stride != 0);
  PreK a{};
  a.planes = planes;
  a.plane_stride = static_cast<int64_t>(p->ny) * pitch;
  a.slice_stride = np * a.plane_stride;
  a.pitch = pitch;
  a.halo = p->H;
  a.nx = p->nx;
  a.ny = p->ny;
  a.ne = p->pre_ne;
  a.nb = p->pre_nb;
  a.nslices = nbatch;
  a.wx = p->dx;
  a.P = prefix;
  a.P_plane = static_cast<int64_t>(p->ny) * (p->pre_ne + 1);
  const int na = (mode == kModePiSphere ? 9 : (mode == kModePiCart ? 5 : nf)) + (def ? 1 : 0);
  a.P_slice = na * a.P_plane;
  a.xe = p->d_xe;
  a.prefix_wx = p->d_prefix_wx;
  a.rows = p->d_prows;
  a.x = p->d_x;
  a.x0 = p->x0;
  a.dx = p->dx;
  a.nrep = p->pre_nrep;
  a.mask = mask;
  a.mask_stride = mask_slice_stride;
  for (int m = 0; m < 9; ++m) a.out[m] = out.o[m];
  a.out_stride = out.slice_stride;
  const bool sph = mode == kModePiSphere;
  a.sinlam = sph ? p->d_sinlam : nullptr;
  a.coslam = sph ? p->d_coslam : nullptr;
  a.sinphi = sph ? p->d_sinphi : nullptr;
  a.cosphi = sph ? p->d_cosphi : nullptr;
  if (mode == kModePiSphere) return dispatch_prefix<kModePiSphere, 1>(def, a, nbatch, p->nx, p->ny, st);
  if (mode == kModePiCart) return dispatch_prefix<kModePiCart, 1>(def, a, nbatch, p->nx, p->ny, st);
  switch (nf) {
    case 1: return dispatch_prefix<kModeFields, 1>(def, a, nbatch, p->nx, p->ny, st);
    case 2: return dispatch_prefix<kModeFields, 2>(def, a, nbatch, p->nx, p->ny, st);
    case 3: return dispatch_prefix<kModeFields, 3>(def, a, nbatch, p->nx, p->ny, st);
    case 4: return dispatch_prefix<kModeFields, 4>(def, a, nbatch, p->nx, p->ny, st);
    default: return fail(CGEF_EINVAL, "prefix: 1..4 fields per pass");
  }
}

int launch_strain(const cgef_plan* p, const StrainArgs& s, cudaStream_t st) {
  StrainK a{};
  a.ub = s.ubar;
  a.vb = s.vbar;
  a.txx = s.txx;
  a.txy = s.txy;
  a.tyy = s.tyy;
  a.in_stride = s.in_slice_stride;
  a.mask = s.mask;
  a.mask_stride = s.mask_slice_stride;
  a.nx = p->nx;
  a.ny = p->ny;
  a.periodic_x = p->periodic_x;
  a.periodic_y = p->periodic_y;
  a.sphere = p->geometry == CGEF_SPHERICAL;
  a.dtype = s.dtype;
  a.dx = p->dx;
  a.dy = p->dy;
  a.yscale = p->geometry == CGEF_SPHERICAL ? 1.0 / p->R : 1.0;
  a.xscale = p->d_xscale;
  a.tanfac = p->d_tanfac;
  a.area = p->d_area;
  a.pi = s.pi;
  a.ub_o = s.ubar_o;
  a.vb_o = s.vbar_o;
  a.txx_o = s.txx_o;
  a.txy_o = s.txy_o;
  a.tyy_o = s.tyy_o;
  a.sxx_o = s.sxx_o;
  a.sxy_o = s.sxy_o;
  a.syy_o = s.syy_o;
  a.out_stride = s.out_slice_stride;
  a.partials = s.energy ? s.partials : nullptr;
  a.grad = s.grad;
  a.grad_stride = s.grad_slice_stride;
  a.grad_scale = s.grad_scale;
  a.gpartials = s.grad_mean ? s.grad_partials : nullptr;
  for (int k = 0; k < 5; ++k) a.sc[k] = s.sc[k];
  a.raw = s.raw;
  a.den_zf = p->d_den_zf;
  a.den_zf_2d = p->den_zf_2d;
  a.sinlam = p->d_sinlam;
  a.coslam = p->d_coslam;
  a.sinphi = p->d_sinphi;
  a.cosphi = p->d_cosphi;
  dim3 block(kStrainBX, kStrainBY), grid((p->nx + kStrainBX - 1) / kStrainBX, (p->ny + kStrainBY - 1) / kStrainBY,
                                         s.nbatch);
  const bool sph = p->geometry == CGEF_SPHERICAL, def = p->strategy == CGEF_DEFORMABLE;
  bool extra = a.ub_o || a.vb_o || a.txx_o || a.txy_o || a.tyy_o || a.sxx_o || a.sxy_o || a.syy_o || a.grad ||
               a.gpartials;
  for (int k = 0; k < 5; ++k) extra = extra || a.sc[k];
  const bool lean = CGEF_STRAIN_LEAN && s.raw != nullptr && !extra;
  prof_begin(CGEF_KERNEL_STRAIN, st);
  if (lean && sph)
    def ? strain_kernel<true, kModePiSphere, true, false><<<grid, block, 0, st>>>(a)
        : strain_kernel<true, kModePiSphere, false, false><<<grid, block, 0, st>>>(a);
  else if (lean)
    def ? strain_kernel<true, kModePiCart, true, false><<<grid, block, 0, st>>>(a)
        : strain_kernel<true, kModePiCart, false, false><<<grid, block, 0, st>>>(a);
  else if (s.raw == nullptr)
    strain_kernel<false, kModePiSphere, false><<<grid, block, 0, st>>>(a);
  else if (sph)
    def ? strain_kernel<true, kModePiSphere, true><<<grid, block, 0, st>>>(a)
        : strain_kernel<true, kModePiSphere, false><<<grid, block, 0, st>>>(a);
  else
    def ? strain_kernel<true, kModePiCart, true><<<grid, block, 0, st>>>(a)
        : strain_kernel<true, kModePiCart, false><<<grid, block, 0, st>>>(a);
  prof_end(CGEF_KERNEL_STRAIN, st);
  int rc = check_launch("strain_kernel");
  if (rc) return rc;
  const int64_t nblk = static_cast<int64_t>(grid.x) * grid.y;
  if (s.grad_mean) {
    energy_finish_kernel<<<s.nbatch, kFinishThreads, 0, st>>>(s.grad_partials, nblk, s.grad_mean, 1, 1.0);
    if ((rc = check_launch("energy_finish_kernel"))) return rc;
  }
  if (!s.energy) return CGEF_OK;
  energy_finish_kernel<<<s.nbatch, kFinishThreads, 0, st>>>(s.partials, nblk, s.energy, s.energy_stride, 0.5);
  return check_launch("energy_finish_kernel");
}

int64_t strain_tiles(const cgef_plan* p) {
  return static_cast<int64_t>((p->nx + kStrainBX - 1) / kStrainBX) * ((p->ny + kStrainBY - 1) / kStrainBY);
}

int launch_energy_finish(const double* partials, int64_t nblk, int nbatch, double* energy, int64_t energy_stride,
                         double factor, cudaStream_t st) {
  energy_finish_kernel<<<nbatch, kFinishThreads, 0, st>>>(partials, nblk, energy, energy_stride, factor);
  return check_launch("energy_finish_kernel");
}

int launch_energy(const cgef_plan* p, const double* ubar, const double* vbar, int64_t slice_stride,
                  const uint8_t* mask, int64_t mask_slice_stride, int nbatch, double* partials, double* energy,
                  int64_t energy_stride, cudaStream_t st) {
  EnergyK a{ubar, vbar, slice_stride, mask, mask_slice_stride, p->nx, p->ny, p->d_area, partials};
  dim3 block(kStrainBX, kStrainBY), grid((p->nx + kStrainBX - 1) / kStrainBX, (p->ny + kStrainBY - 1) / kStrainBY,
                                         nbatch);
  energy_partial_kernel<<<grid, block, 0, st>>>(a);
  int rc = check_launch("energy_partial_kernel");
  if (rc) return rc;
  const int64_t nblk = static_cast<int64_t>(grid.x) * grid.y;
  energy_finish_kernel<<<nbatch, kFinishThreads, 0, st>>>(partials, nblk, energy, energy_stride, 0.5);
  return check_launch("energy_finish_kernel");
}

int launch_derivative(const cgef_plan* p, int axis, int dtype, const void* f, void* out, cudaStream_t st) {
  const int64_t n = static_cast<int64_t>(p->nx) * p->ny;
  void* scratch = nullptr;
  int rc = ensure_ws(const_cast<cgef_plan*>(p), 7, n * sizeof(double), &scratch);
  if (rc) return rc;
  to_f64_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(f, dtype, static_cast<double*>(scratch), n);
  if ((rc = check_launch("to_f64_kernel"))) return rc;
  DerivK a{f, out, dtype, p->d_mask, p->nx, p->ny, p->periodic_x, p->periodic_y, axis, p->dx, p->dy,
           p->geometry == CGEF_SPHERICAL ? 1.0 / p->R : 1.0, p->d_xscale, static_cast<double*>(scratch)};
  dim3 block(kStrainBX, kStrainBY), grid((p->nx + kStrainBX - 1) / kStrainBX, (p->ny + kStrainBY - 1) / kStrainBY);
  derivative_kernel<<<grid, block, 0, st>>>(a);
  return check_launch("derivative_kernel");
}

int launch_convert(const double* src, int64_t src_stride, void* dst, int64_t dst_stride, int dtype, int64_t n,
                   int nbatch, cudaStream_t st) {
  dim3 grid(static_cast<unsigned>((n + 255) / 256), nbatch);
  convert_kernel<<<grid, 256, 0, st>>>(src, src_stride, dst, dst_stride, dtype, n);
  return check_launch("convert_kernel");
}

}  // namespace cgef
