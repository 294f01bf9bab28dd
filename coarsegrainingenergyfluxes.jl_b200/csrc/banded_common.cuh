// Device code shared by the direct banded gather and the row-spectral evaluation of the same
// footprint sums: the per-mode quantity layout, the launch arguments, the expansion of staged
// values into accumulated quantities, and the normalising epilogue.
#pragma once

#include <cstdint>

#include "cgef_internal.h"

namespace cgef {
namespace {

template <int MODE, int NF, bool DEF>
struct Cfg {
  static constexpr int NV = MODE == kModePiSphere ? 3 : (MODE == kModePiCart ? 2 : NF);
  static constexpr int NA0 = MODE == kModePiSphere ? 9 : (MODE == kModePiCart ? 5 : NF);
  static constexpr int NA = NA0 + (DEF ? 1 : 0);
  static constexpr int NP = NV + (DEF ? 1 : 0);
};

struct BandedK {
  const double* planes;
  int64_t plane_stride, slice_stride;
  int pitch, halo;
  const BandRow* rows;
  int band_stride;  // 2D+1 on the sphere (one band per row), 0 on the plane
  const double* w;
  int D;
  const WorkItem* items;
  int nitems;
  int nslices;
  const SplitGroup* groups;
  int ngroups;
  double* partials;
  const double* den_zf;
  int den_zf_2d;
  const uint8_t* mask;
  int64_t mask_stride;
  int nx, ny, periodic_y;
  int periodic_x;  // the zero-weight-skipping gather wraps (or zeroes) its own columns: it needs no halo
  const double* sinlam;
  const double* coslam;
  const double* sinphi;
  const double* cosphi;
  double* out[9];
  int64_t out_stride;
  unsigned long long* queue;  // [next unit, warps finished]; zero when a launch starts
  // The stage's non-finite flags (nslices + 1, the last set when any is; stage_flags): the fast gather
  // skips flagged slices, the zero-weight-skipping gather sums only them.
  const int* flags;
  // nullptr, or the unnormalised sums [slice][NA][ny][nx] are written there instead of the finished
  // outputs (the row-spectral evaluation's layout, which its epilogue then finishes).
  double* raw;
};

// Expands the staged values of one source cell into the accumulated quantities: the fields
// themselves, then (Pi modes) their pairwise products in the reference's order, then the mask.
template <int MODE, int NF, bool DEF>
__device__ __forceinline__ void expand(const double (&v)[Cfg<MODE, NF, DEF>::NP], double (&q)[Cfg<MODE, NF, DEF>::NA]) {
  using C = Cfg<MODE, NF, DEF>;
  if (MODE == kModePiSphere) {
    q[0] = v[0];
    q[1] = v[1];
    q[2] = v[2];
    q[3] = v[0] * v[0];
    q[4] = v[0] * v[1];
    q[5] = v[0] * v[2];
    q[6] = v[1] * v[1];
    q[7] = v[1] * v[2];
    q[8] = v[2] * v[2];
  } else if (MODE == kModePiCart) {
    q[0] = v[0];
    q[1] = v[1];
    q[2] = v[0] * v[0];
    q[3] = v[0] * v[1];
    q[4] = v[1] * v[1];
  } else {
#pragma unroll
    for (int m = 0; m < NF; ++m) q[m] = v[m];
  }
  if (DEF) q[C::NA - 1] = v[C::NP - 1];
}

// Accumulated quantity m of one source cell (the order of expand()): the fields, then (flux modes)
// their pairwise products, then the mask.
template <int MODE, int NF, bool DEF>
__device__ __forceinline__ double quantity(const double (&v)[Cfg<MODE, NF, DEF>::NP], int m) {
  using C = Cfg<MODE, NF, DEF>;
  if (DEF && m == C::NA - 1) return v[C::NP - 1];
  if constexpr (MODE == kModePiSphere) {
    switch (m) {
      case 0: return v[0];
      case 1: return v[1];
      case 2: return v[2];
      case 3: return v[0] * v[0];
      case 4: return v[0] * v[1];
      case 5: return v[0] * v[2];
      case 6: return v[1] * v[1];
      case 7: return v[1] * v[2];
      default: return v[2] * v[2];
    }
  } else if constexpr (MODE == kModePiCart) {
    switch (m) {
      case 0: return v[0];
      case 1: return v[1];
      case 2: return v[0] * v[0];
      case 3: return v[0] * v[1];
      default: return v[1] * v[1];
    }
  } else {
    double r = v[0];
#pragma unroll
    for (int f = 1; f < NF; ++f)
      if (m == f) r = v[f];
    return r;
  }
}

// The quantities of two mirrored source cells added together: sums of the fields, and each product
// of the first cell fused onto the rounded product of the second (one DMUL + one DFMA per product).
template <int MODE, int NF, bool DEF>
__device__ __forceinline__ void expand_pair(const double (&v)[Cfg<MODE, NF, DEF>::NP],
                                            const double (&u)[Cfg<MODE, NF, DEF>::NP],
                                            double (&q)[Cfg<MODE, NF, DEF>::NA]) {
  using C = Cfg<MODE, NF, DEF>;
  if (MODE == kModePiSphere) {
    q[0] = v[0] + u[0];
    q[1] = v[1] + u[1];
    q[2] = v[2] + u[2];
    q[3] = fma(v[0], v[0], u[0] * u[0]);
    q[4] = fma(v[0], v[1], u[0] * u[1]);
    q[5] = fma(v[0], v[2], u[0] * u[2]);
    q[6] = fma(v[1], v[1], u[1] * u[1]);
    q[7] = fma(v[1], v[2], u[1] * u[2]);
    q[8] = fma(v[2], v[2], u[2] * u[2]);
  } else if (MODE == kModePiCart) {
    q[0] = v[0] + u[0];
    q[1] = v[1] + u[1];
    q[2] = fma(v[0], v[0], u[0] * u[0]);
    q[3] = fma(v[0], v[1], u[0] * u[1]);
    q[4] = fma(v[1], v[1], u[1] * u[1]);
  } else {
#pragma unroll
    for (int m = 0; m < NF; ++m) q[m] = v[m] + u[m];
  }
  if (DEF) q[C::NA - 1] = v[C::NP - 1] + u[C::NP - 1];
}

// The local-frame filtered velocity from the planetary one (sphere, Diagnostics.jl:596-610): the
// east and north unit vectors e = (-sin lam, cos lam, 0), n = (-sin phi cos lam, -sin phi sin lam,
// cos phi).  Shared by every epilogue so all of them round alike.
__device__ __forceinline__ void local_velocity(double ub0, double ub1, double ub2, double sl, double cl, double sp,
                                               double cp, double& u, double& v) {
  const double e0 = -sl, e1 = cl, e2 = 0.0;
  const double n0 = -sp * cl, n1 = -sp * sl, n2 = cp;
  u = e0 * ub0 + e1 * ub1 + e2 * ub2;
  v = n0 * ub0 + n1 * ub1 + n2 * ub2;
}

// tau = (u_i u_j)bar - ubar_i ubar_j in the planetary frame, rotated to east/north (Diagnostics.jl:
// 612-650); F holds the normalised quantities of the sphere flux (3 velocities, 6 products).
__device__ __forceinline__ void local_tau_sphere(const double* F, double sl, double cl, double sp, double cp,
                                                 double& txx, double& txy, double& tyy) {
  const double ub0 = F[0], ub1 = F[1], ub2 = F[2];
  const double e0 = -sl, e1 = cl, e2 = 0.0;
  const double n0 = -sp * cl, n1 = -sp * sl, n2 = cp;
  const double t00 = F[3] - ub0 * ub0;
  const double t01 = F[4] - ub0 * ub1;
  const double t02 = F[5] - ub0 * ub2;
  const double t11 = F[6] - ub1 * ub1;
  const double t12 = F[7] - ub1 * ub2;
  const double t22 = F[8] - ub2 * ub2;
  const double te0 = t00 * e0 + t01 * e1 + t02 * e2;
  const double te1 = t01 * e0 + t11 * e1 + t12 * e2;
  const double te2 = t02 * e0 + t12 * e1 + t22 * e2;
  const double tn0 = t00 * n0 + t01 * n1 + t02 * n2;
  const double tn1 = t01 * n0 + t11 * n1 + t12 * n2;
  const double tn2 = t02 * n0 + t12 * n1 + t22 * n2;
  txx = e0 * te0 + e1 * te1 + e2 * te2;
  txy = e0 * tn0 + e1 * tn1 + e2 * tn2;
  tyy = n0 * tn0 + n1 * tn1 + n2 * tn2;
}

// Normalised epilogue shared by the direct-sum engines.  F holds the NA0 filtered quantities
// (already divided by the denominator); writes the mode's outputs at offset o.
template <int MODE, int NA0>
__device__ __forceinline__ void write_outputs(double* const (&out)[9], int64_t o, const double (&F)[NA0], bool zero,
                                              double sl, double cl, double sp, double cp) {
  if (MODE == kModeFields) {
#pragma unroll
    for (int m = 0; m < NA0; ++m) out[m][o] = zero ? 0.0 : F[m];
    return;
  }
  if (zero) {
#pragma unroll
    for (int m = 0; m < 5; ++m) out[m][o] = 0.0;
    return;
  }
  if (MODE == kModePiCart) {
    // Diagnostics.jl:525-527
    out[0][o] = F[0];
    out[1][o] = F[1];
    out[2][o] = F[2] - F[0] * F[0];
    out[3][o] = F[3] - F[0] * F[1];
    out[4][o] = F[4] - F[1] * F[1];
    return;
  }
  // Sphere (Diagnostics.jl:596-650): planetary ubar and tau, rotated to east/north.
  double u, v, txx, txy, tyy;
  local_velocity(F[0], F[1], F[2], sl, cl, sp, cp, u, v);
  local_tau_sphere(F, sl, cl, sp, cp, txx, txy, tyy);
  out[0][o] = u;
  out[1][o] = v;
  out[2][o] = txx;
  out[3][o] = txy;
  out[4][o] = tyy;
}

// Finishes one target (row t of a tile) from its accumulated sums: normalise, then write the
// mode's outputs.
template <int MODE, int NF, bool DEF>
__device__ __forceinline__ void finish_target(const BandedK& a, const double (&acc)[Cfg<MODE, NF, DEF>::NA], int slice,
                                              int j, int col) {
  using C = Cfg<MODE, NF, DEF>;
  const int64_t pix = static_cast<int64_t>(j) * a.nx + col;
  const bool act = a.mask == nullptr || a.mask[slice * a.mask_stride + pix] != 0;
  double den;
  if (DEF)
    den = acc[C::NA - 1];
  else
    den = a.den_zf_2d ? a.den_zf[pix] : a.den_zf[j];
  const bool zero = !act || !(den > kNormEps);
  // one reciprocal per target (every epilogue of the flux normalises this way, so they round alike)
  const double inv = 1.0 / den;
  double F[C::NA0];
#pragma unroll
  for (int m = 0; m < C::NA0; ++m) F[m] = zero ? 0.0 : acc[m] * inv;
  const double sl = a.sinlam ? a.sinlam[col] : 0.0;
  const double cl = a.coslam ? a.coslam[col] : 0.0;
  const double sp = a.sinphi ? a.sinphi[j] : 0.0;
  const double cp = a.cosphi ? a.cosphi[j] : 0.0;
  write_outputs<MODE, C::NA0>(a.out, slice * a.out_stride + pix, F, zero, sl, cl, sp, cp);
}

// Stores the unnormalised sums of one target where the row-spectral evaluation keeps its own.
template <int MODE, int NF, bool DEF>
__device__ __forceinline__ void write_raw(const BandedK& a, const double (&acc)[Cfg<MODE, NF, DEF>::NA], int slice,
                                          int j, int col) {
  using C = Cfg<MODE, NF, DEF>;
  const int64_t plane = static_cast<int64_t>(a.ny) * a.nx;
  double* r = a.raw + static_cast<int64_t>(slice) * C::NA * plane + static_cast<int64_t>(j) * a.nx + col;
#pragma unroll
  for (int m = 0; m < C::NA; ++m) r[m * plane] = acc[m];
}

// The launch arguments both evaluations share: staged planes, band tables and the epilogue's
// inputs and outputs (the direct gather adds its schedule, partials and queue).
inline BandedK make_banded_args(const cgef_plan* p, int mode, const double* planes, int pitch, int np, int nbatch,
                                const uint8_t* mask, int64_t mask_slice_stride, const GatherOut& out) {
  BandedK a{};
  a.planes = planes;
  a.plane_stride = static_cast<int64_t>(p->ny) * pitch;
  a.slice_stride = np * a.plane_stride;
  a.pitch = pitch;
  a.halo = p->H;
  a.rows = p->d_rows;
  a.band_stride = p->geometry == CGEF_SPHERICAL ? 2 * p->D + 1 : 0;
  a.w = p->d_w;
  a.D = p->D;
  a.nslices = nbatch;
  a.den_zf = p->d_den_zf;
  a.den_zf_2d = p->den_zf_2d;
  a.mask = mask;
  a.mask_stride = mask_slice_stride;
  a.nx = p->nx;
  a.ny = p->ny;
  a.periodic_y = p->periodic_y;
  a.periodic_x = p->periodic_x;
  const bool sph = mode == kModePiSphere;
  a.sinlam = sph ? p->d_sinlam : nullptr;
  a.coslam = sph ? p->d_coslam : nullptr;
  a.sinphi = sph ? p->d_sinphi : nullptr;
  a.cosphi = sph ? p->d_cosphi : nullptr;
  for (int m = 0; m < 9; ++m) a.out[m] = out.o[m];
  a.out_stride = out.slice_stride;
  a.flags = stage_flags(p, planes, np, pitch, nbatch);
  return a;
}

}  // namespace
}  // namespace cgef
