// The 2.5-D flux: compute_Π! with the vertical velocity w (Diagnostics.jl:254-260, 483-681).
//
// The velocity has three components -- (u, v, w) on the plane, the planetary (X, Y, Z) with w along the
// local up vector on the sphere -- and the flux filters them and their six products.  That is three
// filter passes of three fields through the plan's own engine (any of them: banded direct or
// row-spectral, separable, prefix sum), framed by two kernels of this file: w_stage_kernel forms the
// nine inputs, pi_w_kernel the local filtered velocity, the stress in full (tau's xz, yz, zz too), the
// strain with the gradient of wbar, Pi and the energy partials.  Compiled with --fmad=false like the
// rest.
#include <cstdint>

#include "cgef_internal.h"
#include "stencil.cuh"

namespace cgef {

namespace {

__device__ __forceinline__ double load_v(const void* p, int dtype, int64_t k) {
  return dtype == CGEF_F32 ? static_cast<double>(static_cast<const float*>(p)[k]) : static_cast<const double*>(p)[k];
}

__device__ __forceinline__ void store_v(void* p, int dtype, int64_t k, double v) {
  if (dtype == CGEF_F32)
    static_cast<float*>(p)[k] = static_cast<float>(v);
  else
    static_cast<double*>(p)[k] = v;
}

struct WStageK {
  const void* u;
  const void* v;
  const void* w;
  int dtype;
  const uint8_t* mask;
  int64_t mask_stride;
  int nx, ny, nbatch, sphere;
  const double* sinlam;
  const double* coslam;
  const double* sinphi;
  const double* cosphi;
  double* out;  // [q][slice][ny*nx], q = 0..8: the three components, then 00, 01, 02, 11, 12, 22
};

// The nine fields the flux filters, zero on masked cells (Diagnostics.jl:503-521, 555-590): the sphere's
// planetary velocity is east * u + north * v + up * w.
__global__ void w_stage_kernel(WStageK a) {
  const int64_t N = static_cast<int64_t>(a.nx) * a.ny;
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (k >= N) return;
  const int64_t o = s * N + k;
  const bool act = a.mask == nullptr || a.mask[s * a.mask_stride + k] != 0;
  double c0 = 0.0, c1 = 0.0, c2 = 0.0;
  if (act) {
    const double u = load_v(a.u, a.dtype, o), v = load_v(a.v, a.dtype, o), w = load_v(a.w, a.dtype, o);
    if (a.sphere) {
      const int i = static_cast<int>(k % a.nx), j = static_cast<int>(k / a.nx);
      const double sl = a.sinlam[i], cl = a.coslam[i], sp = a.sinphi[j], cp = a.cosphi[j];
      c0 = -sl * u - sp * cl * v + cp * cl * w;
      c1 = cl * u - sp * sl * v + cp * sl * w;
      c2 = cp * v + sp * w;
    } else {
      c0 = u;
      c1 = v;
      c2 = w;
    }
  }
  const int64_t q = static_cast<int64_t>(a.nbatch) * N;
  double* d = a.out + o;
  d[0] = c0;
  d[q] = c1;
  d[2 * q] = c2;
  d[3 * q] = c0 * c0;
  d[4 * q] = c0 * c1;
  d[5 * q] = c0 * c2;
  d[6 * q] = c1 * c1;
  d[7 * q] = c1 * c2;
  d[8 * q] = c2 * c2;
}

struct PiWK {
  const double* f;  // [q][slice][ny*nx]: the filtered nine fields
  const uint8_t* mask;
  int64_t mask_stride;
  int nx, ny, nbatch, periodic_x, periodic_y, sphere, dtype;
  double dx, dy, yscale;
  const double* xscale;
  const double* tanfac;
  const double* area;
  const double* sinlam;
  const double* coslam;
  const double* sinphi;
  const double* cosphi;
  void* pi;
  void* o[14];  // ubar, vbar, wbar, txx, txy, tyy, txz, tyz, tzz, sxx, sxy, syy, sxz, syz (nullptr: skip)
  double* partials;  // [slice][block][2], or nullptr
};

// The local filtered velocity at (j, i): the planetary one dotted with east, north and up (sphere).
__device__ __forceinline__ void local_vel3(const PiWK& a, const double* f, int64_t q, int j, int i, double (&l)[3]) {
  const int64_t k = static_cast<int64_t>(j) * a.nx + i;
  const double U0 = f[k], U1 = f[q + k], U2 = f[2 * q + k];
  if (!a.sphere) {
    l[0] = U0;
    l[1] = U1;
    l[2] = U2;
    return;
  }
  const double sl = a.sinlam[i], cl = a.coslam[i], sp = a.sinphi[j], cp = a.cosphi[j];
  const double e[3] = {-sl, cl, 0.0};
  const double n[3] = {-sp * cl, -sp * sl, cp};
  const double r[3] = {cp * cl, cp * sl, sp};
  l[0] = e[0] * U0 + e[1] * U1 + e[2] * U2;
  l[1] = n[0] * U0 + n[1] * U1 + n[2] * U2;
  l[2] = r[0] * U0 + r[1] * U1 + r[2] * U2;
}

constexpr int kWBX = 32, kWBY = 8;

__device__ __forceinline__ double axis_derivative(const PiWK& a, const double* f, int64_t q, const StencilCase& c,
                                                  int comp, int j, int i, bool along_x, double centre) {
  double vm1 = 0.0, vp1 = 0.0, vx2 = 0.0, l[3];
  if (uses_m1(c)) {
    along_x ? local_vel3(a, f, q, j, c.m1, l) : local_vel3(a, f, q, c.m1, i, l);
    vm1 = l[comp];
  }
  if (uses_p1(c)) {
    along_x ? local_vel3(a, f, q, j, c.p1, l) : local_vel3(a, f, q, c.p1, i, l);
    vp1 = l[comp];
  }
  if (uses_x2(c)) {
    along_x ? local_vel3(a, f, q, j, c.x2, l) : local_vel3(a, f, q, c.x2, i, l);
    vx2 = l[comp];
  }
  return stencil_eval(c, centre, vm1, vp1, vx2, along_x ? a.dx : a.dy);
}

// Per target: the local filtered velocity, the stress rotated to east/north/up in full (Diagnostics.jl:
// 612-650; on the plane tau_ij = (u_i u_j)bar - ubar_i ubar_j, 525-535), the ReduceInRun strain of ubar
// and vbar with the sphere's curvature terms and half the gradient of wbar (Diagnostics.jl:537-548,
// 652-667), Pi (463-465, 689-699) and the energy partials of 1/2 |ubar|^2 over the block, wbar^2
// included (1125-1134).
__global__ void __launch_bounds__(kWBX * kWBY) pi_w_kernel(PiWK a) {
  __shared__ double sh[2 * (kWBX * kWBY / 32)];
  const int i = blockIdx.x * kWBX + threadIdx.x;
  const int j = blockIdx.y * kWBY + threadIdx.y;
  const int s = blockIdx.z;
  const int64_t N = static_cast<int64_t>(a.nx) * a.ny;
  const int64_t q = static_cast<int64_t>(a.nbatch) * N;
  const double* f = a.f + s * N;
  double e_num = 0.0, e_area = 0.0;
  if (i < a.nx && j < a.ny) {
    const int64_t pix = static_cast<int64_t>(j) * a.nx + i;
    const uint8_t* mk = a.mask ? a.mask + s * a.mask_stride : nullptr;
    const bool act = mk == nullptr || mk[pix] != 0;
    double vals[14] = {};
    double pi = 0.0;
    if (act) {
      double l[3];
      local_vel3(a, f, q, j, i, l);
      const double U0 = f[pix], U1 = f[q + pix], U2 = f[2 * q + pix];
      double T[3][3];
      T[0][0] = f[3 * q + pix] - U0 * U0;
      T[0][1] = T[1][0] = f[4 * q + pix] - U0 * U1;
      T[0][2] = T[2][0] = f[5 * q + pix] - U0 * U2;
      T[1][1] = f[6 * q + pix] - U1 * U1;
      T[1][2] = T[2][1] = f[7 * q + pix] - U1 * U2;
      T[2][2] = f[8 * q + pix] - U2 * U2;
      double txx, txy, tyy, txz, tyz, tzz;
      if (a.sphere) {
        const double sl = a.sinlam[i], cl = a.coslam[i], sp = a.sinphi[j], cp = a.cosphi[j];
        const double e[3] = {-sl, cl, 0.0};
        const double n[3] = {-sp * cl, -sp * sl, cp};
        const double r[3] = {cp * cl, cp * sl, sp};
        double te[3], tn[3], tr[3];
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          te[b] = T[b][0] * e[0] + T[b][1] * e[1] + T[b][2] * e[2];
          tn[b] = T[b][0] * n[0] + T[b][1] * n[1] + T[b][2] * n[2];
          tr[b] = T[b][0] * r[0] + T[b][1] * r[1] + T[b][2] * r[2];
        }
        txx = e[0] * te[0] + e[1] * te[1] + e[2] * te[2];
        txy = e[0] * tn[0] + e[1] * tn[1] + e[2] * tn[2];
        tyy = n[0] * tn[0] + n[1] * tn[1] + n[2] * tn[2];
        txz = e[0] * tr[0] + e[1] * tr[1] + e[2] * tr[2];
        tyz = n[0] * tr[0] + n[1] * tr[1] + n[2] * tr[2];
        tzz = r[0] * tr[0] + r[1] * tr[1] + r[2] * tr[2];
      } else {
        txx = T[0][0];
        txy = T[0][1];
        tyy = T[1][1];
        txz = T[0][2];
        tyz = T[1][2];
        tzz = T[2][2];
      }
      const Line Lx{nullptr, mk ? mk + static_cast<int64_t>(j) * a.nx : nullptr, 1, a.nx, a.periodic_x, a.dx};
      const Line Ly{nullptr, mk ? mk + i : nullptr, a.nx, a.ny, a.periodic_y, a.dy};
      const StencilCase cx = stencil_case(Lx, i), cy = stencil_case(Ly, j);
      const double xs = a.xscale[j];
      double d[3][2];  // d[comp][0]: d/dx, d[comp][1]: d/dy
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        d[c][0] = a.nx < 2 ? 0.0 : axis_derivative(a, f, q, cx, c, j, i, true, l[c]) * xs;
        d[c][1] = a.ny < 2 ? 0.0 : axis_derivative(a, f, q, cy, c, j, i, false, l[c]) * a.yscale;
      }
      double sxx = d[0][0], syy = d[1][1], sxy;
      if (a.sphere) {
        const double tf = a.tanfac[j];
        sxx -= l[1] * tf;
        sxy = 0.5 * (d[0][1] + d[1][0] + l[0] * tf);
      } else {
        sxy = 0.5 * (d[0][1] + d[1][0]);
      }
      const double sxz = 0.5 * d[2][0], syz = 0.5 * d[2][1], szz = 0.0;
      pi = -(sxx * txx + 2.0 * sxy * txy + syy * tyy + 2.0 * sxz * txz + 2.0 * syz * tyz + szz * tzz);
      const double v14[14] = {l[0], l[1], l[2], txx, txy, tyy, txz, tyz, tzz, sxx, sxy, syy, sxz, syz};
#pragma unroll
      for (int m = 0; m < 14; ++m) vals[m] = v14[m];
      const double ar = a.area[j];
      e_num = (l[0] * l[0] + l[1] * l[1] + l[2] * l[2]) * ar;
      e_area = ar;
    }
    const int64_t o = s * N + pix;
    if (a.pi) store_v(a.pi, a.dtype, o, pi);
#pragma unroll
    for (int m = 0; m < 14; ++m)
      if (a.o[m]) store_v(a.o[m], a.dtype, o, vals[m]);
  }
  if (a.partials) {
    // deterministic block sums: warp shuffles in a fixed tree, then the warps in order
    for (int off = 16; off > 0; off >>= 1) {
      e_num += __shfl_down_sync(0xffffffffu, e_num, off);
      e_area += __shfl_down_sync(0xffffffffu, e_area, off);
    }
    const int tid = threadIdx.y * kWBX + threadIdx.x;
    if ((tid & 31) == 0) {
      sh[2 * (tid >> 5)] = e_num;
      sh[2 * (tid >> 5) + 1] = e_area;
    }
    __syncthreads();
    if (tid == 0) {
      double x = 0.0, y = 0.0;
      for (int w = 0; w < kWBX * kWBY / 32; ++w) {
        x += sh[2 * w];
        y += sh[2 * w + 1];
      }
      const int64_t nblk = static_cast<int64_t>(gridDim.x) * gridDim.y;
      const int64_t b = static_cast<int64_t>(blockIdx.y) * gridDim.x + blockIdx.x;
      a.partials[(s * nblk + b) * 2] = x;
      a.partials[(s * nblk + b) * 2 + 1] = y;
    }
  }
}

int w_check(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, what);
  count_launch();
  return CGEF_OK;
}

}  // namespace

int compute_pi_w_device(cgef_plan* p, int dtype, const void* u, const void* v, const void* w, int64_t nbatch64,
                        const uint8_t* slice_masks, const cgef_pi_w_outputs* out, cudaStream_t st) {
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (!u || !v || !w) return fail(CGEF_EINVAL, "u, v and w must be non-NULL");
  if (nbatch64 < 1 || nbatch64 > kMaxSlices) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  const int nbatch = static_cast<int>(nbatch64);
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const uint8_t* mask = slice_masks ? slice_masks : p->d_mask;
  const int64_t mstride = slice_masks ? N : 0;
  const bool sphere = p->geometry == CGEF_SPHERICAL;
  // [before | after] filtering: nine FP64 fields each, [q][slice][ny*nx]
  void* buf = nullptr;
  const int64_t q = static_cast<int64_t>(nbatch) * N;
  if ((rc = ensure_ws(p, kSlotW, sizeof(double) * 18 * q, &buf))) return rc;
  double* in = static_cast<double*>(buf);
  double* fl = in + 9 * q;
  WStageK sa{u, v, w, dtype, mask, mstride, p->nx, p->ny, nbatch, sphere ? 1 : 0,
             p->d_sinlam, p->d_coslam, p->d_sinphi, p->d_cosphi, in};
  w_stage_kernel<<<dim3(static_cast<unsigned>((N + 255) / 256), nbatch), 256, 0, st>>>(sa);
  if ((rc = w_check("w_stage_kernel"))) return rc;
  // three filter passes of three fields through the plan's engine
  for (int pass = 0; pass < 3; ++pass) {
    const void* fields[3] = {in + (3 * pass) * q, in + (3 * pass + 1) * q, in + (3 * pass + 2) * q};
    double* outs[3] = {fl + (3 * pass) * q, fl + (3 * pass + 1) * q, fl + (3 * pass + 2) * q};
    if ((rc = filter_fields_device(p, CGEF_F64, fields, 3, outs, N, nbatch, mask, mstride, st))) return rc;
  }
  cgef_pi_w_outputs none{};
  const cgef_pi_w_outputs* o = out ? out : &none;
  PiWK a{};
  a.f = fl;
  a.mask = mask;
  a.mask_stride = mstride;
  a.nx = p->nx;
  a.ny = p->ny;
  a.nbatch = nbatch;
  a.periodic_x = p->periodic_x;
  a.periodic_y = p->periodic_y;
  a.sphere = sphere ? 1 : 0;
  a.dtype = dtype;
  a.dx = p->dx;
  a.dy = p->dy;
  a.yscale = sphere ? 1.0 / p->R : 1.0;
  a.xscale = p->d_xscale;
  a.tanfac = p->d_tanfac;
  a.area = p->d_area;
  a.sinlam = p->d_sinlam;
  a.coslam = p->d_coslam;
  a.sinphi = p->d_sinphi;
  a.cosphi = p->d_cosphi;
  a.pi = o->pi;
  void* const outs14[14] = {o->ubar, o->vbar, o->wbar, o->tau_xx, o->tau_xy, o->tau_yy, o->tau_xz,
                            o->tau_yz, o->tau_zz, o->s_xx, o->s_xy, o->s_yy, o->s_xz, o->s_yz};
  for (int m = 0; m < 14; ++m) a.o[m] = outs14[m];
  const dim3 grid((p->nx + kWBX - 1) / kWBX, (p->ny + kWBY - 1) / kWBY, nbatch);
  const int64_t nblk = static_cast<int64_t>(grid.x) * grid.y;
  if (o->energy) {
    void* part = nullptr;
    if ((rc = ensure_ws(p, kSlotPartials, sizeof(double) * 2 * nblk * nbatch, &part))) return rc;
    a.partials = static_cast<double*>(part);
  }
  pi_w_kernel<<<grid, dim3(kWBX, kWBY), 0, st>>>(a);
  if ((rc = w_check("pi_w_kernel"))) return rc;
  if (o->energy) {
    if ((rc = launch_energy_finish(a.partials, nblk, nbatch, o->energy, 1, 0.5, st))) return rc;
  }
  return CGEF_OK;
}

}  // namespace cgef
