// The ReduceInRun 3-node stencil (Derivatives.jl:26-31) shared by the strain passes: the case a
// point's neighbours' activity picks along one axis, and the case's formula on the values.
#pragma once

#include <cstdint>

namespace cgef {
namespace {

__device__ __forceinline__ int stencil_wrap(int a, int n) {
  int r = a % n;
  return r < 0 ? r + n : r;
}

// ReduceInRun 3-node first derivative along one axis (Derivatives.jl:26-31): centred with both
// neighbours active; 3-node one-sided when only one side has two active cells (the bounded end
// too); 2-node in a run of two; 0 for an isolated cell.
struct Line {
  const double* f;
  const uint8_t* m;  // activity, same indexing as f; nullptr = all active
  int64_t stride;    // element stride along the axis (f and m)
  int n;
  int periodic;
  double h;
};

__device__ __forceinline__ int nb_index(int p, int off, int n, int periodic) {
  int q = p + off;
  if (q < 0 || q >= n) {
    if (!periodic || n < 2) return -1;
    q = stencil_wrap(q, n);
  }
  return q;
}

__device__ __forceinline__ bool act_at(const Line& L, int q) { return q >= 0 && (L.m == nullptr || L.m[q * L.stride] != 0); }

// The ReduceInRun stencil of stencil() split in two: the neighbours' activity picks the case once per
// axis (the same for every field on that axis), then apply_stencil() evaluates it for one field with
// the same expressions, so results are identical.
struct StencilCase {
  int kind;  // 0: none, 1: centred, 2: forward 3-node, 3: forward 2-node, 4: backward 3-node, 5: backward 2-node
  int m1, p1, x2;
};

__device__ __forceinline__ StencilCase stencil_case(const Line& L, int p) {
  StencilCase c{0, nb_index(p, -1, L.n, L.periodic), nb_index(p, 1, L.n, L.periodic), -1};
  const bool am1 = act_at(L, c.m1), ap1 = act_at(L, c.p1);
  if (am1 && ap1) {
    c.kind = 1;
  } else if (ap1) {
    c.x2 = nb_index(p, 2, L.n, L.periodic);
    c.kind = (act_at(L, c.x2) && c.x2 != p) ? 2 : 3;
  } else if (am1) {
    c.x2 = nb_index(p, -2, L.n, L.periodic);
    c.kind = (act_at(L, c.x2) && c.x2 != p) ? 4 : 5;
  }
  return c;
}

// The case's formula on the values at the point (f0) and at its neighbours m1, p1 and x2 (the second
// neighbour on the case's side); values a case does not use are ignored.
__device__ __forceinline__ double stencil_eval(const StencilCase& c, double f0, double fm1, double fp1, double fx2,
                                               double h) {
  switch (c.kind) {
    case 1: return (fp1 - fm1) / (2.0 * h);
    case 2: return (-3.0 * f0 + 4.0 * fp1 - fx2) / (2.0 * h);
    case 3: return (fp1 - f0) / h;
    case 4: return (3.0 * f0 - 4.0 * fm1 + fx2) / (2.0 * h);
    case 5: return (f0 - fm1) / h;
    default: return 0.0;
  }
}

// Which neighbours a case reads.
__device__ __forceinline__ bool uses_m1(const StencilCase& c) { return c.kind == 1 || c.kind == 4 || c.kind == 5; }
__device__ __forceinline__ bool uses_p1(const StencilCase& c) { return c.kind == 1 || c.kind == 2 || c.kind == 3; }
__device__ __forceinline__ bool uses_x2(const StencilCase& c) { return c.kind == 2 || c.kind == 4; }

__device__ __forceinline__ double apply_stencil(const StencilCase& c, const double* f, int64_t stride, int p,
                                                double h) {
  const double f0 = f[p * stride];
  const double fm1 = uses_m1(c) ? f[c.m1 * stride] : 0.0;
  const double fp1 = uses_p1(c) ? f[c.p1 * stride] : 0.0;
  const double fx2 = uses_x2(c) ? f[c.x2 * stride] : 0.0;
  return stencil_eval(c, f0, fm1, fp1, fx2, h);
}

}  // namespace
}  // namespace cgef
