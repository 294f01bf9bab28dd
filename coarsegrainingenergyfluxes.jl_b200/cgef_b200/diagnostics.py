"""Cross-scale energy flux and filtering energies (Diagnostics.jl), strain stencils
(Derivatives.jl), all computed by the CUDA library.

Pi = -(S_xx tau_xx + 2 S_xy tau_xy + S_yy tau_yy) with no rho0 factor, exactly as the
reference's `compute_Π!` returns it (Diagnostics.jl:689-699); multiply by rho0 yourself for
the README's -rho0 tau:S form.
"""
from __future__ import annotations

import ctypes as C
import warnings
from typing import Dict, Optional, Sequence

import numpy as np

from . import _arrays as A
from . import _lib
from .errors import ArgumentError, DimensionMismatch
from .filtering import AbstractMaskStrategy, PhysicalFilterPlan, ZeroFill, plan_filter
from .grids import StructuredGrid
from .kernels import AbstractFilterKernel, check_spectrum_kernel, transfer_monotone

PI_OUTPUTS = ("Pi", "ubar", "vbar", "tau_xx", "tau_xy", "tau_yy", "S_xx", "S_xy", "S_yy")
_FIELD = {"Pi": "pi", "ubar": "ubar", "vbar": "vbar", "tau_xx": "tau_xx", "tau_xy": "tau_xy", "tau_yy": "tau_yy",
          "S_xx": "s_xx", "S_xy": "s_xy", "S_yy": "s_yy"}
# the 2.5-D flux (compute_Pi with w): the vertical velocity and the stress and strain terms it adds
PI_W_OUTPUTS = ("Pi", "ubar", "vbar", "wbar", "tau_xx", "tau_xy", "tau_yy", "tau_xz", "tau_yz", "tau_zz",
                "S_xx", "S_xy", "S_yy", "S_xz", "S_yz")


# ------------------------------------------------------------------------------------------
# Spectrum admissibility policy (Diagnostics.jl:17-81)
# ------------------------------------------------------------------------------------------
class AbstractSpectrumPolicy:
    def __eq__(self, other):
        return type(self) is type(other)

    def __hash__(self):
        return hash(type(self))


class StrictSpectrum(AbstractSpectrumPolicy):
    """Refuse a density for a kernel with non-monotone |G|^2 (the default)."""


class ForceSpectrum(AbstractSpectrumPolicy):
    """Compute the density anyway, warning once."""


class NoSpectrum(AbstractSpectrumPolicy):
    """Skip the density; it is filled with NaN."""


def gate_spectrum(kernel: AbstractFilterKernel, policy: AbstractSpectrumPolicy) -> bool:
    """Throw (StrictSpectrum, non-monotone kernel) / warn and compute (ForceSpectrum) / skip
    (NoSpectrum).  A policy that is not one of the three types is a TypeError, as the reference's
    typed keyword makes `spectrum = false` or `spectrum = :force` (Diagnostics.jl:17-81)."""
    if not isinstance(policy, AbstractSpectrumPolicy):
        raise TypeError(f"spectrum must be StrictSpectrum(), ForceSpectrum() or NoSpectrum(), got {policy!r}")
    if isinstance(policy, StrictSpectrum):
        check_spectrum_kernel(kernel)
        return True
    if isinstance(policy, NoSpectrum):
        return False
    if not transfer_monotone(kernel):
        warnings.warn(f"ForceSpectrum with {type(kernel).__name__}: |G(k)|^2 is not monotone, so the filtering "
                      "spectral density is not guaranteed non-negative.", stacklevel=2)
    return True


# ------------------------------------------------------------------------------------------
def _batch_shape(a, grid: StructuredGrid, name: str):
    shp = tuple(a.shape)
    if len(shp) < 2 or shp[-2:] != grid.shape:
        raise DimensionMismatch(f"{name}'s trailing axes {shp[-2:]} do not match the grid's (ny, nx) {grid.shape}")
    return shp[:-2]


def _nbatch(bshape) -> int:
    return int(np.prod(bshape)) if bshape else 1


def _slice_masks(slice_masks, u, nb: int, grid: StructuredGrid):
    if slice_masks is None:
        return None
    m = A.mask_bytes(slice_masks, u)
    if tuple(m.shape[-2:]) != grid.shape or int(np.prod(m.shape)) != nb * grid.nx * grid.ny:
        raise DimensionMismatch("slice_masks must hold one (ny, nx) mask per slice")
    return m


def compute_Pi(Pi, u, v, w, grid: StructuredGrid, kernel: AbstractFilterKernel, scale: float, *,
               filter_plan: Optional[PhysicalFilterPlan] = None,
               mask_strategy: AbstractMaskStrategy = ZeroFill(),
               outputs: Optional[Dict[str, object]] = None,
               energy: Optional[np.ndarray] = None,
               slice_masks=None):
    """Diagnostics.compute_Π! (Diagnostics.jl:389-416) on a 2-D StructuredGrid.

    u, v: (..., ny, nx) -- leading axes are independent slices sharing the grid (the reference's
    trailing batch axes), computed in one fused pass.  `outputs` may map any of ubar, vbar, tau_xx,
    tau_xy, tau_yy, S_xx, S_xy, S_yy to preallocated arrays to receive the local-frame intermediate
    fields; `energy` (one float64 per slice) receives E = 1/2 <|ubar|^2>.  `slice_masks` gives one
    mask per slice (coarse_grain_slices! semantics).  Host arrays run through the synchronous C ABI,
    CUDA tensors through the stream-ordered device entry point.
    """
    if w is not None:
        return _compute_Pi_w(Pi, u, v, w, grid, kernel, scale, filter_plan=filter_plan, mask_strategy=mask_strategy,
                             outputs=outputs, energy=energy, slice_masks=slice_masks)
    bs = _batch_shape(u, grid, "u")
    if _batch_shape(v, grid, "v") != bs:
        raise DimensionMismatch("v's batch axes do not match u's")
    nb = _nbatch(bs)
    plan = filter_plan if filter_plan is not None else plan_filter(grid, kernel, scale, mask_strategy=mask_strategy)
    if Pi is None:
        Pi = A.empty_like(u)
    if tuple(Pi.shape) != tuple(u.shape):
        raise DimensionMismatch(f"Pi {tuple(Pi.shape)} does not match u {tuple(u.shape)}")
    dt = A.dtype_code(u)
    if A.dtype_code(v) != dt or A.dtype_code(Pi) != dt:
        raise ArgumentError("u, v and Pi must share a dtype")
    outs = _lib.PiOutputs()
    outs.pi = A.ptr(Pi)
    keep = []
    for k, arr in (outputs or {}).items():
        if k not in _FIELD or k == "Pi":
            raise ArgumentError(f"unknown output {k!r}; choose from {PI_OUTPUTS[1:]}")
        if tuple(arr.shape) != tuple(u.shape) or A.dtype_code(arr) != dt:
            raise DimensionMismatch(f"output {k} must match u's shape and dtype")
        setattr(outs, _FIELD[k], A.ptr(arr))
    if energy is not None:
        if int(np.prod(energy.shape)) != nb:
            raise DimensionMismatch("energy needs one entry per slice")
        outs.energy = A.ptr(energy)
    L = _lib.load()
    m = _slice_masks(slice_masks, u, nb, grid)
    keep.append(m)
    if A.is_device(u):
        _lib.check(L.cgef_compute_pi_device(plan.handle, dt, A.ptr(u), A.ptr(v), nb,
                                            None if m is None else A.ptr(m), C.byref(outs), A.stream_of(u)))
    else:
        u = np.ascontiguousarray(u)
        v = np.ascontiguousarray(v)
        _lib.check(L.cgef_compute_pi(plan.handle, dt, A.ptr(u), A.ptr(v), nb,
                                     None if m is None else A.ptr(m), C.byref(outs)))
    return Pi


compute_Π = compute_Pi


def _compute_Pi_w(Pi, u, v, w, grid, kernel, scale, *, filter_plan, mask_strategy, outputs, energy, slice_masks):
    """compute_Π! with the vertical velocity (Diagnostics.jl:254-260, 483-681): cgef_compute_pi_w."""
    bs = _batch_shape(u, grid, "u")
    if _batch_shape(v, grid, "v") != bs or _batch_shape(w, grid, "w") != bs:
        raise DimensionMismatch("v's and w's batch axes must match u's")
    nb = _nbatch(bs)
    plan = filter_plan if filter_plan is not None else plan_filter(grid, kernel, scale, mask_strategy=mask_strategy)
    if Pi is None:
        Pi = A.empty_like(u)
    if tuple(Pi.shape) != tuple(u.shape):
        raise DimensionMismatch(f"Pi {tuple(Pi.shape)} does not match u {tuple(u.shape)}")
    dt = A.dtype_code(u)
    if A.dtype_code(v) != dt or A.dtype_code(w) != dt or A.dtype_code(Pi) != dt:
        raise ArgumentError("u, v, w and Pi must share a dtype")
    outs = _lib.PiWOutputs()
    outs.pi = A.ptr(Pi)
    for k, arr in (outputs or {}).items():
        if k not in PI_W_OUTPUTS or k == "Pi":
            raise ArgumentError(f"unknown output {k!r}; choose from {PI_W_OUTPUTS[1:]}")
        if tuple(arr.shape) != tuple(u.shape) or A.dtype_code(arr) != dt:
            raise DimensionMismatch(f"output {k} must match u's shape and dtype")
        setattr(outs, k.lower() if k.startswith("S_") else k, A.ptr(arr))
    if energy is not None:
        if int(np.prod(energy.shape)) != nb:
            raise DimensionMismatch("energy needs one entry per slice")
        outs.energy = A.ptr(energy)
    L = _lib.load()
    m = _slice_masks(slice_masks, u, nb, grid)
    if A.is_device(u):
        _lib.check(L.cgef_compute_pi_w_device(plan.handle, dt, A.ptr(u), A.ptr(v), A.ptr(w), nb,
                                              None if m is None else A.ptr(m), C.byref(outs), A.stream_of(u)))
    else:
        u, v, w = (np.ascontiguousarray(x) for x in (u, v, w))
        _lib.check(L.cgef_compute_pi_w(plan.handle, dt, A.ptr(u), A.ptr(v), A.ptr(w), nb,
                                       None if m is None else A.ptr(m), C.byref(outs)))
    return Pi


def compute_Pi_fields(u, v, grid: StructuredGrid, kernel: AbstractFilterKernel, scale: float, *,
                      mask_strategy: AbstractMaskStrategy = ZeroFill(),
                      filter_plan: Optional[PhysicalFilterPlan] = None, slice_masks=None, w=None) -> Dict[str, object]:
    """compute_Π! returning every intermediate (the reference's ΠWorkspace contents) and E; with the
    vertical velocity w, the 2.5-D path's as well (wbar, tau_xz, tau_yz, tau_zz, S_xz, S_yz)."""
    outs = {k: A.empty_like(u) for k in (PI_OUTPUTS if w is None else PI_W_OUTPUTS)[1:]}
    nb = _nbatch(tuple(u.shape[:-2]))
    if A.is_device(u):
        import torch
        energy = torch.empty(nb, dtype=torch.float64, device=u.device)
    else:
        energy = np.empty(nb, dtype=np.float64)
    Pi = compute_Pi(None, u, v, w, grid, kernel, scale, filter_plan=filter_plan, mask_strategy=mask_strategy,
                    outputs=outs, energy=energy, slice_masks=slice_masks)
    outs["Pi"] = Pi
    outs["energy"] = energy
    return outs


def active_area(grid: StructuredGrid) -> float:
    """Diagnostics.active_area (Diagnostics.jl:1051-1059)."""
    ar = grid.area()
    total = float((ar[:, None] * (np.ones(grid.shape) if grid.mask is None else grid.mask)).sum())
    if not total > 0:
        raise ArgumentError("grid has no active cells (all masked out)")
    return total


def cumulative_energy(u, v, w, grid: StructuredGrid, kernel: AbstractFilterKernel, scales: Sequence[float], *,
                      mask_strategy: AbstractMaskStrategy = ZeroFill(),
                      filter_plans: Optional[Sequence[PhysicalFilterPlan]] = None, method=None) -> np.ndarray:
    """Diagnostics.cumulative_energy (Diagnostics.jl:1144-1251): E(l) = 1/2 <|ubar_l|^2> with u, v (and
    w, whose wbar^2 joins the sum, Diagnostics.jl:1203-1211) filtered as scalars at every scale (host
    arrays).  `method` as for plan_filter."""
    if tuple(u.shape) != grid.shape or tuple(v.shape) != grid.shape:
        raise DimensionMismatch(f"u and v must have the grid's shape {grid.shape}")
    if w is not None and tuple(w.shape) != grid.shape:
        raise DimensionMismatch(f"w must have the grid's shape {grid.shape}")
    active_area(grid)
    plans = list(filter_plans) if filter_plans is not None else [
        plan_filter(grid, kernel, float(s), mask_strategy=mask_strategy, method=method) for s in scales]
    if len(plans) != len(scales):
        raise DimensionMismatch("one plan per scale")
    dt = A.dtype_code(u)
    if A.dtype_code(v) != dt or (w is not None and A.dtype_code(w) != dt):
        raise ArgumentError("u, v and w must share a dtype")
    arr = (C.c_void_p * len(plans))(*[p.handle.value for p in plans])

    def half_energy(a, b):
        ha = np.ascontiguousarray(A.host(a))
        hb = np.ascontiguousarray(A.host(b))
        e = np.zeros(len(plans), dtype=np.float64)
        _lib.check(_lib.load().cgef_cumulative_energy(arr, len(plans), dt, ha.ctypes.data, hb.ctypes.data,
                                                      e.ctypes.data))
        return e

    spec = half_energy(u, v)
    if w is not None:
        hw = A.host(w)
        spec = spec + half_energy(hw, np.zeros_like(hw))
    return spec


def spectral_density(Cv, k) -> np.ndarray:
    """Diagnostics.spectral_density (Diagnostics.jl:1319-1343): central differences, one-sided ends."""
    Cv = np.asarray(Cv, dtype=np.float64)
    k = np.asarray(k, dtype=np.float64)
    n = len(Cv)
    if len(k) != n:
        raise DimensionMismatch("C and k lengths differ")
    g = np.zeros(n)
    if n < 2:
        return g
    g[0] = (Cv[1] - Cv[0]) / (k[1] - k[0])
    g[-1] = (Cv[-1] - Cv[-2]) / (k[-1] - k[-2])
    if n > 2:
        g[1:-1] = (Cv[2:] - Cv[:-2]) / (k[2:] - k[:-2])
    return g


def filtering_spectrum(u, v, w, grid: StructuredGrid, kernel: AbstractFilterKernel, scales, *, L: float = 1.0,
                       mask_strategy: AbstractMaskStrategy = ZeroFill(),
                       policy: AbstractSpectrumPolicy = StrictSpectrum(), method=None):
    """Diagnostics.filtering_spectrum (Diagnostics.jl:1292-1310) -> (k_l, dE/dk_l)."""
    compute = gate_spectrum(kernel, policy)
    cum = cumulative_energy(u, v, w, grid, kernel, scales, mask_strategy=mask_strategy, method=method)
    kl = float(L) / np.asarray(scales, dtype=np.float64)
    if not compute:
        return kl, np.full(len(kl), np.nan)
    return kl, spectral_density(cum, kl)


# ------------------------------------------------------------------------------------------
# Decompositions (Diagnostics.jl:1350-1527, 1724-1852)
# ------------------------------------------------------------------------------------------
def tau_decomposition(u, v, grid: StructuredGrid, kernel: AbstractFilterKernel, scale: float, *,
                      mask_strategy: AbstractMaskStrategy = ZeroFill(),
                      filter_plan: Optional[PhysicalFilterPlan] = None) -> Dict[str, Dict[str, object]]:
    """Diagnostics.tau_decomposition (Diagnostics.jl:1350-1527): tau = Leonard + Cross + Reynolds with
    generalized central moments (Germano 1992).  Returns {"L": {"xx", "xy", "yy"}, "C": ..., "R": ...};
    on the sphere the components are east-east, east-north, north-north."""
    if tuple(u.shape) != grid.shape or tuple(v.shape) != grid.shape:
        raise DimensionMismatch(f"u and v must have the grid's shape {grid.shape}")
    plan = filter_plan if filter_plan is not None else plan_filter(grid, kernel, scale, mask_strategy=mask_strategy)
    dt = A.dtype_code(u)
    if A.dtype_code(v) != dt:
        raise ArgumentError("u and v must share a dtype")
    outs = {part: {c: A.empty_like(u) for c in ("xx", "xy", "yy")} for part in ("L", "C", "R")}
    tp = _lib.TauParts()
    for field, part in (("leonard", "L"), ("cross", "C"), ("reynolds", "R")):
        arr = getattr(tp, field)
        for k, c in enumerate(("xx", "xy", "yy")):
            arr[k] = A.ptr(outs[part][c])
    L = _lib.load()
    if A.is_device(u):
        _lib.check(L.cgef_tau_decomposition_device(plan.handle, dt, A.ptr(u.contiguous()), A.ptr(v.contiguous()),
                                                   C.byref(tp), A.stream_of(u)))
    else:
        _lib.check(L.cgef_tau_decomposition(plan.handle, dt, A.ptr(np.ascontiguousarray(u)),
                                            A.ptr(np.ascontiguousarray(v)), C.byref(tp)))
    return outs


def compute_Pi_strain_convergence(u, v, grid: StructuredGrid, kernel: AbstractFilterKernel, scale: float, *,
                                  mask_strategy: AbstractMaskStrategy = ZeroFill(),
                                  filter_plan: Optional[PhysicalFilterPlan] = None) -> Dict[str, object]:
    """Diagnostics.compute_Π_strain_convergence (Diagnostics.jl:1724-1852): the flux split into
    deformation (`strain`) and convergence production, Pi = strain - convergence, with the two
    rotation invariants `divergence` and `strain_magnitude`.  Cartesian grids only, as in the
    reference; u, v may carry leading batch axes."""
    if grid.is_spherical:
        raise ArgumentError("compute_Pi_strain_convergence is defined for Cartesian grids only")
    bs = _batch_shape(u, grid, "u")
    if _batch_shape(v, grid, "v") != bs:
        raise DimensionMismatch("v's batch axes do not match u's")
    nb = _nbatch(bs)
    plan = filter_plan if filter_plan is not None else plan_filter(grid, kernel, scale, mask_strategy=mask_strategy)
    dt = A.dtype_code(u)
    if A.dtype_code(v) != dt:
        raise ArgumentError("u and v must share a dtype")
    names = ("total", "strain", "convergence", "divergence", "strain_magnitude")
    outs = {n: A.empty_like(u) for n in names}
    so = _lib.StrainConvOutputs(*[A.ptr(outs[n]) for n in names])
    L = _lib.load()
    if A.is_device(u):
        _lib.check(L.cgef_pi_strain_convergence_device(plan.handle, dt, A.ptr(u.contiguous()), A.ptr(v.contiguous()),
                                                       nb, None, C.byref(so), A.stream_of(u)))
    else:
        _lib.check(L.cgef_pi_strain_convergence(plan.handle, dt, A.ptr(np.ascontiguousarray(u)),
                                                A.ptr(np.ascontiguousarray(v)), nb, C.byref(so)))
    return outs


compute_Π_strain_convergence = compute_Pi_strain_convergence


# ------------------------------------------------------------------------------------------
# Derivatives.jl
# ------------------------------------------------------------------------------------------
def _deriv(axis_fn: str, out, f, grid_or_plan):
    plan = grid_or_plan if isinstance(grid_or_plan, PhysicalFilterPlan) else _stencil_plan(grid_or_plan)
    if tuple(f.shape) != plan.grid.shape:
        raise DimensionMismatch(f"field shape {tuple(f.shape)} != grid {plan.grid.shape}")
    f = np.ascontiguousarray(f)
    if out is None:
        out = np.empty_like(f)
    _lib.check(getattr(_lib.load(), axis_fn)(plan.handle, A.dtype_code(f), f.ctypes.data, out.ctypes.data))
    return out


_STENCIL_PLANS: dict = {}


def _stencil_plan(grid: StructuredGrid) -> PhysicalFilterPlan:
    """Derivatives.StencilPlan: the grid's stencil tables (carried by a minimal plan)."""
    from .kernels import TopHatKernel
    key = id(grid)
    p = _STENCIL_PLANS.get(key)
    if p is None or p.grid is not grid:
        step = max(grid.x.step, grid.y.step) * (grid.geometry.R if grid.is_spherical else 1.0)
        p = plan_filter(grid, TopHatKernel(), step)
        _STENCIL_PLANS[key] = p
    return p


def ddx(out, f, grid):
    """Derivatives.ddx! (Derivatives.jl:42-44): 3-node, ReduceInRun at mask edges; the sphere
    divides by R cos(phi) (0 at the pole guard)."""
    return _deriv("cgef_ddx", out, f, grid)


def ddy(out, f, grid):
    """Derivatives.ddy! (Derivatives.jl:51): 3-node, ReduceInRun; the sphere divides by R."""
    return _deriv("cgef_ddy", out, f, grid)
