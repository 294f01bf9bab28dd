"""Scale sweeps (Pipeline.jl): Pi at every scale and slice, E(l), k_l and the spectral density.

One C-ABI call (`cgef_sweep`) computes the whole (slice x scale) sweep on the GPU: the inputs are
staged once, every scale's plan runs its fused footprint pass over all slices, and E(l) is read
from the same filtered velocities (Pipeline.jl:455-463).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _arrays as A
from . import _lib
from .diagnostics import AbstractSpectrumPolicy, NoSpectrum, StrictSpectrum, gate_spectrum, spectral_density
from .errors import ArgumentError, DimensionMismatch
from .filtering import AbstractMaskStrategy, PhysicalFilterPlan, ZeroFill, plan_filter
from .grids import StructuredGrid
from .kernels import AbstractFilterKernel, TopHatKernel


@dataclass
class CoarseGrainResult:
    """Pipeline.CoarseGrainResult (Pipeline.jl:270-284); Pi has shape (nscales, ny, nx)."""

    scales: np.ndarray
    Pi: object
    cumulative_energy: np.ndarray
    wavenumber: np.ndarray
    filtering_spectrum: np.ndarray

    @property
    def Π(self):
        return self.Pi


@dataclass
class CoarseGrainBatchResult:
    """Pipeline.CoarseGrainBatchResult (Pipeline.jl:606-651): Pi (batch..., nscales, ny, nx),
    per-scale vectors (batch..., nscales) -- the reference's trailing axes in C order."""

    Pi: object
    scales: np.ndarray
    cumulative_energy: np.ndarray
    wavenumber: np.ndarray
    filtering_spectrum: np.ndarray
    batch_size: tuple

    @property
    def Π(self):
        return self.Pi

    @property
    def slices(self) -> List[CoarseGrainResult]:
        nb = int(np.prod(self.batch_size)) if self.batch_size else 1
        flatPi = self.Pi.reshape((nb,) + tuple(self.Pi.shape[-3:]))
        out = []
        for t in range(nb):
            idx = np.unravel_index(t, self.batch_size) if self.batch_size else ()
            out.append(CoarseGrainResult(self.scales[idx], flatPi[t], self.cumulative_energy[idx],
                                         self.wavenumber[idx], self.filtering_spectrum[idx]))
        return out


def _plans(grid, kernel, scales, mask_strategy, filter_plans, method=None):
    if filter_plans is not None:
        plans = list(filter_plans)
        if len(plans) != len(scales):
            raise DimensionMismatch("filter_plans must hold one plan per scale")
        return plans
    return [plan_filter(grid, kernel, float(s), mask_strategy=mask_strategy, method=method) for s in scales]


def _sweep_w(u, v, w, grid, plans, nb, slice_masks, want_pi=True):
    """The sweep with the vertical velocity: compute_Pi with w per scale (cgef_compute_pi_w) over the
    whole batch; E includes wbar^2 (Diagnostics.jl:1125-1134)."""
    from .diagnostics import compute_Pi

    ns = len(plans)
    ny, nx = grid.shape
    Pi = np.empty((nb, ns, ny, nx), dtype=np.asarray(u).dtype)
    E = np.empty((nb, ns), dtype=np.float64)
    e = np.empty(nb, dtype=np.float64)
    for q, p in enumerate(plans):
        Pi[:, q] = compute_Pi(None, u, v, w, grid, p.kernel, p.scale, filter_plan=p, energy=e,
                              slice_masks=slice_masks)
        E[:, q] = e
    return (Pi if want_pi else None), E


def _sweep(u, v, grid, plans, nb, slice_masks, want_pi=True):
    dt = A.dtype_code(u)
    if A.dtype_code(v) != dt:
        raise ArgumentError("u and v must share a dtype")
    ns = len(plans)
    L = _lib.load()
    arr = (C.c_void_p * ns)(*[p.handle.value for p in plans])
    ny, nx = grid.shape
    if A.is_device(u):
        import torch
        Pi = torch.empty((nb, ns, ny, nx), dtype=u.dtype, device=u.device) if want_pi else None
        E = torch.empty((nb, ns), dtype=torch.float64, device=u.device)
        m = None if slice_masks is None else A.mask_bytes(slice_masks, u)
        _lib.check(L.cgef_sweep_device(arr, ns, dt, A.ptr(u), A.ptr(v), nb, None if m is None else A.ptr(m),
                                       None if Pi is None else A.ptr(Pi), A.ptr(E), A.stream_of(u)))
        return Pi, E.cpu().numpy()
    u = np.ascontiguousarray(u)
    v = np.ascontiguousarray(v)
    Pi = np.empty((nb, ns, ny, nx), dtype=u.dtype) if want_pi else None
    E = np.empty((nb, ns), dtype=np.float64)
    m = None if slice_masks is None else A.mask_bytes(slice_masks)
    _lib.check(L.cgef_sweep(arr, ns, dt, A.ptr(u), A.ptr(v), nb, None if m is None else A.ptr(m),
                            None if Pi is None else A.ptr(Pi), E.ctypes.data))
    return Pi, E


def _spectrum(E, k, spectrum):
    if isinstance(spectrum, NoSpectrum):
        return np.full_like(E, np.nan)
    return spectral_density(E, k)


def coarse_grain(u, v, grid: StructuredGrid, *, scales: Sequence[float], w=None,
                 kernel: AbstractFilterKernel = TopHatKernel(), mask_strategy: AbstractMaskStrategy = ZeroFill(),
                 filter_plans: Optional[Sequence[PhysicalFilterPlan]] = None, L: float = 1.0,
                 spectrum: AbstractSpectrumPolicy = StrictSpectrum(), method=None) -> CoarseGrainResult:
    """Pipeline.coarse_grain (Pipeline.jl:342-360, 412-468) for one (ny, nx) slice; `w` (the vertical
    velocity) runs the 2.5-D flux, `method` is plan_filter's."""
    if tuple(u.shape) != grid.shape or tuple(v.shape) != grid.shape:
        raise DimensionMismatch(f"u and v must have the grid's shape {grid.shape}")
    if w is not None and tuple(w.shape) != grid.shape:
        raise DimensionMismatch(f"w must have the grid's shape {grid.shape}")
    gate_spectrum(kernel, spectrum)
    scales = np.asarray(scales, dtype=np.float64)
    plans = _plans(grid, kernel, scales, mask_strategy, filter_plans, method)
    if w is not None:
        Pi, E = _sweep_w(np.asarray(u)[None], np.asarray(v)[None], np.asarray(w)[None], grid, plans, 1, None)
    else:
        Pi, E = _sweep(u, v, grid, plans, 1, None)
    k = float(L) / scales
    return CoarseGrainResult(scales.copy(), Pi[0], E[0], k, _spectrum(E[0], k, spectrum))


def coarse_grain_batch(u, v, grid: StructuredGrid, *, scales: Sequence[float], w=None,
                       kernel: AbstractFilterKernel = TopHatKernel(),
                       mask_strategy: AbstractMaskStrategy = ZeroFill(),
                       filter_plans: Optional[Sequence[PhysicalFilterPlan]] = None, L: float = 1.0,
                       spectrum: AbstractSpectrumPolicy = StrictSpectrum(), slice_masks=None,
                       method=None) -> CoarseGrainBatchResult:
    """Pipeline.coarse_grain_batch! (Pipeline.jl:686-717): u, v (and w) of shape (batch..., ny, nx) share
    the grid; the whole batch runs batch-native, one fused pass per scale (the GPU driver,
    Pipeline.jl:519-563).  `slice_masks` (batch..., ny, nx) gives every slice its own mask."""
    shp = tuple(u.shape)
    if len(shp) < 3 or shp[-2:] != grid.shape or tuple(v.shape) != shp:
        raise DimensionMismatch(f"u and v must be (batch..., {grid.ny}, {grid.nx}) and equal")
    if w is not None and tuple(w.shape) != shp:
        raise DimensionMismatch("w must match u's shape")
    bsz = shp[:-2]
    nb = int(np.prod(bsz))
    gate_spectrum(kernel, spectrum)
    scales = np.asarray(scales, dtype=np.float64)
    plans = _plans(grid, kernel, scales, mask_strategy, filter_plans, method)
    if w is not None:
        Pi, E = _sweep_w(u.reshape((nb,) + grid.shape), v.reshape((nb,) + grid.shape), w.reshape((nb,) + grid.shape),
                         grid, plans, nb, None if slice_masks is None else np.asarray(slice_masks).reshape(
                             (nb,) + grid.shape))
    else:
        Pi, E = _sweep(u.reshape((nb,) + grid.shape), v.reshape((nb,) + grid.shape), grid, plans, nb, slice_masks)
    ns = len(scales)
    k = float(L) / scales
    spec = np.stack([_spectrum(E[t], k, spectrum) for t in range(nb)])
    return CoarseGrainBatchResult(Pi.reshape(bsz + (ns,) + grid.shape), np.broadcast_to(scales, bsz + (ns,)).copy(),
                                  E.reshape(bsz + (ns,)), np.broadcast_to(k, bsz + (ns,)).copy(),
                                  spec.reshape(bsz + (ns,)), bsz)


def coarse_grain_profile(u, v, grid: StructuredGrid, **kw) -> CoarseGrainBatchResult:
    """Pipeline.coarse_grain_profile! (Pipeline.jl:991-1007): levels are a batch axis."""
    return coarse_grain_batch(u, v, grid, **kw)


def coarse_grain_slices(us: Sequence, vs: Sequence, grids: Sequence[StructuredGrid], *, scales: Sequence[float],
                        kernel: AbstractFilterKernel = TopHatKernel(),
                        mask_strategy: AbstractMaskStrategy = ZeroFill(), L: float = 1.0,
                        spectrum: AbstractSpectrumPolicy = StrictSpectrum(), method=None) -> List[CoarseGrainResult]:
    """Pipeline.coarse_grain_slices! (Pipeline.jl:866-904): each slice brings its own grid.  Slices whose
    grids differ only in their masks (levels under bathymetry) run as one batched sweep with a mask
    per slice; any other group runs per grid."""
    n = len(us)
    if len(vs) != n or len(grids) != n:
        raise DimensionMismatch("us, vs and grids must have equal length")
    gate_spectrum(kernel, spectrum)
    scales = np.asarray(scales, dtype=np.float64)
    results: List[Optional[CoarseGrainResult]] = [None] * n
    groups: List[List[int]] = []
    for t in range(n):
        for g in groups:
            if grids[g[0]].same_geometry(grids[t]):
                g.append(t)
                break
        else:
            groups.append([t])
    k = float(L) / scales
    for g in groups:
        base = grids[g[0]].with_mask(None)
        plans = _plans(base, kernel, scales, mask_strategy, None, method)
        masks = np.stack([np.ones(base.shape, np.uint8) if grids[t].mask is None else grids[t].mask.astype(np.uint8)
                          for t in g])
        u = np.stack([np.asarray(us[t]) for t in g])
        v = np.stack([np.asarray(vs[t]) for t in g])
        Pi, E = _sweep(u, v, base, plans, len(g), masks)
        for q, t in enumerate(g):
            results[t] = CoarseGrainResult(scales.copy(), Pi[q], E[q], k, _spectrum(E[q], k, spectrum))
    return results  # type: ignore[return-value]


class SnapshotStream:
    """A time series of snapshots streamed through a sweep (`cgef_pipeline_*`): every `submit` copies
    one snapshot's u, v in, sweeps it over the plans' scales and copies its Pi (nbatch, nscales, ny, nx)
    and E (nbatch, nscales) out, while neighbouring snapshots' copies and sweeps overlap on the GPU.
    Host buffers must stay alive and untouched until `drain()`; they overlap the GPU's work only when
    pinned (e.g. torch tensors from `.pin_memory()`)."""

    def __init__(self, plans: Sequence[PhysicalFilterPlan], *, nbatch: int = 1, dtype=np.float64,
                 slice_masks=None, want_pi: bool = True):
        if not plans:
            raise ArgumentError("need at least one plan")
        self.plans = list(plans)
        self.grid = plans[0].grid
        self.nbatch = int(nbatch)
        self.dtype = np.dtype(dtype)
        self.want_pi = bool(want_pi)
        code = _lib.F32 if self.dtype == np.float32 else _lib.F64
        if self.dtype not in (np.float32, np.float64):
            raise ArgumentError("dtype must be float32 or float64")
        m = None if slice_masks is None else np.ascontiguousarray(slice_masks, dtype=np.uint8)
        if m is not None and m.size != self.nbatch * self.grid.nx * self.grid.ny:
            raise DimensionMismatch("slice_masks must hold one (ny, nx) mask per slice")
        self._keep = []
        arr = (C.c_void_p * len(self.plans))(*[p.handle.value for p in self.plans])
        self._h = C.c_void_p()
        _lib.check(_lib.load().cgef_pipeline_create(C.byref(self._h), arr, len(self.plans), code, self.nbatch,
                                                    None if m is None else m.ctypes.data, int(self.want_pi)))

    def _shape_ok(self, a, shape, name, itemsize=None):
        if tuple(a.shape) != shape:
            raise DimensionMismatch(f"{name} must have shape {shape}")
        if A.is_device(a):
            raise ArgumentError(f"{name} must be host memory")
        size = a.element_size() if hasattr(a, "element_size") else a.itemsize
        if size != (self.dtype.itemsize if itemsize is None else itemsize):
            raise ArgumentError(f"{name} has the wrong element type")

    def submit(self, u, v, pi=None, energy=None) -> None:
        ny, nx = self.grid.shape
        fs = (self.nbatch, ny, nx)
        self._shape_ok(u, fs, "u")
        self._shape_ok(v, fs, "v")
        if self.want_pi:
            if pi is None:
                raise ArgumentError("this stream returns Pi: pass a (nbatch, nscales, ny, nx) buffer")
            self._shape_ok(pi, (self.nbatch, len(self.plans), ny, nx), "pi")
        if energy is not None:
            self._shape_ok(energy, (self.nbatch, len(self.plans)), "energy", itemsize=8)
        self._keep.append((u, v, pi, energy))
        _lib.check(_lib.load().cgef_pipeline_submit(self._h, A.ptr(u), A.ptr(v), None if pi is None else A.ptr(pi),
                                                    None if energy is None else A.ptr(energy)))

    def drain(self) -> None:
        _lib.check(_lib.load().cgef_pipeline_drain(self._h))
        self._keep.clear()

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value and _lib._lib is not None:
            _lib._lib.cgef_pipeline_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
