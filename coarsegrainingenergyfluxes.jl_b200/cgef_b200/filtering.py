"""Filter plans and applies (Filtering.jl's public API for the real-space path).

`plan_filter` builds the footprint once and keeps it resident on the GPU, as the reference's
GPU extension does through `prepare_workspace` (Filtering.jl:2910-2912, 2931-2954); every
`filter_apply*` call then runs the CUDA engines of libcgef_b200.so.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _arrays as A
from . import _lib
from .errors import ArgumentError, DimensionMismatch
from .grids import StructuredGrid
from .kernels import AbstractFilterKernel, GaussianKernel, TopHatKernel


class AbstractMaskStrategy:
    code = -1

    def __eq__(self, other):
        return type(self) is type(other)

    def __hash__(self):
        return hash(type(self))

    def __repr__(self):
        return f"{type(self).__name__}()"


class ZeroFill(AbstractMaskStrategy):
    """Masked cells count in the denominator as zero-valued (Filtering.jl:36-48)."""

    code = _lib.ZEROFILL


class Deformable(AbstractMaskStrategy):
    """Masked cells leave numerator and denominator (Filtering.jl:50-57)."""

    code = _lib.DEFORMABLE


_ENGINES = {"auto": _lib.ENGINE_AUTO, "banded": _lib.ENGINE_BANDED, "separable": _lib.ENGINE_SEPARABLE,
            "prefixsum": _lib.ENGINE_PREFIXSUM}
_ENGINE_NAMES = {v: k for k, v in _ENGINES.items()}
_ENGINE_NAMES[_lib.ENGINE_SPECTRAL] = "spectral"


class AbstractFilterMethod:
    """How the convolution is evaluated (Filtering.jl:52-85)."""

    def __eq__(self, other):
        return type(self) is type(other)

    def __hash__(self):
        return hash(type(self))

    def __repr__(self):
        return f"{type(self).__name__}()"


class RealSpace(AbstractFilterMethod):
    """The physical-space footprint sum, any grid and mask (Filtering.jl:58-65): the banded, separable and
    prefix-sum engines."""


class Spectral(AbstractFilterMethod):
    """A periodic convolution by the kernel's transfer function (Filtering.jl:66-74, FFTWExt.jl:121-206):
    a doubly-periodic Cartesian grid only; the output is defined on masked cells too."""


class AutoMethod(AbstractFilterMethod):
    """Spectral where it is the exact filter -- a Cartesian grid periodic along both axes, with transform
    lengths the spectral engine covers -- else RealSpace (Filtering.jl:3008-3019)."""


def _smooth(n: int) -> bool:
    for r in (2, 3, 5):
        while n > 1 and n % r == 0:
            n //= r
    return n == 1


def spectral_exact(grid: StructuredGrid) -> bool:
    """Filtering._spectral_exact (Filtering.jl:2996-3004): Cartesian and periodic along both axes (the
    axes are uniform ranges by construction here)."""
    return (not grid.is_spherical) and bool(grid.periodic[0]) and bool(grid.periodic[1])


def spectral_sizes_ok(grid: StructuredGrid) -> bool:
    """The transform lengths the spectral engine covers: nx even, nx/2 and ny with prime factors 2, 3 and 5
    only, both at most 4096."""
    nx, ny = grid.nx, grid.ny
    return nx % 2 == 0 and nx <= 4096 and ny <= 4096 and _smooth(nx // 2) and _smooth(ny)


def resolve_method(grid: StructuredGrid, kernel: AbstractFilterKernel, method) -> AbstractFilterMethod:
    """Filtering._resolve_method (Filtering.jl:3012-3019); also accepts "realspace", "spectral", "auto"."""
    if method is None:
        return RealSpace()
    if isinstance(method, str):
        named = {"realspace": RealSpace(), "spectral": Spectral(), "auto": AutoMethod()}.get(method.lower())
        if named is None:
            raise ArgumentError("method must be RealSpace(), Spectral() or AutoMethod()")
        method = named
    if not isinstance(method, AbstractFilterMethod):
        raise ArgumentError("method must be RealSpace(), Spectral() or AutoMethod()")
    if isinstance(method, AutoMethod):
        return Spectral() if spectral_exact(grid) and spectral_sizes_ok(grid) else RealSpace()
    return method


def _validate_scale(scale: float) -> None:
    # Filtering.jl:2917-2922
    if not (np.isfinite(scale) and scale > 0):
        raise ArgumentError(f"filter scale must be finite and positive, got {scale}")


class PhysicalFilterPlan:
    """A prebuilt, device-resident filter (Filtering.jl:2894-2901)."""

    _engine_code = None  # set by subclasses that fix the engine

    def __init__(self, grid: StructuredGrid, kernel: AbstractFilterKernel, scale: float,
                 mask_strategy: AbstractMaskStrategy = ZeroFill(), engine: str = "auto"):
        if not isinstance(grid, StructuredGrid):
            raise ArgumentError("plan_filter needs a StructuredGrid")
        if not isinstance(kernel, (TopHatKernel, GaussianKernel)):
            raise ArgumentError(f"{type(kernel).__name__} is outside the supported path (TopHat, Gaussian)")
        _validate_scale(float(scale))
        if self._engine_code is None and engine not in _ENGINES:
            raise ArgumentError(f"engine must be one of {sorted(_ENGINES)}")
        code = self._engine_code if self._engine_code is not None else _ENGINES[engine]
        L = _lib.load()
        keep: list = []
        desc = grid._desc(keep)
        h = C.c_void_p()
        _lib.check(L.cgef_plan_create(C.byref(h), C.byref(desc), kernel.code, float(kernel.alpha), float(scale),
                                      mask_strategy.code, code))
        self._h = h
        self.grid = grid
        self.kernel = kernel
        self.scale = float(scale)
        self.strategy = mask_strategy
        info = _lib.PlanInfo()
        _lib.check(L.cgef_plan_get_info(h, C.byref(info)))
        self.info = info
        self.engine = _ENGINE_NAMES[info.engine]

    @property
    def handle(self) -> C.c_void_p:
        if self._h is None:
            raise ArgumentError("plan has been closed")
        return self._h

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib._lib.cgef_plan_destroy(h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def autotune(self, nbatch: int = 1) -> float:
        """Times the banded engine's candidate schedules on this plan's grid and keeps the fastest;
        returns the chosen split granularity (0 for the separable and prefix engines)."""
        w = C.c_double()
        _lib.check(_lib.load().cgef_plan_autotune(self.handle, int(nbatch), C.byref(w)))
        self.split_waves = w.value
        return w.value

    def set_filter_rows(self, rows: int) -> None:
        """Tile height (4 or 8 target rows per thread) of the banded engine's filter passes."""
        _lib.check(_lib.load().cgef_plan_set_filter_rows(self.handle, int(rows)))

    def schedule(self):
        """(split granularity of the flux gather, tile height of the filter passes)."""
        w, r = C.c_double(), C.c_int32()
        _lib.check(_lib.load().cgef_plan_get_schedule(self.handle, C.byref(w), C.byref(r)))
        return w.value, r.value

    def set_split_waves(self, waves: float) -> None:
        """Sets the banded schedule's split granularity (rounds of resident warps per SM)."""
        _lib.check(_lib.load().cgef_plan_set_split_waves(self.handle, float(waves)))
        self.split_waves = float(waves)

    def set_row_spectral(self, enable: bool) -> None:
        """Evaluate the banded sums through ring spectra (True) or directly (False); results agree to
        FP64 rounding.  Raises ArgumentError where the plan cannot use the spectral evaluation."""
        if enable and not self.row_spectral[0]:
            raise ArgumentError("row-spectral evaluation is not available for this plan: it needs the banded "
                                "engine, a periodic x axis or symmetric rows, and an even FFT length whose "
                                "half has no prime factor above 5")
        _lib.check(_lib.load().cgef_plan_set_row_spectral(self.handle, 1 if enable else 0))

    @property
    def footprint_build(self) -> str:
        """Where the plan's footprint weights were computed: "host" or "device" (set_footprint_build)."""
        w = C.c_int32()
        _lib.check(_lib.load().cgef_plan_get_build(self.handle, C.byref(w)))
        return "device" if w.value == _lib.BUILD_DEVICE else "host"

    @property
    def row_spectral(self):
        """(available, enabled, fft_length) of the row-spectral evaluation."""
        a, e, n = C.c_int32(), C.c_int32(), C.c_int32()
        _lib.check(_lib.load().cgef_plan_get_row_spectral(self.handle, C.byref(a), C.byref(e), C.byref(n)))
        return bool(a.value), bool(e.value), int(n.value)

    def footprint(self):
        """The banded footprint in the reference's CSR form (di, dj, w, ptr), 0-based."""
        n = int(self.info.nentries)
        nb = int(self.info.nbands)
        di = np.zeros(n, np.int32)
        dj = np.zeros(n, np.int32)
        w = np.zeros(n, np.float64)
        ptr = np.zeros(nb + 1, np.int64)
        _lib.check(_lib.load().cgef_plan_get_footprint(self.handle, di.ctypes.data, dj.ctypes.data,
                                                       w.ctypes.data, ptr.ctypes.data))
        return di, dj, w, ptr

    def band_counts(self) -> np.ndarray:
        """Footprint entries per band (banded engine), without materialising the entries."""
        nb = int(self.info.nbands)
        ptr = np.zeros(nb + 1, np.int64)
        _lib.check(_lib.load().cgef_plan_get_footprint(self.handle, None, None, None, ptr.ctypes.data))
        return np.diff(ptr)

    def __repr__(self):
        return (f"PhysicalFilterPlan(engine={self.engine}, kernel={self.kernel!r}, scale={self.scale}, "
                f"strategy={self.strategy!r})")


class SpectralFilterPlan(PhysicalFilterPlan):
    """A spectral-method plan (the FFTW extension's FFTWFilterPlan, FFTWExt.jl:19-49): the transforms and
    the transfer function Ghat(|k|, l) on the rfft grid, resident on the GPU.  Applies through the same
    calls as a real-space plan; its output is defined on masked cells too."""

    _engine_code = _lib.ENGINE_SPECTRAL

    def __init__(self, grid: StructuredGrid, kernel: AbstractFilterKernel, scale: float,
                 mask_strategy: AbstractMaskStrategy = ZeroFill()):
        if not spectral_exact(grid):
            # FFTWExt.jl:130-135
            raise ArgumentError("Spectral FFT filtering requires a doubly-periodic Cartesian grid; build it with "
                                "periodic=(True, True)")
        super().__init__(grid, kernel, scale, mask_strategy)

    def transfer(self) -> np.ndarray:
        """Ghat(|k|, l) on the rfft grid, (ny, nx // 2 + 1), as the host computed it for the device."""
        ny, nk = self.grid.ny, self.grid.nx // 2 + 1
        out = np.zeros((ny, nk), np.float64)
        _lib.check(_lib.load().cgef_plan_get_transfer(self.handle, out.ctypes.data))
        return out


def set_footprint_build(where: str = "auto") -> None:
    """Where later plans build large spherical footprints: "auto" (the default: on the device from about
    2e6 half-row weights), "host" or "device".  The entry set is decided on the host either way; see
    cgef_set_footprint_build in include/cgef_b200.h."""
    code = {"auto": _lib.BUILD_AUTO, "host": _lib.BUILD_HOST, "device": _lib.BUILD_DEVICE}.get(where)
    if code is None:
        raise ArgumentError("footprint build must be 'auto', 'host' or 'device'")
    _lib.check(_lib.load().cgef_set_footprint_build(code))


def plan_filter(grid: StructuredGrid, kernel: AbstractFilterKernel, scale: float, *,
                mask_strategy: AbstractMaskStrategy = ZeroFill(), engine: str = "auto",
                method=None) -> PhysicalFilterPlan:
    """Filtering.plan_filter (Filtering.jl:2931-2954): `method` RealSpace() (the default) dispatches the
    engine as the reference does (Gaussian on the plane -> separable, top-hat -> prefix sum, Gaussian on
    the sphere -> banded footprint); Spectral() builds a SpectralFilterPlan; AutoMethod() picks Spectral()
    where it is the exact filter."""
    m = resolve_method(grid, kernel, method)
    if isinstance(m, Spectral):
        if engine != "auto":
            raise ArgumentError("engine selects a real-space engine; it cannot be combined with Spectral()")
        _validate_scale(float(scale))
        return SpectralFilterPlan(grid, kernel, scale, mask_strategy)
    return PhysicalFilterPlan(grid, kernel, scale, mask_strategy, engine)


def _check_field(a, grid: StructuredGrid, name: str, batched: bool = False):
    shp = tuple(a.shape)
    if batched:
        if len(shp) != 3 or shp[1:] != grid.shape:
            raise DimensionMismatch(f"{name} has shape {shp}; expected (batch, {grid.ny}, {grid.nx})")
    elif shp != grid.shape:
        raise DimensionMismatch(f"{name} has shape {shp}; grid expects {grid.shape} (ny, nx)")


def filter_apply_batched(out, field, plan: PhysicalFilterPlan):
    """Filtering.filter_apply_batched! over a leading batch axis of shape (batch, ny, nx) -- the
    reference's trailing batch axis in column-major order (Filtering.jl:3286-3305).  One fused launch
    covers the whole batch."""
    _check_field(field, plan.grid, "field", batched=True)
    if out is None:
        out = A.empty_like(field)
    if tuple(out.shape) != tuple(field.shape):
        raise DimensionMismatch(f"out {tuple(out.shape)} and field {tuple(field.shape)} differ")
    L = _lib.load()
    dt = A.dtype_code(field)
    if A.dtype_code(out) != dt:
        raise ArgumentError("out and field must share a dtype")
    nb = int(field.shape[0])
    if A.is_device(field):
        _lib.check(L.cgef_filter_device(plan.handle, dt, A.ptr(field), A.ptr(out), nb, A.stream_of(field)))
    else:
        field = np.ascontiguousarray(field)
        _lib.check(L.cgef_filter(plan.handle, dt, A.ptr(field), A.ptr(out), nb))
    return out


def filter_apply(out, field, plan: PhysicalFilterPlan):
    """Filtering.filter_apply! (Filtering.jl:3242-3256) on one (ny, nx) field."""
    _check_field(field, plan.grid, "field")
    if out is None:
        out = A.empty_like(field)
    _check_field(out, plan.grid, "out")
    filter_apply_batched(out.reshape((1,) + tuple(out.shape)), field.reshape((1,) + tuple(field.shape)), plan)
    return out


def filter_apply_batch(outs: Optional[Sequence], fields: Sequence, plan: PhysicalFilterPlan) -> List:
    """Filtering.filter_apply_batch! (Filtering.jl:3360-3375): several fields, one traversal."""
    fields = list(fields)
    if outs is None:
        outs = [A.empty_like(f) for f in fields]
    outs = list(outs)
    if len(outs) != len(fields):
        raise DimensionMismatch("outs and fields must have equal length")
    for f in fields:
        _check_field(f, plan.grid, "field")
    if any(A.is_device(f) for f in fields):
        # device fields: one fused launch per field group through the batched entry point
        for o, f in zip(outs, fields):
            filter_apply(o, f, plan)
        return outs
    dt = A.dtype_code(fields[0])
    hf = [np.ascontiguousarray(f) for f in fields]
    K = len(hf)
    fin = (C.c_void_p * K)(*[f.ctypes.data for f in hf])
    fout = (C.c_void_p * K)(*[A.ptr(o) for o in outs])
    _lib.check(_lib.load().cgef_filter_batch(plan.handle, dt, fin, fout, K))
    return outs


def filter_field(out, field, grid: StructuredGrid, kernel: AbstractFilterKernel, scale: float, *,
                 mask_strategy: AbstractMaskStrategy = ZeroFill(), filter_plan: Optional[PhysicalFilterPlan] = None,
                 method=None):
    """Filtering.filter_field! (Filtering.jl:168-217, 276-290): plan (unless given) then apply."""
    plan = filter_plan if filter_plan is not None else plan_filter(grid, kernel, scale, mask_strategy=mask_strategy,
                                                                   method=method)
    return filter_apply(out, field, plan)


def filter_fields(outs, fields, grid: StructuredGrid, kernel: AbstractFilterKernel, scale: float, *,
                  mask_strategy: AbstractMaskStrategy = ZeroFill(), filter_plan: Optional[PhysicalFilterPlan] = None,
                  method=None):
    """Filtering.filter_fields!: several fields sharing one plan."""
    plan = filter_plan if filter_plan is not None else plan_filter(grid, kernel, scale, mask_strategy=mask_strategy,
                                                                   method=method)
    return filter_apply_batch(outs, fields, plan)
