"""ctypes binding of the CPU FP64 oracle (``cgef_oracle.c``).

TEST INFRASTRUCTURE ONLY.  The oracle restates the reference's arithmetic on the CPU so that
the CUDA library can be checked against it; ``bench.py`` also times it as the CPU baseline.
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` use this module, and never as
the thing that is measured or shipped.

Arrays are numpy float64 of shape ``(ny, nx)`` -- the reference's column-major ``(Nx, Ny)``
with the longitude index fastest.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "libcgef_oracle.so")

CART, SPHERE = 0, 1
TOPHAT, GAUSSIAN = 0, 1
ZEROFILL, DEFORMABLE = 0, 1
ENGINE_AUTO, ENGINE_BANDED, ENGINE_SEPARABLE, ENGINE_PREFIXSUM = 0, 1, 2, 3

_lib = None


def build() -> str:
    """Compile the oracle in place (``make -C oracle``)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.orc_plan_new.restype = C.c_void_p
        L.orc_plan_new.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_double, C.c_double,
                                   C.c_int, C.c_int]
        L.orc_plan_new_rows.restype = C.c_void_p
        L.orc_plan_new_rows.argtypes = L.orc_plan_new.argtypes + [C.c_void_p]
        L.orc_plan_free.argtypes = [C.c_void_p]
        L.orc_plan_engine.argtypes = [C.c_void_p]
        L.orc_plan_nentries.argtypes = [C.c_void_p]
        L.orc_plan_nentries.restype = C.c_int64
        L.orc_plan_nbands.argtypes = [C.c_void_p]
        L.orc_plan_footprint.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_plan_separable_lims.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_filter_batch.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
        L.orc_ddx.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_ddy.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_compute_pi.argtypes = [C.c_void_p] + [C.c_void_p] * 11 + [C.c_int]
        L.orc_compute_pi_w.argtypes = [C.c_void_p] * 6 + [C.c_int]
        L.orc_active_area.argtypes = [C.c_void_p]
        L.orc_active_area.restype = C.c_double
        L.orc_energy_from_filtered.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]
        L.orc_energy_from_filtered.restype = C.c_double
        L.orc_cumulative_energy_one.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.orc_cumulative_energy_one.restype = C.c_double
        L.orc_spectral_density.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        L.orc_kernel_radius.argtypes = [C.c_int, C.c_double, C.c_double]
        L.orc_kernel_radius.restype = C.c_double
        L.orc_kernel_weight.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double]
        L.orc_kernel_weight.restype = C.c_double
        L.orc_max_threads.restype = C.c_int
        L.orc_coords.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_count_entries.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]
        L.orc_count_entries.restype = C.c_int64
        L.orc_closure_nparam.restype = C.c_int
        L.orc_bf16.argtypes = [C.c_float]
        L.orc_bf16.restype = C.c_float
        L.orc_closure_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
        L.orc_closure_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
        L.orc_closure_adamw.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float,
                                        C.c_float, C.c_float, C.c_float, C.c_float]
        _ = dp
        _lib = L
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


@dataclass
class Grid:
    """Uniform structured grid: x_i = x0 + i*dx, y_j = y0 + j*dy (radians on the sphere)."""
    geometry: int
    nx: int
    ny: int
    x0: float
    dx: float
    y0: float
    dy: float
    R: float = 6.371e6
    periodic_x: bool = False
    periodic_y: bool = False
    mask: Optional[np.ndarray] = None  # (ny, nx) bool/uint8, None = all active

    def mask_u8(self) -> Optional[np.ndarray]:
        if self.mask is None:
            return None
        return np.ascontiguousarray(self.mask, dtype=np.uint8)


class Plan:
    """One oracle filter plan (engine chosen as the reference dispatches, unless forced).

    `rows` (banded engine): None, or the target rows to evaluate; every other row of a filter output
    reads 0 and only those rows' footprint bands are built.  Use `rows_for_pi` to widen the rows a
    test compares by the strain stencil's reach, so Pi at those rows equals the full plan's.
    """

    def __init__(self, grid: Grid, kernel: int, alpha: float, ell: float, strategy: int = ZEROFILL,
                 engine: int = ENGINE_AUTO, rows: Optional[Sequence[int]] = None):
        self.grid = grid
        self._mask = grid.mask_u8()
        self._rows = None
        if rows is not None:
            self._rows = np.zeros(grid.ny, np.uint8)
            self._rows[np.asarray(rows, dtype=np.int64)] = 1
        self.h = lib().orc_plan_new_rows(grid.geometry, grid.nx, grid.ny, grid.x0, grid.dx, grid.y0, grid.dy,
                                         grid.R, int(grid.periodic_x), int(grid.periodic_y), _ptr(self._mask),
                                         kernel, alpha, ell, strategy, engine, _ptr(self._rows))
        self.kernel, self.alpha, self.ell, self.strategy = kernel, alpha, ell, strategy

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().orc_plan_free(h)
            self.h = None

    def coords(self):
        x = np.zeros(self.grid.nx)
        y = np.zeros(self.grid.ny)
        lib().orc_coords(self.h, _ptr(x), _ptr(y))
        return x, y

    @property
    def engine(self) -> int:
        return lib().orc_plan_engine(self.h)

    def footprint(self):
        n = lib().orc_plan_nentries(self.h)
        nb = lib().orc_plan_nbands(self.h)
        di = np.zeros(n, np.int32)
        dj = np.zeros(n, np.int32)
        w = np.zeros(n, np.float64)
        ptr = np.zeros(nb + 1, np.int64)
        lib().orc_plan_footprint(self.h, _ptr(di), _ptr(dj), _ptr(w), _ptr(ptr))
        return di, dj, w, ptr

    def filter_batch(self, fields: Sequence[np.ndarray], nthreads: int = 1):
        fs = [_f64(f) for f in fields]
        outs = [np.zeros_like(f) for f in fs]
        K = len(fs)
        fin = (C.c_void_p * K)(*[f.ctypes.data for f in fs])
        fout = (C.c_void_p * K)(*[o.ctypes.data for o in outs])
        lib().orc_filter_batch(self.h, K, fin, fout, nthreads)
        return outs

    def filter(self, field: np.ndarray, nthreads: int = 1) -> np.ndarray:
        return self.filter_batch([field], nthreads)[0]

    def ddx(self, f: np.ndarray) -> np.ndarray:
        f = _f64(f)
        out = np.zeros_like(f)
        lib().orc_ddx(self.h, _ptr(f), _ptr(out))
        return out

    def ddy(self, f: np.ndarray) -> np.ndarray:
        f = _f64(f)
        out = np.zeros_like(f)
        lib().orc_ddy(self.h, _ptr(f), _ptr(out))
        return out

    def compute_pi(self, u: np.ndarray, v: np.ndarray, nthreads: int = 1) -> dict:
        u, v = _f64(u), _f64(v)
        names = ["Pi", "ubar", "vbar", "tau_xx", "tau_xy", "tau_yy", "S_xx", "S_xy", "S_yy"]
        out = {k: np.zeros_like(u) for k in names}
        lib().orc_compute_pi(self.h, _ptr(u), _ptr(v), *[_ptr(out[k]) for k in names], nthreads)
        return out

    W_OUTPUTS = ["ubar", "vbar", "wbar", "tau_xx", "tau_xy", "tau_yy", "tau_xz", "tau_yz", "tau_zz",
                 "S_xx", "S_xy", "S_yy", "S_xz", "S_yz"]

    def compute_pi_w(self, u: np.ndarray, v: np.ndarray, w: np.ndarray, nthreads: int = 1) -> dict:
        """compute_Pi! with the vertical velocity (the 2.5-D path): Pi and the 14 local fields."""
        u, v, w = _f64(u), _f64(v), _f64(w)
        out = {k: np.zeros_like(u) for k in ["Pi"] + self.W_OUTPUTS}
        arr = (C.c_void_p * 14)(*[out[k].ctypes.data for k in self.W_OUTPUTS])
        lib().orc_compute_pi_w(self.h, _ptr(u), _ptr(v), _ptr(w), _ptr(out["Pi"]), arr, nthreads)
        return out

    def active_area(self) -> float:
        return lib().orc_active_area(self.h)

    def energy_from_filtered(self, ubar: np.ndarray, vbar: np.ndarray, total_area: Optional[float] = None) -> float:
        ta = self.active_area() if total_area is None else total_area
        return lib().orc_energy_from_filtered(self.h, _ptr(_f64(ubar)), _ptr(_f64(vbar)), ta)

    def cumulative_energy_one(self, u: np.ndarray, v: np.ndarray, nthreads: int = 1) -> float:
        return lib().orc_cumulative_energy_one(self.h, _ptr(_f64(u)), _ptr(_f64(v)), nthreads)


def rows_for_pi(rows: Sequence[int], ny: int, periodic_y: bool = False) -> np.ndarray:
    """The rows a row-subset plan must evaluate for compute_pi's Pi to be exact at `rows`: the
    3-node ReduceInRun stencil along y reads up to two rows either side."""
    out = set()
    for j in rows:
        for d in range(-2, 3):
            jj = j + d
            if periodic_y:
                out.add(jj % ny)
            elif 0 <= jj < ny:
                out.add(jj)
    return np.array(sorted(out), dtype=np.int64)


def kernel_radius(kernel: int, alpha: float, ell: float) -> float:
    return lib().orc_kernel_radius(kernel, alpha, ell)


def kernel_weight(kernel: int, alpha: float, d: float, ell: float) -> float:
    return lib().orc_kernel_weight(kernel, alpha, d, ell)


def spectral_density(Cv: np.ndarray, k: np.ndarray) -> np.ndarray:
    Cv, k = _f64(Cv), _f64(k)
    g = np.zeros_like(Cv)
    lib().orc_spectral_density(_ptr(Cv), _ptr(k), len(Cv), _ptr(g))
    return g


def cumulative_energy(grid: Grid, u, v, kernel: int, alpha: float, scales, strategy: int = ZEROFILL,
                      nthreads: int = 1) -> np.ndarray:
    return np.array([Plan(grid, kernel, alpha, float(s), strategy).cumulative_energy_one(u, v, nthreads)
                     for s in scales])


def coarse_grain(grid: Grid, u, v, scales, kernel: int = GAUSSIAN, alpha: float = 6.0, strategy: int = ZEROFILL,
                 L: float = 1.0, nthreads: int = 1) -> dict:
    """Pipeline.coarse_grain! (Pipeline.jl:412-468): Pi per scale, E(l) from the filtered
    local velocities that compute_Pi! leaves behind, k_l = L/l and the spectral density."""
    scales = np.asarray(scales, dtype=np.float64)
    Pis, E = [], []
    for s in scales:
        p = Plan(grid, kernel, alpha, float(s), strategy)
        r = p.compute_pi(u, v, nthreads)
        Pis.append(r["Pi"])
        E.append(p.energy_from_filtered(r["ubar"], r["vbar"]))
    E = np.array(E)
    k = L / scales
    return {"Pi": np.stack(Pis), "cumulative_energy": E, "wavenumber": k, "filtering_spectrum": spectral_density(E, k)}


def count_entries(grid: Grid, kernel: int, alpha: float, ell: float) -> int:
    """Entries of the banded footprint (all bands), without building it."""
    return int(lib().orc_count_entries(grid.geometry, grid.nx, grid.ny, grid.x0, grid.dx, grid.y0, grid.dy, grid.R,
                                       int(grid.periodic_x), int(grid.periodic_y), kernel, alpha, ell))


def max_threads() -> int:
    return lib().orc_max_threads()


# ---- learned closure (closure_oracle.c): the checker of the tensor-core MLP kernels ----
def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def closure_nparam() -> int:
    return int(lib().orc_closure_nparam())


def closure_forward(params, x) -> np.ndarray:
    """y (n, 3) of the MLP with BF16 operands and FP32 sums for features x (n, 5)."""
    P, X = _f32(params), _f32(x)
    y = np.empty((X.shape[0], 3), np.float32)
    lib().orc_closure_forward(_ptr(P), _ptr(X), X.shape[0], _ptr(y))
    return y


def closure_grad(params, x, t):
    """(gradient (float64, nparam), loss) of mean_i sum_o (y_io - t_io)^2."""
    P, X, T = _f32(params), _f32(x), _f32(t)
    g = np.empty(closure_nparam(), np.float64)
    loss = C.c_double()
    lib().orc_closure_grad(_ptr(P), _ptr(X), _ptr(T), X.shape[0], _ptr(g), C.byref(loss))
    return g, loss.value


def closure_adamw(params, m, v, g, step, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
    """One AdamW step in place on float32 arrays (weight decay on weight matrices only)."""
    for a in (params, m, v):
        assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    G = _f32(g)
    lib().orc_closure_adamw(_ptr(params), _ptr(m), _ptr(v), _ptr(G), int(step), lr, b1, b2, eps, wd)
