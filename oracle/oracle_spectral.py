"""CPU restatement of the spectral (FFT) filter method on a doubly periodic Cartesian grid, for tests.

Test infrastructure: only tests/ and bench.py's CPU arms import it; the product never does.

The method (ext/CoarseGrainingEnergyFluxesFFTWExt.jl:121-206): the field, zeroed on masked cells, is
transformed with a 2-D real DFT, multiplied by the kernel's isotropic transfer function Ghat(|k|, l)
on the rfft grid, and transformed back.  ZeroFill stops there (filter(mask * f), no renormalisation);
Deformable multiplies by 1 / filter(mask) where |filter(mask)| >= 0.01, else by 0.  A fully active grid
skips the renormalisation.  The output is defined on every cell, masked ones included.

Transfer functions (Kernels.jl:394-406, ext/CoarseGrainingEnergyFluxesSpecialFunctionsExt.jl:10-17):
    Gaussian(alpha): exp(-k^2 l^2 / (4 alpha));   TopHat: 2 J1(k R) / (k R), R = l / 2, 1 at k = 0.
Wavenumbers (FFTWExt.jl:138-146): kx = 2 pi rfftfreq(nx, dx), ky = 2 pi fftfreq(ny, dy), dx = period / nx.

compute_pi() composes the Cartesian flux from these filtered fields exactly as the real-space path
does (Diagnostics.jl:485-548, 689-699), with the oracle's ReduceInRun derivatives (orc_ddx / orc_ddy).
"""
from __future__ import annotations

from typing import Optional

import numpy as np
from scipy.special import j1

TOPHAT, GAUSSIAN = 0, 1
ZEROFILL, DEFORMABLE = 0, 1
RENORM_FLOOR = 0.01  # FFTWExt.jl:170-172


def transfer(kernel: int, alpha: float, scale: float, nx: int, ny: int, dx: float, dy: float) -> np.ndarray:
    """Ghat(|k|, l) on the rfft grid, shape (ny, nx // 2 + 1) (FFTWExt.jl:138-146)."""
    kx = 2.0 * np.pi * np.fft.rfftfreq(nx, dx)
    ky = 2.0 * np.pi * np.fft.fftfreq(ny, dy)
    k = np.sqrt(kx[None, :] ** 2 + ky[:, None] ** 2)
    if kernel == GAUSSIAN:
        return np.exp(-(k ** 2) * scale ** 2 / (4.0 * alpha))
    x = k * (scale / 2.0)
    out = np.ones_like(x)
    nz = x != 0
    out[nz] = 2.0 * j1(x[nz]) / x[nz]
    return out


def _apply(field: np.ndarray, T: np.ndarray) -> np.ndarray:
    return np.fft.irfft2(np.fft.rfft2(field) * T, s=field.shape)


def filter_field(field: np.ndarray, T: np.ndarray, mask: Optional[np.ndarray] = None,
                 strategy: int = ZEROFILL) -> np.ndarray:
    """filter_apply! of an FFTWFilterPlan (FFTWExt.jl:184-206)."""
    f = np.asarray(field, dtype=np.float64)
    full = mask is None or bool(np.all(mask))
    if full:
        return _apply(f, T)
    m = np.asarray(mask, dtype=np.float64)
    out = _apply(m * f, T)
    if strategy == DEFORMABLE:
        out = out * inverse_renorm(m, T)
    return out


def inverse_renorm(mask: np.ndarray, T: np.ndarray) -> np.ndarray:
    """1 / filter(mask) where it is at least 0.01 in magnitude, else 0 (FFTWExt.jl:163-173)."""
    r = _apply(np.asarray(mask, dtype=np.float64), T)
    ir = np.zeros_like(r)
    big = np.abs(r) >= RENORM_FLOOR
    ir[big] = 1.0 / r[big]
    return ir


def compute_pi(oplan, u: np.ndarray, v: np.ndarray, T: np.ndarray, mask: Optional[np.ndarray],
               strategy: int = ZEROFILL) -> dict:
    """compute_Pi! on the plane through a spectral plan: the five filtered fields, tau, the strain of
    the filtered velocity (the oracle plan's ReduceInRun derivatives, which read `mask`) and
    Pi = mask ? -(Sxx txx + 2 Sxy txy + Syy tyy) : 0."""
    u = np.asarray(u, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    F = [filter_field(q, T, mask, strategy) for q in (u, v, u * u, u * v, v * v)]
    ub, vb = F[0], F[1]
    txx, txy, tyy = F[2] - ub * ub, F[3] - ub * vb, F[4] - vb * vb
    sxx = oplan.ddx(ub)
    syy = oplan.ddy(vb)
    sxy = 0.5 * (oplan.ddy(ub) + oplan.ddx(vb))
    act = np.ones(u.shape, bool) if mask is None else np.asarray(mask, bool)
    Pi = np.where(act, -(sxx * txx + 2.0 * sxy * txy + syy * tyy), 0.0)
    return {"Pi": Pi, "ubar": ub, "vbar": vb, "tau_xx": txx, "tau_xy": txy, "tau_yy": tyy,
            "S_xx": sxx, "S_xy": sxy, "S_yy": syy}
