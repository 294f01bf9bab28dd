"""Seeded synthetic inputs at the benchmark shapes (no public dataset is involved).

- cartesian_fields: doubly periodic streamfunction with |psi_hat|^2 ~ k^-5 and random phases,
  u = -dpsi/dy, v = dpsi/dx taken spectrally, scaled to an RMS speed (256^2, 1 km, 0.3 m/s).
- sphere_grid / sphere_fields: 0.25-degree global grid (cell centres), a random-phase
  spherical-harmonic streamfunction with velocity energy per degree ~ l^-3, u = -(1/R) dpsi/dphi,
  v = dpsi/dlambda / (R cos phi), plus a 0.5 m/s zonal jet at 40 S (sigma 5 degrees).
- land_mask: white noise smoothed at a 10-degree correlation scale on the sphere, land below its
  30th percentile.
- regional_levels: a 0.25-degree regional box, a smooth random bathymetry and one mask per level,
  with the Cartesian spectrum decaying as exp(-z/800 m) with depth.
"""
from __future__ import annotations

import math
from typing import Tuple

import numpy as np

from .grids import CartesianGeometry, SphericalGeometry, StructuredGrid, axis

R_EARTH = 6.371e6


def cartesian_fields(n: int = 256, dx: float = 1000.0, slope: float = 5.0, rms: float = 0.3, seed: int = 0
                     ) -> Tuple[np.ndarray, np.ndarray]:
    rng = np.random.default_rng(seed)
    k1 = 2 * np.pi * np.fft.fftfreq(n, d=dx)
    KX, KY = np.meshgrid(k1, k1)  # (ny, nx): KX varies along x (axis 1)
    kk = np.sqrt(KX ** 2 + KY ** 2)
    amp = np.zeros_like(kk)
    nz = kk > 0
    amp[nz] = kk[nz] ** (-slope / 2.0)
    psih = amp * np.exp(2j * np.pi * rng.random(kk.shape))
    psi = np.real(np.fft.ifft2(psih))
    psih = np.fft.fft2(psi)  # Hermitian
    u = np.real(np.fft.ifft2(-1j * KY * psih))
    v = np.real(np.fft.ifft2(1j * KX * psih))
    s = rms / math.sqrt(np.mean(u ** 2 + v ** 2))
    return np.ascontiguousarray(u * s), np.ascontiguousarray(v * s)


def cartesian_grid(n: int = 256, dx: float = 1000.0, periodic=(True, True), mask=None) -> StructuredGrid:
    return StructuredGrid(CartesianGeometry(), axis(0.0, dx, n), axis(0.0, dx, n), mask, periodic)


def sphere_grid(nlon: int = 1440, nlat: int = 720, mask=None, R: float = R_EARTH) -> StructuredGrid:
    d = 2 * math.pi / nlon
    dlat = math.pi / nlat
    return StructuredGrid(SphericalGeometry(R), axis(d / 2, d, nlon), axis(-math.pi / 2 + dlat / 2, dlat, nlat),
                          mask, (True, False))


def _sh_synthesis(coef: np.ndarray, lat: np.ndarray, nlon: int) -> np.ndarray:
    """f(lat, lon) = Re sum_{l,m} c_lm Pbar_l^m(sin lat) e^{i m lon} for c of shape (L+1, L+1) [l, m],
    with fully normalised associated Legendre functions by the standard three-term recurrence."""
    L = coef.shape[0] - 1
    x = np.sin(lat)
    c = np.cos(lat)
    ms = np.arange(L + 1)
    # sectoral Pbar_m^m
    pmm = np.empty((L + 1, lat.size))
    pmm[0] = 1.0
    for m in range(1, L + 1):
        pmm[m] = pmm[m - 1] * c * math.sqrt((2 * m + 1) / (2 * m))
    fm = np.zeros((L + 1, lat.size), dtype=np.complex128)  # sum over l per m
    p_lm2 = np.zeros((L + 1, lat.size))
    p_lm1 = pmm.copy()  # P_{m,m}
    fm += coef[ms, ms][:, None] * p_lm1
    # P_{m+1,m} = x sqrt(2m+3) P_mm
    p_l = np.zeros_like(p_lm1)
    for l in range(1, L + 1):
        # rows m < l are advanced to degree l
        m = ms[:l]
        if l - 1 >= 0:
            a = np.sqrt((4.0 * l * l - 1.0) / (l * l - m * m))
            b = np.sqrt(((l - 1.0) ** 2 - m * m) / (4.0 * (l - 1.0) ** 2 - 1.0))
            prev2 = np.where((m <= l - 2)[:, None], p_lm2[:l], 0.0)
            p_l[:l] = a[:, None] * (x[None, :] * p_lm1[:l] - b[:, None] * prev2)
            fm[:l] += coef[l, m][:, None] * p_l[:l]
            p_lm2[:l] = p_lm1[:l]
            p_lm1[:l] = p_l[:l]
    spec = np.zeros((lat.size, nlon), dtype=np.complex128)
    mmax = min(L, nlon // 2 - 1)
    spec[:, : mmax + 1] = fm[: mmax + 1].T
    return np.real(np.fft.ifft(spec, axis=1) * nlon)


def _random_sh(L: int, amp_l: np.ndarray, rng) -> np.ndarray:
    coef = np.zeros((L + 1, L + 1), dtype=np.complex128)
    for l in range(L + 1):
        coef[l, : l + 1] = amp_l[l] * np.exp(2j * np.pi * rng.random(l + 1)) * rng.standard_normal(l + 1)
    return coef


def sphere_fields(grid: StructuredGrid, seed: int = 0, lmax: int = 719, rms: float = 0.3, jet: float = 0.5,
                  jet_lat_deg: float = -40.0, jet_sigma_deg: float = 5.0) -> Tuple[np.ndarray, np.ndarray]:
    rng = np.random.default_rng(seed)
    lon, lat = grid.coords()
    l = np.arange(lmax + 1, dtype=np.float64)
    # velocity energy per degree ~ l^-3  =>  psi power per degree ~ l^-5 R^2; per coefficient / (2l+1)
    amp = np.zeros(lmax + 1)
    amp[1:] = np.sqrt(l[1:] ** -5.0 / (2 * l[1:] + 1))
    psi = _sh_synthesis(_random_sh(lmax, amp, rng), lat, grid.nx)
    R = grid.geometry.R
    dlat = grid.y.step
    dpsi_dphi = np.gradient(psi, dlat, axis=0, edge_order=2)
    k = np.fft.fftfreq(grid.nx, d=1.0 / grid.nx)
    dpsi_dlam = np.real(np.fft.ifft(1j * k[None, :] * np.fft.fft(psi, axis=1), axis=1))
    u = -dpsi_dphi / R
    v = dpsi_dlam / (R * np.cos(lat)[:, None])
    s = rms / math.sqrt(np.mean(u ** 2 + v ** 2))
    u *= s
    v *= s
    u += jet * np.exp(-(((np.degrees(lat) - jet_lat_deg) / jet_sigma_deg) ** 2))[:, None]
    return np.ascontiguousarray(u), np.ascontiguousarray(v)


def land_mask(grid: StructuredGrid, seed: int = 1, corr_deg: float = 10.0, land_fraction: float = 0.3) -> np.ndarray:
    """True = ocean (active).  White noise smoothed with a Gaussian of `corr_deg` on the sphere (as a
    spectral multiplier exp(-l(l+1) sigma^2 / 2) on random harmonics), land below its quantile."""
    rng = np.random.default_rng(seed)
    sig = math.radians(corr_deg)
    L = int(min(grid.ny - 1, max(8, 6.0 / sig)))
    l = np.arange(L + 1, dtype=np.float64)
    amp = np.exp(-l * (l + 1) * sig * sig / 4.0)
    _, lat = grid.coords()
    f = _sh_synthesis(_random_sh(L, amp, rng), lat, grid.nx)
    thr = np.quantile(f, land_fraction)
    return np.ascontiguousarray(f > thr)


def rigid_rotation(grid: StructuredGrid, U: float = 10.0) -> Tuple[np.ndarray, np.ndarray]:
    """Solid-body rotation u = U cos(phi), v = 0."""
    _, lat = grid.coords()
    u = np.broadcast_to(U * np.cos(lat)[:, None], grid.shape).copy()
    return u, np.zeros(grid.shape)


def regional_levels(nlat: int = 400, nlon: int = 600, nlev: int = 40, seed: int = 2, dtype=np.float32,
                    lat0_deg: float = -50.0, lon0_deg: float = 0.0):
    """Regional 0.25-degree box (non-periodic), nlev levels: returns (grid, u, v, masks, depths),
    u, v, masks of shape (nlev, nlat, nlon); level k is active where the bathymetry is deeper than z_k,
    z_k spaced so the active fraction falls from 100% to about 20%."""
    d = math.radians(0.25)
    grid = StructuredGrid(SphericalGeometry(R_EARTH), axis(math.radians(lon0_deg) + d / 2, d, nlon),
                          axis(math.radians(lat0_deg) + d / 2, d, nlat), None, (False, False))
    rng = np.random.default_rng(seed)
    # smooth random bathymetry in [0, 5000] m
    noise = rng.standard_normal((nlat, nlon))
    ky = np.fft.fftfreq(nlat)[:, None]
    kx = np.fft.fftfreq(nlon)[None, :]
    smooth = np.real(np.fft.ifft2(np.fft.fft2(noise) * np.exp(-(kx ** 2 + ky ** 2) * (2 * np.pi * 25) ** 2 / 2)))
    smooth = (smooth - smooth.min()) / (smooth.max() - smooth.min())
    depth = 5000.0 * smooth
    frac = np.linspace(1.0, 0.2, nlev)
    z = np.quantile(depth, 1.0 - frac)
    z[0] = -1.0
    masks = np.stack([depth > zk for zk in z])
    n = max(nlat, nlon)
    u2, v2 = cartesian_fields(n=n, dx=1.0, seed=seed + 10)
    u2, v2 = u2[:nlat, :nlon], v2[:nlat, :nlon]
    decay = np.exp(-np.maximum(z, 0.0) / 800.0)
    u = np.stack([u2 * a for a in decay]).astype(dtype)
    v = np.stack([v2 * a for a in decay]).astype(dtype)
    return grid, np.ascontiguousarray(u), np.ascontiguousarray(v), np.ascontiguousarray(masks), z
