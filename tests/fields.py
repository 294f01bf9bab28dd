"""Seeded synthetic fields shared by the tests (numpy only, no GPU).

`spectral_field` restates the reference's own test generator (test/test_validation.jl:21-41):
a streamfunction with |psi_hat| = k^-(alpha+3)/2 and phases from an irrational rotation, so
E(k) ~ k^-alpha; `symbol="stencil"` makes the field divergence-free for the 3-point centred
derivative instead of the spectral one.
"""
import numpy as np


def kaxis(N, dx):
    i = np.arange(N)
    return 2 * np.pi / (N * dx) * np.where(i <= N // 2, i, i - N)


def spectral_field(N, dx, alpha, symbol="exact"):
    k = kaxis(N, dx)
    ii, jj = np.meshgrid(np.arange(1, N + 1), np.arange(1, N + 1), indexing="ij")  # Julia (i, j)
    phase = 2 * np.pi * np.mod(0.7548776662466927 * ii + 0.5698402909980532 * jj, 1.0)
    KX, KY = np.meshgrid(k, k, indexing="ij")  # KX varies with i (axis 1), KY with j (axis 2)
    kmag = np.sqrt(KX ** 2 + KY ** 2)
    with np.errstate(divide="ignore"):
        amp = np.where(kmag > 0, kmag ** (-(alpha + 3) / 2), 0.0)
    psih = amp * np.exp(1j * phase)
    psih = np.fft.fft2(np.real(np.fft.ifft2(psih)))
    sym = (lambda kk: kk) if symbol == "exact" else (lambda kk: np.sin(kk * dx) / dx)
    uh = -1j * sym(KY) * psih
    vh = 1j * sym(KX) * psih
    u = np.real(np.fft.ifft2(uh))
    v = np.real(np.fft.ifft2(vh))
    # Julia arrays are (Nx, Ny) column-major == numpy (ny, nx): transpose the (i, j) arrays.
    return np.ascontiguousarray(u.T), np.ascontiguousarray(v.T)


def fourier_slope(u, v, dx, nlo, nhi):
    """Shell-averaged KE spectrum slope (test/test_validation.jl:51-64)."""
    ut, vt = u.T, v.T
    N = ut.shape[0]
    kx = kaxis(N, dx)
    dk = 2 * np.pi / (N * dx)
    uh = np.fft.fft2(ut) / N ** 2
    vh = np.fft.fft2(vt) / N ** 2
    E = np.zeros(N // 2 + 1)
    KX, KY = np.meshgrid(kx, kx, indexing="ij")
    n = np.rint(np.sqrt(KX ** 2 + KY ** 2) / dk).astype(int)
    sel = (n >= 1) & (n <= N // 2)
    np.add.at(E, n[sel], 0.5 * (np.abs(uh[sel]) ** 2 + np.abs(vh[sel]) ** 2))
    ns = np.array([m for m in range(nlo, nhi + 1) if E[m] > 0])
    return logfit(ns.astype(float), E[ns])


def logfit(x, y):
    lx, ly = np.log10(x), np.log10(y)
    xb, yb = lx.mean(), ly.mean()
    return np.sum((lx - xb) * (ly - yb)) / np.sum((lx - xb) ** 2)
