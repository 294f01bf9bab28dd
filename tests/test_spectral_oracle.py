"""Pins the spectral-method oracle (oracle/oracle_spectral.py) against the reference's own tests of its
FFTW spectral filter (test/test_spectral.jl:2-106), restated on the same grid: 32 x 32 cells of 1 m,
doubly periodic, Gaussian alpha = 6 and top-hat at l = 4 m.  Julia's (x, y) arrays are numpy (y, x)
here, and its 1-based index ranges 0-based.  No GPU is needed.

Julia's `a ≈ b rtol = r` on arrays is norm(a - b) <= r * max(norm(a), norm(b)); `approx_arr` restates it.
"""
import math

import numpy as np
import pytest

import oracle as O
import oracle_spectral as SP

N, DX, ELL = 32, 1.0, 4.0
L = N * DX
X = np.arange(N) * DX


def approx_arr(a, b, rtol):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) <= rtol * max(np.linalg.norm(a), np.linalg.norm(b))


def T(kernel, alpha=6.0, ell=ELL):
    return SP.transfer(kernel, alpha, ell, N, N, DX, DX)


def mode_field(m=3):
    kx0 = 2 * math.pi * m / L
    return kx0, np.tile(np.cos(kx0 * X), (N, 1))  # field[j, i] = cos(kx0 x_i)


def test_fourier_mode_is_an_eigenfunction():
    # test_spectral.jl:13-20 (Gaussian alpha = 6: Ghat = exp(-k^2 l^2 / 24))
    kx0, f = mode_field()
    out = SP.filter_field(f, T(SP.GAUSSIAN))
    assert approx_arr(out, math.exp(-kx0 ** 2 * ELL ** 2 / 24) * f, 1e-10)


def test_constant_is_preserved():
    # test_spectral.jl:22-26: Ghat(0) = 1
    c = np.full((N, N), 2.5)
    assert approx_arr(SP.filter_field(c, T(SP.GAUSSIAN)), c, 1e-12)


def test_tophat_mode_uses_the_bessel_transfer_and_tracks_real_space():
    # test_spectral.jl:36-50: Ghat = 2 J1(kR)/(kR), R = l/2, and RealSpace within 2 %
    from scipy.special import j1

    kx0, f = mode_field()
    R = ELL / 2
    g = 2 * j1(kx0 * R) / (kx0 * R)
    out = SP.filter_field(f, T(SP.TOPHAT))
    assert approx_arr(out, g * f, 1e-8)
    grid = O.Grid(O.CART, N, N, 0.0, DX, 0.0, DX, 6.371e6, True, True)
    ds = O.Plan(grid, O.TOPHAT, 0.0, ELL).filter(f)
    assert approx_arr(out, ds, 0.02)


def _masked():
    mask = np.ones((N, N), bool)
    mask[9:14, 9:14] = False  # Julia mask[10:14, 10:14]
    return mask


@pytest.mark.parametrize("strategy", [SP.DEFORMABLE, SP.ZEROFILL])
def test_masked_spectral_matches_real_space_on_active_cells(strategy):
    # test_spectral.jl:66-79: the same normalised-convolution identity, active cells, rtol 1e-4
    mask = _masked()
    Xg, Yg = np.meshgrid(X, X)  # Xg[j, i] = x_i
    rf = np.sin(2 * math.pi * 3 * Xg / L) * np.cos(2 * math.pi * 2 * Yg / L) + 0.3 * np.cos(2 * math.pi * 5 * Xg / L)
    spec = SP.filter_field(rf, T(SP.GAUSSIAN), mask, strategy)
    grid = O.Grid(O.CART, N, N, 0.0, DX, 0.0, DX, 6.371e6, True, True, mask)
    st = O.DEFORMABLE if strategy == SP.DEFORMABLE else O.ZEROFILL
    ds = O.Plan(grid, O.GAUSSIAN, 6.0, ELL, st).filter(rf)
    assert approx_arr(spec[mask], ds[mask], 1e-4)


def test_deformable_keeps_a_constant_everywhere():
    # test_spectral.jl:80-85
    mask = _masked()
    c = np.full((N, N), 1.7)
    out = SP.filter_field(c, T(SP.GAUSSIAN), mask, SP.DEFORMABLE)
    assert np.all(np.abs(out - 1.7) <= 1e-6)


def test_zerofill_is_the_unrenormalised_numerator_and_overshoots():
    # test_spectral.jl:87-103
    mask = _masked()
    c = np.full((N, N), 1.7)
    cz = SP.filter_field(c, T(SP.GAUSSIAN), mask)
    mz = SP.filter_field(mask.astype(np.float64), T(SP.GAUSSIAN), mask)
    assert approx_arr(cz, 1.7 * mz, 1e-12)
    assert cz.min() < 1.7 - 1e-3
    assert 0 < mz.max() - 1 < 1e-4
    grid = O.Grid(O.CART, N, N, 0.0, DX, 0.0, DX, 6.371e6, True, True, mask)
    mr = O.Plan(grid, O.GAUSSIAN, 6.0, ELL).filter(mask.astype(np.float64))
    assert mr.max() <= 1 + 1e-12


def test_transfer_grid_follows_rfftfreq_and_fftfreq():
    # FFTWExt.jl:138-146 on a non-square grid with different spacings
    nx, ny, dx, dy = 12, 10, 2.0, 3.0
    t = SP.transfer(SP.GAUSSIAN, 4.0, 7.0, nx, ny, dx, dy)
    assert t.shape == (ny, nx // 2 + 1)
    for (jj, ii) in ((0, 0), (3, 2), (7, 6), (5, 0)):
        ky = 2 * math.pi * (jj if jj < (ny + 1) // 2 else jj - ny) / (ny * dy)
        kx = 2 * math.pi * ii / (nx * dx)
        assert t[jj, ii] == pytest.approx(math.exp(-(kx * kx + ky * ky) * 49.0 / 16.0), rel=1e-14)
