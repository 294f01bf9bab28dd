"""The spectral method (plan_filter(method=Spectral()), the FFTW extension's filter,
ext/CoarseGrainingEnergyFluxesFFTWExt.jl:121-206) on the GPU: the reference's own known answers
(test/test_spectral.jl:2-106) through the CUDA path, and parity with the numpy oracle
(oracle/oracle_spectral.py) for filters, the flux and the sweep.

Bounds: the device transforms in FP64 in another order than numpy's pocketfft, so filtered fields agree
to ~1e-15 of their magnitude; the asserted bounds are 1e-12 (max relative) on filters, 1e-9 relative L2
on Pi and 1e-10 on the flux's fields, as for the real-space engines.
"""
import math

import numpy as np
import pytest

import cgef_b200 as cg
import oracle as O
import oracle_spectral as SP
from helpers import max_rel, oracle_grid, rel_l2

pytestmark = pytest.mark.gpu

N, ELL = 32, 4.0
X = np.arange(N) * 1.0


def cart(nx=N, ny=None, mask=None, dx=1.0, dy=None, periodic=(True, True)):
    ny = nx if ny is None else ny
    dy = dx if dy is None else dy
    return cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0, dx, nx), cg.axis(0, dy, ny), mask, periodic)


def approx_arr(a, b, rtol):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) <= rtol * max(np.linalg.norm(a), np.linalg.norm(b))


def spec_filter(field, g, kernel, strategy=cg.ZeroFill()):
    out = np.zeros(g.shape)
    cg.filter_field(out, field, g, kernel, ELL, mask_strategy=strategy, method=cg.Spectral())
    return out


def test_reference_known_answers_unmasked():
    # test_spectral.jl:13-50
    g = cart()
    kx0 = 2 * math.pi * 3 / N
    f = np.tile(np.cos(kx0 * X), (N, 1))
    out = spec_filter(f, g, cg.GaussianKernel())
    assert approx_arr(out, math.exp(-kx0 ** 2 * ELL ** 2 / 24) * f, 1e-10)
    c = np.full((N, N), 2.5)
    assert approx_arr(spec_filter(c, g, cg.GaussianKernel()), c, 1e-12)
    from scipy.special import j1
    R = ELL / 2
    th = spec_filter(f, g, cg.TopHatKernel())
    assert approx_arr(th, 2 * j1(kx0 * R) / (kx0 * R) * f, 1e-8)
    ds = np.zeros(g.shape)
    cg.filter_field(ds, f, g, cg.TopHatKernel(), ELL)  # RealSpace
    assert approx_arr(th, ds, 0.02)


def _hole():
    m = np.ones((N, N), bool)
    m[9:14, 9:14] = False
    return m


@pytest.mark.parametrize("strategy", [cg.Deformable(), cg.ZeroFill()])
def test_reference_known_answers_masked(strategy):
    # test_spectral.jl:66-79: spectral and real space agree on active cells
    mask = _hole()
    g = cart(mask=mask)
    Xg, Yg = np.meshgrid(X, X)
    rf = np.sin(2 * math.pi * 3 * Xg / N) * np.cos(2 * math.pi * 2 * Yg / N) + 0.3 * np.cos(2 * math.pi * 5 * Xg / N)
    spec = spec_filter(rf, g, cg.GaussianKernel(), strategy)
    ds = np.zeros(g.shape)
    cg.filter_field(ds, rf, g, cg.GaussianKernel(), ELL, mask_strategy=strategy)
    assert approx_arr(spec[mask], ds[mask], 1e-4)


def test_reference_known_answers_constants():
    # test_spectral.jl:80-103
    mask = _hole()
    g = cart(mask=mask)
    c = np.full((N, N), 1.7)
    cd = spec_filter(c, g, cg.GaussianKernel(), cg.Deformable())
    assert np.all(np.abs(cd - 1.7) <= 1e-6)
    cz = spec_filter(c, g, cg.GaussianKernel())
    mz = spec_filter(mask.astype(np.float64), g, cg.GaussianKernel())
    assert approx_arr(cz, 1.7 * mz, 1e-12)
    assert cz.min() < 1.7 - 1e-3
    assert 0 < mz.max() - 1 < 1e-4


def _masked_grid(nx=96, ny=80, dx=1500.0, dy=1000.0):
    m = np.ones((ny, nx), bool)
    m[20:35, 30:70] = False
    m[60:64, :] = False
    return cart(nx, ny, m, dx, dy)


@pytest.mark.parametrize("strategy", [cg.ZeroFill(), cg.Deformable()], ids=["zerofill", "deformable"])
@pytest.mark.parametrize("kernel", [cg.GaussianKernel(4.0), cg.TopHatKernel()], ids=["gaussian", "tophat"])
def test_filter_matches_oracle(kernel, strategy):
    g = _masked_grid()
    rng = np.random.default_rng(3)
    f = rng.standard_normal(g.shape)
    p = cg.plan_filter(g, kernel, 9000.0, mask_strategy=strategy, method=cg.Spectral())
    got = cg.filter_apply(None, f, p)
    k = SP.GAUSSIAN if isinstance(kernel, cg.GaussianKernel) else SP.TOPHAT
    T = SP.transfer(k, float(kernel.alpha), 9000.0, g.nx, g.ny, 1500.0, 1000.0)
    ref = SP.filter_field(f, T, g.mask, SP.DEFORMABLE if isinstance(strategy, cg.Deformable) else SP.ZEROFILL)
    assert max_rel(got, ref) < 1e-12
    # batched applies equal single ones, bit for bit (each quantity is transformed on its own)
    fb = np.stack([f, 2 * f, rng.standard_normal(g.shape)])
    gb = cg.filter_apply_batched(None, fb, p)
    assert np.array_equal(gb[0], got)
    # FP32 storage
    g32 = cg.filter_apply(None, f.astype(np.float32), p)
    assert g32.dtype == np.float32 and max_rel(g32, ref) < 1e-6


def test_fully_active_grid_needs_no_renormalisation():
    g = cart(64, 48, None, 2.0, 3.0)
    f = np.random.default_rng(4).standard_normal(g.shape)
    for st in (cg.ZeroFill(), cg.Deformable()):
        got = cg.filter_apply(None, f, cg.plan_filter(g, cg.GaussianKernel(6.0), 10.0, mask_strategy=st,
                                                      method=cg.Spectral()))
        T = SP.transfer(SP.GAUSSIAN, 6.0, 10.0, 64, 48, 2.0, 3.0)
        assert max_rel(got, SP.filter_field(f, T)) < 1e-12


@pytest.mark.parametrize("strategy", [cg.ZeroFill(), cg.Deformable()], ids=["zerofill", "deformable"])
def test_flux_matches_oracle(strategy):
    g = _masked_grid()
    rng = np.random.default_rng(5)
    u, v = rng.standard_normal(g.shape), rng.standard_normal(g.shape)
    k = cg.GaussianKernel(4.0)
    p = cg.plan_filter(g, k, 7000.0, mask_strategy=strategy, method=cg.Spectral())
    r = cg.compute_Pi_fields(u, v, g, k, 7000.0, filter_plan=p)
    T = SP.transfer(SP.GAUSSIAN, 4.0, 7000.0, g.nx, g.ny, 1500.0, 1000.0)
    op = O.Plan(oracle_grid(g), O.GAUSSIAN, 4.0, 7000.0)
    ref = SP.compute_pi(op, u, v, T, g.mask, SP.DEFORMABLE if isinstance(strategy, cg.Deformable) else SP.ZEROFILL)
    assert rel_l2(r["Pi"], ref["Pi"]) < 1e-9
    for name in ("ubar", "vbar", "tau_xx", "tau_xy", "tau_yy", "S_xx", "S_xy", "S_yy"):
        assert rel_l2(r[name], ref[name]) < 1e-10, name
    e = op.energy_from_filtered(ref["ubar"], ref["vbar"])
    assert abs(float(r["energy"][0]) - e) <= 1e-12 * abs(e)
    # masked cells: Pi and S are zero there, the filtered fields are not (the spectral filter is global)
    assert np.all(r["Pi"][~g.mask] == 0) and np.any(r["ubar"][~g.mask] != 0)


def test_sweep_and_slice_masks():
    g = _masked_grid()
    rng = np.random.default_rng(6)
    nb = 3
    U, V = rng.standard_normal((nb,) + g.shape), rng.standard_normal((nb,) + g.shape)
    k = cg.GaussianKernel(4.0)
    scales = [3000.0, 7000.0, 15000.0]
    res = cg.coarse_grain_batch(U, V, g, scales=scales, kernel=k, spectrum=cg.NoSpectrum(), method=cg.Spectral())
    T = {s: SP.transfer(SP.GAUSSIAN, 4.0, s, g.nx, g.ny, 1500.0, 1000.0) for s in scales}
    op = O.Plan(oracle_grid(g), O.GAUSSIAN, 4.0, 3000.0)
    for t in range(nb):
        for q, s in enumerate(scales):
            ref = SP.compute_pi(op, U[t], V[t], T[s], g.mask)
            assert rel_l2(res.Pi[t, q], ref["Pi"]) < 1e-9
            e = op.energy_from_filtered(ref["ubar"], ref["vbar"])
            assert abs(res.cumulative_energy[t, q] - e) <= 1e-12 * abs(e)
    # one mask per slice
    base = g.with_mask(None)
    sm = np.stack([g.mask, np.roll(g.mask, 11, axis=1), np.roll(g.mask, -7, axis=0)])
    p = cg.plan_filter(base, k, 7000.0, mask_strategy=cg.Deformable(), method=cg.Spectral())
    Pi = cg.compute_Pi(None, U, V, None, base, k, 7000.0, filter_plan=p, slice_masks=sm)
    for t in range(nb):
        gt = base.with_mask(sm[t])
        opt = O.Plan(oracle_grid(gt), O.GAUSSIAN, 4.0, 7000.0)
        ref = SP.compute_pi(opt, U[t], V[t], T[7000.0], sm[t], SP.DEFORMABLE)
        assert rel_l2(Pi[t], ref["Pi"]) < 1e-9


def test_cumulative_energy_and_w():
    g = _masked_grid()
    rng = np.random.default_rng(7)
    u, v, w = (rng.standard_normal(g.shape) for _ in range(3))
    k = cg.GaussianKernel(4.0)
    scales = [4000.0, 12000.0]
    E = cg.cumulative_energy(u, v, None, g, k, scales, method=cg.Spectral())
    Ew = cg.cumulative_energy(u, v, w, g, k, scales, method=cg.Spectral())
    op = O.Plan(oracle_grid(g), O.GAUSSIAN, 4.0, 4000.0)
    for q, s in enumerate(scales):
        T = SP.transfer(SP.GAUSSIAN, 4.0, s, g.nx, g.ny, 1500.0, 1000.0)
        ub, vb, wb = (SP.filter_field(x, T, g.mask) for x in (u, v, w))
        e = op.energy_from_filtered(ub, vb)
        assert abs(E[q] - e) <= 1e-12 * e
        assert abs(Ew[q] - (e + op.energy_from_filtered(wb, np.zeros_like(wb)))) <= 1e-12 * Ew[q]
    # the 2.5-D flux through a spectral plan: w = 0 is the 2-D flux
    p = cg.plan_filter(g, k, 8000.0, method=cg.Spectral())
    r3 = cg.compute_Pi_fields(u, v, g, k, 8000.0, filter_plan=p, w=np.zeros(g.shape))
    r2 = cg.compute_Pi_fields(u, v, g, k, 8000.0, filter_plan=p)
    assert rel_l2(r3["Pi"], r2["Pi"]) < 1e-13


def test_device_tensors_and_noalloc():
    import torch

    g = _masked_grid()
    f = np.random.default_rng(8).standard_normal(g.shape)
    p = cg.plan_filter(g, cg.GaussianKernel(4.0), 9000.0, mask_strategy=cg.Deformable(), method=cg.Spectral())
    host = cg.filter_apply(None, f, p)
    dev = cg.filter_apply(None, torch.from_numpy(f).cuda(), p)
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), host)
    L = cg.load()
    fd = torch.from_numpy(f).cuda()
    od = torch.empty_like(fd)
    cg._lib.check(L.cgef_filter_device_noalloc(p.handle, cg._lib.F64, fd.data_ptr(), od.data_ptr(), 1, None))
    torch.cuda.synchronize()
    assert np.array_equal(od.cpu().numpy(), host)
