"""GPU parity: the CUDA library (through its C ABI) against the FP64 oracle on the same seeded
inputs, plus the reference's own exactness properties (batched == per-slice, batch == per-field).

Tolerances: the device computes in FP64 like the oracle, differing only in summation order, so
filtered fields agree to ~1e-13 relative; the asserted bounds are 1e-10 on filtered fields and
1e-9 relative L2 on Pi -- four orders inside the contract's 1e-5 relative L2 for Pi.
"""
import math
import os

import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import synthetic as S
import oracle as O
from helpers import max_rel, oracle_grid, oracle_plan, rel_l2

pytestmark = pytest.mark.gpu

PI_CONTRACT = 1e-5     # relative L2 of Pi against the FP64 oracle, the path's stated bound
PI_FP64 = 1e-9         # what an FP64 device path must reach
FIELD_TOL = 1e-10
NTH = max(1, os.cpu_count() or 1)


def sphere2(mask=True, seed=5):
    g = S.sphere_grid(180, 90)
    m = S.land_mask(g, seed=seed) if mask else None
    return g.with_mask(m)


def test_banded_filter_sphere_matches_oracle():
    g = sphere2()
    rng = np.random.default_rng(0)
    f = rng.standard_normal(g.shape)
    for strat in (cg.ZeroFill(), cg.Deformable()):
        for alpha, scale in ((4.0, 5e5), (6.0, 1.5e6)):
            p = cg.plan_filter(g, cg.GaussianKernel(alpha), scale, mask_strategy=strat)
            assert p.engine == "banded"
            got = cg.filter_apply(None, f, p)
            ref = oracle_plan(g, cg.GaussianKernel(alpha), scale, strat).filter(f, NTH)
            assert max_rel(got, ref) < FIELD_TOL


def test_banded_filter_over_the_pole_matches_oracle():
    # the reference's high-latitude configuration (test/test_filtering.jl:733-768): rings close
    nlat, nlon = 60, 120
    g = cg.StructuredGrid(cg.SphericalGeometry(), cg.axis(0.0, 2 * math.pi / nlon, nlon),
                          cg.axis(-math.pi / 2 + 1e-6, (math.pi - 2e-6) / (nlat - 1), nlat), periodic=(True, False))
    lon, lat = g.coords()
    LON, LAT = np.meshgrid(lon, lat)
    fld = np.cos(3 * LON) * np.exp(-(((np.abs(LAT) - 1.40) / 0.12) ** 2))
    p = cg.plan_filter(g, cg.GaussianKernel(6.0), 3.0e6)
    got = cg.filter_apply(None, fld, p)
    ref = oracle_plan(g, cg.GaussianKernel(6.0), 3.0e6).filter(fld, NTH)
    assert max_rel(got, ref) < FIELD_TOL


@pytest.mark.parametrize("periodic", [(True, True), (False, False)])
@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
def test_separable_filter_matches_oracle(periodic, strat):
    n = 96
    m = np.ones((n, n), bool)
    m[30:50, 40:70] = False
    g = cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0, 1000.0, n), cg.axis(0, 1500.0, n), m, periodic)
    f = np.random.default_rng(1).standard_normal(g.shape)
    p = cg.plan_filter(g, cg.GaussianKernel(4.0), 8000.0, mask_strategy=strat)
    assert p.engine == "separable"
    got = cg.filter_apply(None, f, p)
    ref = oracle_plan(g, cg.GaussianKernel(4.0), 8000.0, strat).filter(f)
    assert max_rel(got, ref) < FIELD_TOL


@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
def test_banded_engine_on_a_cartesian_grid_matches_oracle(strat):
    n = 80
    m = np.ones((n, n), bool)
    m[10:20, 10:60] = False
    g = cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0, 1000.0, n), cg.axis(0, 1000.0, n), m, (True, False))
    f = np.random.default_rng(2).standard_normal(g.shape)
    p = cg.plan_filter(g, cg.GaussianKernel(6.0), 7000.0, mask_strategy=strat, engine="banded")
    got = cg.filter_apply(None, f, p)
    ref = oracle_plan(g, cg.GaussianKernel(6.0), 7000.0, strat, O.ENGINE_BANDED).filter(f)
    assert max_rel(got, ref) < FIELD_TOL


@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
def test_prefix_tophat_matches_oracle(strat):
    g = sphere2()
    f = np.random.default_rng(3).standard_normal(g.shape)
    p = cg.plan_filter(g, cg.TopHatKernel(), 9e5, mask_strategy=strat)
    assert p.engine == "prefixsum"
    got = cg.filter_apply(None, f, p)
    ref = oracle_plan(g, cg.TopHatKernel(), 9e5, strat).filter(f)
    assert max_rel(got, ref) < FIELD_TOL
    n = 70
    m = np.ones((n, n), bool)
    m[:, 50:] = False
    gc = cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0, 1000.0, n), cg.axis(0, 1000.0, n), m)
    fc = np.random.default_rng(4).standard_normal(gc.shape)
    pc = cg.plan_filter(gc, cg.TopHatKernel(), 9000.0, mask_strategy=strat)
    assert max_rel(cg.filter_apply(None, fc, pc), oracle_plan(gc, cg.TopHatKernel(), 9000.0, strat).filter(fc)) < FIELD_TOL


def _pi_parity(g, kernel, scale, u, v, strat=cg.ZeroFill(), tol=PI_FP64):
    r = cg.compute_Pi_fields(u, v, g, kernel, scale, mask_strategy=strat)
    ref = oracle_plan(g, kernel, scale, strat).compute_pi(u, v, NTH)
    for k in ("ubar", "vbar", "tau_xx", "tau_xy", "tau_yy", "S_xx", "S_xy", "S_yy"):
        assert rel_l2(r[k], ref[k]) < FIELD_TOL * 10, k
    e = rel_l2(r["Pi"], ref["Pi"])
    assert e < tol and e < PI_CONTRACT
    op = oracle_plan(g, kernel, scale, strat)
    e_ref = op.energy_from_filtered(ref["ubar"], ref["vbar"])
    assert float(r["energy"][0]) == pytest.approx(e_ref, rel=1e-12)
    return r, ref


@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
def test_compute_pi_sphere_banded_matches_oracle(strat):
    g = sphere2()
    u, v = S.sphere_fields(g, seed=7, lmax=89)
    _pi_parity(g, cg.GaussianKernel(4.0), 5e5, u, v, strat)


@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
def test_compute_pi_sphere_banded_alpha6_matches_oracle(strat):
    # the narrower Gaussian (Kernels.jl:59-62, radius 1.959 l)
    g = sphere2(seed=6)
    u, v = S.sphere_fields(g, seed=17, lmax=89)
    _pi_parity(g, cg.GaussianKernel(6.0), 7e5, u, v, strat)


@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
def test_compute_pi_cartesian_alpha6_matches_oracle(strat):
    n = 96
    u, v = S.cartesian_fields(n=n, seed=4)
    m = np.ones((n, n), bool)
    m[20:40, 30:70] = False
    g = S.cartesian_grid(n, 1000.0, (True, False), m)
    _pi_parity(g, cg.GaussianKernel(6.0), 7000.0, u, v, strat)


def test_filter_alpha6_batched_matches_oracle():
    g = sphere2(seed=9)
    rng = np.random.default_rng(6)
    f = rng.standard_normal((3,) + g.shape)
    p = cg.plan_filter(g, cg.GaussianKernel(6.0), 9e5)
    got = cg.filter_apply_batched(None, f, p)
    op = oracle_plan(g, cg.GaussianKernel(6.0), 9e5)
    for t in range(3):
        assert max_rel(got[t], op.filter(f[t])) < FIELD_TOL


def test_compute_pi_sphere_tophat_matches_oracle():
    g = sphere2()
    u, v = S.sphere_fields(g, seed=8, lmax=89)
    _pi_parity(g, cg.TopHatKernel(), 8e5, u, v)


@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
def test_compute_pi_cartesian_separable_matches_oracle(strat):
    n = 128
    u, v = S.cartesian_fields(n=n)
    m = np.ones((n, n), bool)
    m[:, 100:] = False
    g = S.cartesian_grid(n, 1000.0, (True, True), m)
    _pi_parity(g, cg.GaussianKernel(4.0), 8000.0, u, v, strat)


def test_compute_pi_config0_cartesian_256():
    """256^2 doubly periodic, dx = 1 km, Gaussian alpha=4, l = 8 km, ZeroFill, no mask."""
    u, v = S.cartesian_fields()
    g = S.cartesian_grid()
    r, ref = _pi_parity(g, cg.GaussianKernel(4.0), 8000.0, u, v)
    rho0 = 1025.0
    assert rel_l2(rho0 * r["Pi"], rho0 * ref["Pi"]) < PI_FP64


def test_rigid_rotation_sphere_pi_is_zero():
    """Solid-body rotation u = U cos(phi): Pi = 0 up to the 3-node stencil's O(h^2) error in the
    strain of ubar (test/test_grids.jl:167-179 asserts |Pi| < 1e-6 at U = 5, l = 500 km)."""
    g = S.sphere_grid(360, 180)
    u, v = S.rigid_rotation(g, U=10.0)
    Pi = cg.compute_Pi(None, u, v, None, g, cg.GaussianKernel(4.0), 4e5)
    ref = oracle_plan(g, cg.GaussianKernel(4.0), 4e5).compute_pi(u, v, NTH)["Pi"]
    uf, vf = S.sphere_fields(g, seed=3, lmax=179)
    Pf = cg.compute_Pi(None, uf, vf, None, g, cg.GaussianKernel(4.0), 4e5)
    # Both the device and the oracle return rounding noise (~1e-20 W/kg here), ten orders below a
    # turbulent field's flux on the same grid, so the two are compared by size, not value.
    assert np.max(np.abs(Pi)) < 1e-6
    assert np.max(np.abs(Pi)) < 1e-9 * np.max(np.abs(Pf))
    assert np.max(np.abs(ref)) < 1e-9 * np.max(np.abs(Pf))


def test_batched_apply_equals_per_slice_exactly():
    # test/test_backends.jl:555-592: the fused batched apply is exactly the per-slice loop
    g = sphere2()
    rng = np.random.default_rng(9)
    F = rng.standard_normal((3,) + g.shape)
    p = cg.plan_filter(g, cg.GaussianKernel(4.0), 6e5)
    out = cg.filter_apply_batched(None, F, p)
    for t in range(3):
        assert np.array_equal(out[t], cg.filter_apply(None, F[t].copy(), p))


def test_filter_apply_batch_equals_per_field_exactly():
    # test/test_filtering.jl:377-470: batch apply bit-identical to per-field apply
    g = sphere2()
    rng = np.random.default_rng(10)
    fs = [rng.standard_normal(g.shape) for _ in range(6)]
    p = cg.plan_filter(g, cg.GaussianKernel(4.0), 6e5, mask_strategy=cg.Deformable())
    outs = cg.filter_apply_batch(None, fs, p)
    for f, o in zip(fs, outs):
        assert np.array_equal(o, cg.filter_apply(None, f, p))


def test_batched_pi_equals_per_slice_and_oracle():
    # test/test_backends.jl:694-793: batched compute_Pi / energy == per-slice
    g = sphere2()
    us, vs = zip(*[S.sphere_fields(g, seed=20 + t, lmax=60) for t in range(3)])
    U, V = np.stack(us), np.stack(vs)
    E = np.empty(3)
    Pi = cg.compute_Pi(None, U, V, None, g, cg.GaussianKernel(4.0), 5e5, energy=E)
    for t in range(3):
        e1 = np.empty(1)
        P1 = cg.compute_Pi(None, us[t], vs[t], None, g, cg.GaussianKernel(4.0), 5e5, energy=e1)
        assert np.array_equal(Pi[t], P1)
        assert E[t] == e1[0]


def test_coarse_grain_sweep_matches_oracle():
    g = sphere2()
    u, v = S.sphere_fields(g, seed=11, lmax=89)
    scales = [3e5, 6e5, 1.2e6]
    res = cg.coarse_grain(u, v, g, scales=scales, kernel=cg.GaussianKernel(4.0))
    ref = O.coarse_grain(oracle_grid(g), u, v, scales, O.GAUSSIAN, 4.0, O.ZEROFILL, 1.0, NTH)
    for s in range(len(scales)):
        assert rel_l2(res.Pi[s], ref["Pi"][s]) < PI_FP64
    np.testing.assert_allclose(res.cumulative_energy, ref["cumulative_energy"], rtol=1e-12)
    np.testing.assert_allclose(res.filtering_spectrum, ref["filtering_spectrum"], rtol=1e-9)


def test_cumulative_energy_matches_oracle():
    g = sphere2()
    u, v = S.sphere_fields(g, seed=12, lmax=89)
    scales = [2e5, 4e5, 8e5, 1.6e6]
    got = cg.cumulative_energy(u, v, None, g, cg.GaussianKernel(4.0), scales)
    ref = O.cumulative_energy(oracle_grid(g), u, v, O.GAUSSIAN, 4.0, scales, O.ZEROFILL, NTH)
    np.testing.assert_allclose(got, ref, rtol=1e-12)
    k, Et = cg.filtering_spectrum(u, v, None, g, cg.GaussianKernel(4.0), scales)
    np.testing.assert_allclose(Et, O.spectral_density(ref, 1.0 / np.asarray(scales)), rtol=1e-9)
    with pytest.raises(cg.ArgumentError):
        cg.filtering_spectrum(u, v, None, g, cg.TopHatKernel(), scales)


def test_derivatives_match_oracle():
    g = sphere2()
    f = np.random.default_rng(13).standard_normal(g.shape)
    op = oracle_plan(g, cg.GaussianKernel(4.0), 5e5)
    np.testing.assert_allclose(cg.ddx(None, f, g), op.ddx(f), rtol=1e-13, atol=1e-13 * np.max(np.abs(op.ddx(f))))
    np.testing.assert_allclose(cg.ddy(None, f, g), op.ddy(f), rtol=1e-13, atol=1e-13 * np.max(np.abs(op.ddy(f))))


def test_slices_with_per_level_masks_fp32_match_oracle():
    """Regional levels with one mask per level, FP32 storage (coarse_grain_slices! semantics)."""
    grid, U, V, M, _ = S.regional_levels(nlat=60, nlon=80, nlev=4)
    scales = [5e4, 1e5]
    grids = [grid.with_mask(M[k]) for k in range(4)]
    res = cg.coarse_grain_slices(list(U), list(V), grids, scales=scales, kernel=cg.GaussianKernel(4.0))
    for k in range(4):
        ref = O.coarse_grain(oracle_grid(grid, M[k]), U[k].astype(np.float64), V[k].astype(np.float64), scales,
                             O.GAUSSIAN, 4.0, O.ZEROFILL, 1.0, NTH)
        assert res[k].Pi.dtype == np.float32
        for s in range(2):
            # FP32 storage of the output: relative L2 at float32 rounding
            assert rel_l2(res[k].Pi[s], ref["Pi"][s]) < 1e-6
        np.testing.assert_allclose(res[k].cumulative_energy, ref["cumulative_energy"], rtol=1e-10)


def test_device_tensors_match_host_path():
    torch = pytest.importorskip("torch")
    g = sphere2()
    u, v = S.sphere_fields(g, seed=14, lmax=60)
    host = cg.compute_Pi(None, u, v, None, g, cg.GaussianKernel(4.0), 5e5)
    du, dv = torch.from_numpy(u).cuda(), torch.from_numpy(v).cuda()
    dev = cg.compute_Pi(None, du, dv, None, g, cg.GaussianKernel(4.0), 5e5)
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), host)


def test_config1_full_size_pi_matches_oracle():
    """0.25-degree global sphere, 1440 x 720, Gaussian alpha=4, l = 100 km, ZeroFill, ~30% land."""
    g = S.sphere_grid()
    g = g.with_mask(S.land_mask(g))
    u, v = S.sphere_fields(g, seed=0)
    r = cg.compute_Pi_fields(u, v, g, cg.GaussianKernel(4.0), 1e5)
    ref = oracle_plan(g, cg.GaussianKernel(4.0), 1e5).compute_pi(u, v, NTH)
    act = g.mask
    errs = {k: rel_l2(r[k], ref[k], act) for k in ("Pi", "ubar", "vbar", "tau_xx", "tau_xy", "tau_yy")}
    assert errs["Pi"] < PI_FP64 and errs["Pi"] < PI_CONTRACT, errs
    for k in ("ubar", "vbar", "tau_xx", "tau_xy", "tau_yy"):
        assert errs[k] < 1e-10, errs
