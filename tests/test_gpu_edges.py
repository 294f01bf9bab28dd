"""Edge cases on the GPU, each against the FP64 oracle: tiny grids, footprints wider than the
domain (periodic multi-wrap), all-masked and single-active-cell masks, NaN on masked cells (land
stored as NaN), FP32 storage, and large batches."""
import math

import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import synthetic as S
import oracle as O
from helpers import max_rel, oracle_grid, oracle_plan, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-10


def cart(nx, ny, dx=1000.0, periodic=(False, False), mask=None):
    return cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0, dx, nx), cg.axis(0, dx, ny), mask, periodic)


@pytest.mark.parametrize("engine", ["banded", "separable", "prefixsum"])
@pytest.mark.parametrize("nx,ny", [(2, 2), (3, 5), (7, 2), (33, 9)])
def test_tiny_cartesian_grids(engine, nx, ny):
    kern = cg.TopHatKernel() if engine == "prefixsum" else cg.GaussianKernel(4.0)
    for periodic in ((False, False), (True, True)):
        g = cart(nx, ny, periodic=periodic)
        f = np.random.default_rng(nx * ny).standard_normal(g.shape)
        p = cg.plan_filter(g, kern, 3500.0, engine=engine)
        eng = {"banded": O.ENGINE_BANDED, "separable": O.ENGINE_SEPARABLE, "prefixsum": O.ENGINE_PREFIXSUM}[engine]
        ref = oracle_plan(g, kern, 3500.0, engine=eng).filter(f)
        assert max_rel(cg.filter_apply(None, f, p), ref) < TOL


@pytest.mark.parametrize("engine", ["banded", "separable"])
def test_footprint_wider_than_a_periodic_domain(engine):
    # radius 2.4 x 30 km = 72 km over a 10 x 12 km periodic box: offsets wrap several times, exactly as
    # the reference's mod1 wrap does (Filtering.jl:2567-2575, 1211-1255)
    g = cart(10, 12, periodic=(True, True))
    f = np.random.default_rng(3).standard_normal(g.shape)
    p = cg.plan_filter(g, cg.GaussianKernel(4.0), 30000.0, engine=engine)
    eng = O.ENGINE_BANDED if engine == "banded" else O.ENGINE_SEPARABLE
    assert max_rel(cg.filter_apply(None, f, p), oracle_plan(g, cg.GaussianKernel(4.0), 30000.0, engine=eng).filter(f)) < TOL


@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
def test_all_masked_and_single_active_cell(strat):
    g0 = S.sphere_grid(72, 36)
    f = np.random.default_rng(5).standard_normal(g0.shape)
    none = np.zeros(g0.shape, bool)
    one = none.copy()
    one[20, 30] = True
    for m in (none, one):
        g = g0.with_mask(m) if m.any() else cg.StructuredGrid(g0.geometry, g0.x, g0.y, m, g0.periodic)
        p = cg.plan_filter(g, cg.GaussianKernel(4.0), 8e5, mask_strategy=strat)
        got = cg.filter_apply(None, f, p)
        ref = oracle_plan(g, cg.GaussianKernel(4.0), 8e5, strat, mask=m).filter(f)
        assert np.all(np.isfinite(got))
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-300)
    # Pi on an all-masked slice is zero everywhere
    u, v = S.sphere_fields(g0, seed=1, lmax=30)
    Pi = cg.compute_Pi(None, np.stack([u, u]), np.stack([v, v]), None, g0, cg.GaussianKernel(4.0), 8e5,
                       mask_strategy=strat, slice_masks=np.stack([none, one]))
    assert np.all(Pi[0] == 0) and np.all(np.isfinite(Pi[1]))


def test_nan_on_masked_cells_is_ignored():
    g = S.sphere_grid(90, 45)
    m = S.land_mask(g, seed=2)
    g = g.with_mask(m)
    u, v = S.sphere_fields(g, seed=4, lmax=40)
    un, vn = u.copy(), v.copy()
    un[~m] = np.nan
    vn[~m] = np.nan
    a = cg.compute_Pi(None, un, vn, None, g, cg.GaussianKernel(4.0), 6e5)
    b = cg.compute_Pi(None, u, v, None, g, cg.GaussianKernel(4.0), 6e5)
    assert np.array_equal(a, b)
    f = np.where(m, u, np.nan)
    p = cg.plan_filter(g, cg.TopHatKernel(), 6e5)
    assert np.all(np.isfinite(cg.filter_apply(None, f, p)))


def test_float32_storage_filter_and_pi():
    g = S.sphere_grid(120, 60)
    g = g.with_mask(S.land_mask(g, seed=3))
    u, v = S.sphere_fields(g, seed=6, lmax=50)
    u32, v32 = u.astype(np.float32), v.astype(np.float32)
    p = cg.plan_filter(g, cg.GaussianKernel(4.0), 5e5)
    got = cg.filter_apply(None, u32, p)
    assert got.dtype == np.float32
    ref = oracle_plan(g, cg.GaussianKernel(4.0), 5e5).filter(u32.astype(np.float64))
    assert max_rel(got, ref) < 1e-6
    Pi = cg.compute_Pi(None, u32, v32, None, g, cg.GaussianKernel(4.0), 5e5)
    refPi = oracle_plan(g, cg.GaussianKernel(4.0), 5e5).compute_pi(u32.astype(np.float64), v32.astype(np.float64))["Pi"]
    assert Pi.dtype == np.float32 and rel_l2(Pi, refPi) < 1e-6


def test_large_batch_of_small_slices():
    g = cart(24, 20, periodic=(True, False))
    rng = np.random.default_rng(8)
    U = rng.standard_normal((64,) + g.shape)
    V = rng.standard_normal((64,) + g.shape)
    Pi = cg.compute_Pi(None, U, V, None, g, cg.GaussianKernel(4.0), 5000.0)
    op = oracle_plan(g, cg.GaussianKernel(4.0), 5000.0)
    for t in (0, 17, 63):
        assert rel_l2(Pi[t], op.compute_pi(U[t], V[t])["Pi"]) < 1e-9


def test_regional_sphere_bounded_x_denominator():
    # bounded longitude: the ZeroFill denominator varies along x near the edges (den per cell)
    d = math.radians(0.5)
    g = cg.StructuredGrid(cg.SphericalGeometry(), cg.axis(0.3, d, 50), cg.axis(-0.4, d, 40), periodic=(False, False))
    f = np.random.default_rng(9).standard_normal(g.shape)
    for strat in (cg.ZeroFill(), cg.Deformable()):
        p = cg.plan_filter(g, cg.GaussianKernel(4.0), 2e5, mask_strategy=strat)
        assert max_rel(cg.filter_apply(None, f, p), oracle_plan(g, cg.GaussianKernel(4.0), 2e5, strat).filter(f)) < TOL
