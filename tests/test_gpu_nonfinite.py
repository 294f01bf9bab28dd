"""Non-finite values in active cells keep the reference's local semantics on the default evaluation.

The reference adds an active source cell's value only into the targets whose footprint holds that cell
(Filtering.jl:2575-2585), so a NaN or Inf there reaches only those targets (and, through the strain
stencil, their neighbours in Pi).  The row-spectral evaluation would spread it along every bin of the
row's spectrum; instead its forward transform flags the slice and the direct gather sums that slice
again.  These tests check, on the full 0.25-degree sphere, that the flagged slice equals the direct
evaluation bit for bit, that the NaN set is exactly the cell's footprint, and that other slices of the
same launch keep their spectral results.
"""
import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import synthetic as S

pytestmark = pytest.mark.gpu

OUTS = ("Pi", "ubar", "vbar", "tau_xx", "tau_xy", "tau_yy")


@pytest.fixture(scope="module")
def c1():
    g = S.sphere_grid()
    g = g.with_mask(S.land_mask(g))
    u, v = S.sphere_fields(g, seed=0)
    return g, u, v


def _active_cell(mask, j0):
    i0 = int(np.flatnonzero(mask[j0])[len(np.flatnonzero(mask[j0])) // 2])
    return j0, i0


def _reach(plan, g, j0, i0):
    """Targets (j, i) whose footprint holds source cell (j0, i0): band j's entries with dj = j0 - j."""
    di, dj, w, ptr = plan.footprint()
    hit = np.zeros(g.shape, bool)
    for j in range(max(0, j0 - plan.info.dj_lim), min(g.ny, j0 + plan.info.dj_lim + 1)):
        sl = slice(ptr[j], ptr[j + 1])
        sel = dj[sl] == j0 - j
        hit[j, (i0 - di[sl][sel]) % g.nx] = True
    return hit


@pytest.mark.parametrize("value", [np.nan, np.inf])
def test_nonfinite_active_cell_stays_local_and_matches_direct(c1, value):
    g, u, v = c1
    j0, i0 = _active_cell(g.mask, 250)
    un = u.copy()
    un[j0, i0] = value
    k4 = cg.GaussianKernel(4.0)
    spec = cg.plan_filter(g, k4, 1e5)
    assert spec.row_spectral[1]
    direct = cg.plan_filter(g, k4, 1e5)
    direct.set_row_spectral(False)
    r_s = cg.compute_Pi_fields(un, v, g, k4, 1e5, filter_plan=spec)
    r_d = cg.compute_Pi_fields(un, v, g, k4, 1e5, filter_plan=direct)
    for k in OUTS:
        assert np.array_equal(r_s[k], r_d[k], equal_nan=True), k
    # the filtered velocity is non-finite exactly on the active targets whose footprint holds the cell
    reach = _reach(spec, g, j0, i0) & g.mask
    assert reach.sum() > 100
    assert np.array_equal(~np.isfinite(r_s["ubar"]), reach)
    # Pi also through the 3-node stencil: within two cells of that set, nowhere else
    bad = ~np.isfinite(r_s["Pi"])
    assert bad.any()
    grown = reach.copy()
    for d in (1, 2):
        grown |= np.roll(reach, d, 1) | np.roll(reach, -d, 1)
        grown[d:] |= reach[:-d]
        grown[:-d] |= reach[d:]
    assert not np.any(bad & ~grown)


def test_flagged_slice_falls_back_alone_in_a_batch_and_a_sweep(c1):
    g, u, v = c1
    j0, i0 = _active_cell(g.mask, 500)
    un = u.copy()
    un[j0, i0] = np.nan
    U, V = np.stack([u, un, u]), np.stack([v, v, v])
    k4 = cg.GaussianKernel(4.0)
    spec = cg.plan_filter(g, k4, 2e5)
    direct = cg.plan_filter(g, k4, 2e5)
    direct.set_row_spectral(False)
    Ps = cg.compute_Pi(None, U, V, None, g, k4, 2e5, filter_plan=spec)
    clean = cg.compute_Pi(None, u, v, None, g, k4, 2e5, filter_plan=spec)
    assert np.array_equal(Ps[0], clean) and np.array_equal(Ps[2], clean)
    assert np.array_equal(Ps[1], cg.compute_Pi(None, un, v, None, g, k4, 2e5, filter_plan=direct), equal_nan=True)
    # a sweep whose row-spectral scales share one forward transform carries the flag to all of them
    scales = [2e5, 5e5, 1e6]
    plans = [cg.plan_filter(g, k4, s) for s in scales]
    dplans = [cg.plan_filter(g, k4, s) for s in scales]
    for p in dplans:
        p.set_row_spectral(False)
    a = cg.coarse_grain_batch(U, V, g, scales=scales, kernel=k4, filter_plans=plans)
    b = cg.coarse_grain_batch(U[1:2], V[1:2], g, scales=scales, kernel=k4, filter_plans=dplans)
    assert np.array_equal(a.Pi[1], b.Pi[0], equal_nan=True)
    c = cg.coarse_grain_batch(U[:1], V[:1], g, scales=scales, kernel=k4, filter_plans=plans)
    assert np.array_equal(a.Pi[0], c.Pi[0])


def test_filter_with_an_infinite_active_value_matches_direct(c1):
    g, u, _ = c1
    j0, i0 = _active_cell(g.mask, 100)
    f = u.copy()
    f[j0, i0] = -np.inf
    spec = cg.plan_filter(g, cg.GaussianKernel(4.0), 3e5)
    direct = cg.plan_filter(g, cg.GaussianKernel(4.0), 3e5)
    direct.set_row_spectral(False)
    a = cg.filter_apply(None, f, spec)
    b = cg.filter_apply(None, f, direct)
    assert np.array_equal(a, b, equal_nan=True)
    assert np.array_equal(~np.isfinite(a), _reach(spec, g, j0, i0) & g.mask)


@pytest.mark.parametrize("periodic", [(True, True), (False, False)], ids=["periodic", "bounded"])
def test_nonfinite_next_to_the_row_ends_matches_direct(periodic):
    """The row-spectral planes are staged without a column halo, so the direct re-sum of a flagged slice
    wraps its columns (periodic x) or reads zeros past the row's ends (bounded x) itself: a NaN beside the
    seam or the edge must still give the direct evaluation's outputs bit for bit."""
    n = 120
    m = np.ones((n, n), bool)
    m[40:60, 50:80] = False
    g = cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0, 1000.0, n), cg.axis(0, 1000.0, n), m, periodic)
    rng = np.random.default_rng(2)
    u, v = rng.standard_normal(g.shape), rng.standard_normal(g.shape)
    u[30, 1] = np.nan
    v[90, n - 2] = np.inf
    k = cg.GaussianKernel(4.0)
    spec = cg.plan_filter(g, k, 9000.0, engine="banded")
    assert spec.row_spectral[0], "the banded Cartesian plan must offer the row-spectral evaluation"
    spec.set_row_spectral(True)
    direct = cg.plan_filter(g, k, 9000.0, engine="banded")
    direct.set_row_spectral(False)
    for name in ("ZeroFill", "Deformable"):
        strat = cg.ZeroFill() if name == "ZeroFill" else cg.Deformable()
        ps = cg.plan_filter(g, k, 9000.0, mask_strategy=strat, engine="banded")
        pd = cg.plan_filter(g, k, 9000.0, mask_strategy=strat, engine="banded")
        pd.set_row_spectral(False)
        a = cg.compute_Pi_fields(u, v, g, k, 9000.0, filter_plan=ps, mask_strategy=strat)
        b = cg.compute_Pi_fields(u, v, g, k, 9000.0, filter_plan=pd, mask_strategy=strat)
        for key in OUTS:
            assert np.array_equal(a[key], b[key], equal_nan=True), (name, key)
    # a sweep of both evaluations against the direct one
    res = cg.coarse_grain(u, v, g, scales=[9000.0], kernel=k, spectrum=cg.NoSpectrum(), filter_plans=[spec])
    ref = cg.coarse_grain(u, v, g, scales=[9000.0], kernel=k, spectrum=cg.NoSpectrum(), filter_plans=[direct])
    assert np.array_equal(res.Pi, ref.Pi, equal_nan=True)
