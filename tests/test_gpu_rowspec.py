"""GPU parity of the row-spectral evaluation of the banded sums (ring FFTs along x) against the
FP64 oracle's direct sums, and against the library's own direct gather on the same plan.

The spectral evaluation is the same linear operator as the footprint sum (Filtering.jl:1569-1744,
2536-2598) evaluated through DFTs, so it differs from the direct sum only by FP64 rounding of the
transforms: filtered fields agree to ~1e-14 relative, and the asserted bounds are the direct
path's own (1e-10 on filtered fields, 1e-9 relative L2 on Pi).
"""
import math
import os

import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import synthetic as S
import oracle as O
from helpers import max_rel, oracle_plan, rel_l2

pytestmark = pytest.mark.gpu

PI_FP64 = 1e-9
FIELD_TOL = 1e-10
NTH = max(1, os.cpu_count() or 1)


def _sphere(nlon=180, nlat=90, seed=5, mask=True):
    g = S.sphere_grid(nlon, nlat)
    return g.with_mask(S.land_mask(g, seed=seed) if mask else None)


def _evaluate(plan, fn):
    """fn() with the plan's sums evaluated spectrally, then directly."""
    plan.set_row_spectral(True)
    a = fn()
    plan.set_row_spectral(False)
    b = fn()
    plan.set_row_spectral(True)
    return a, b


@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
@pytest.mark.parametrize("kernel,scale", [(cg.GaussianKernel(4.0), 5e5), (cg.GaussianKernel(6.0), 2.5e6),
                                          (cg.TopHatKernel(), 1.2e6)])
def test_sphere_filter_spectral_matches_oracle_and_direct(strat, kernel, scale):
    g = _sphere()
    f = np.random.default_rng(0).standard_normal(g.shape)
    p = cg.plan_filter(g, kernel, scale, mask_strategy=strat, engine="banded")
    avail, on, L = p.row_spectral
    assert avail and on and L == g.nx
    spec, direct = _evaluate(p, lambda: cg.filter_apply(None, f, p))
    ref = oracle_plan(g, kernel, scale, strat, O.ENGINE_BANDED).filter(f, NTH)
    assert max_rel(spec, ref) < FIELD_TOL
    assert max_rel(spec, direct) < FIELD_TOL


@pytest.mark.parametrize("nf", [1, 2, 3, 4])
def test_multi_field_filter_spectral(nf):
    g = _sphere(seed=7)
    rng = np.random.default_rng(nf)
    fields = [rng.standard_normal(g.shape) for _ in range(nf)]
    p = cg.plan_filter(g, cg.GaussianKernel(4.0), 8e5)
    spec, direct = _evaluate(p, lambda: cg.filter_apply_batch(None, fields, p))
    refs = oracle_plan(g, cg.GaussianKernel(4.0), 8e5).filter_batch(fields, NTH)
    for s, d, r in zip(spec, direct, refs):
        assert max_rel(s, r) < FIELD_TOL
        assert max_rel(s, d) < FIELD_TOL


@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
@pytest.mark.parametrize("scale", [3e5, 1.5e6])
def test_sphere_pi_spectral_matches_oracle(strat, scale):
    g = _sphere(seed=3)
    u, v = S.sphere_fields(g, seed=11, lmax=89)
    k = cg.GaussianKernel(4.0)
    p = cg.plan_filter(g, k, scale, mask_strategy=strat)
    spec, direct = _evaluate(p, lambda: cg.compute_Pi_fields(u, v, g, k, scale, mask_strategy=strat, filter_plan=p))
    ref = oracle_plan(g, k, scale, strat).compute_pi(u, v, NTH)
    for key in ("ubar", "vbar", "tau_xx", "tau_xy", "tau_yy"):
        assert rel_l2(spec[key], ref[key]) < FIELD_TOL * 10, key
    assert rel_l2(spec["Pi"], ref["Pi"]) < PI_FP64
    assert rel_l2(spec["Pi"], direct["Pi"]) < PI_FP64


def test_pole_closing_rings_spectral():
    # rings close near the poles (a = Nx/2, the reference visits [-a, a-1]): the extra column -a is
    # the column +a on the ring, so the row's kernel stays symmetric there
    nlat, nlon = 60, 120
    g = cg.StructuredGrid(cg.SphericalGeometry(), cg.axis(0.0, 2 * math.pi / nlon, nlon),
                          cg.axis(-math.pi / 2 + 1e-6, (math.pi - 2e-6) / (nlat - 1), nlat), periodic=(True, False))
    lon, lat = g.coords()
    LON, LAT = np.meshgrid(lon, lat)
    fld = np.cos(3 * LON) * np.exp(-(((np.abs(LAT) - 1.40) / 0.12) ** 2))
    p = cg.plan_filter(g, cg.GaussianKernel(6.0), 3.0e6)
    assert p.row_spectral[1]
    spec, direct = _evaluate(p, lambda: cg.filter_apply(None, fld, p))
    ref = oracle_plan(g, cg.GaussianKernel(6.0), 3.0e6).filter(fld, NTH)
    assert max_rel(spec, ref) < FIELD_TOL
    assert max_rel(spec, direct) < FIELD_TOL


@pytest.mark.parametrize("periodic", [(True, False), (True, True), (False, False)])
@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
def test_cartesian_banded_spectral(periodic, strat):
    # on a bounded x axis the rows are zero-padded to an FFT length >= Nx + the widest half-width
    n = 80
    m = np.ones((n, n), bool)
    m[10:20, 10:60] = False
    g = cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0, 1000.0, n), cg.axis(0, 1000.0, n), m, periodic)
    f = np.random.default_rng(2).standard_normal(g.shape)
    p = cg.plan_filter(g, cg.GaussianKernel(6.0), 7000.0, mask_strategy=strat, engine="banded")
    avail, on, L = p.row_spectral
    assert avail and on
    assert L == n if periodic[0] else L >= n
    spec, direct = _evaluate(p, lambda: cg.filter_apply(None, f, p))
    ref = oracle_plan(g, cg.GaussianKernel(6.0), 7000.0, strat, O.ENGINE_BANDED).filter(f, NTH)
    assert max_rel(spec, ref) < FIELD_TOL
    assert max_rel(spec, direct) < FIELD_TOL


def test_batched_slices_with_their_own_masks_spectral():
    # coarse_grain_slices! semantics: one mask per slice, inputs masked per slice before the FFT
    g = _sphere(mask=False)
    masks = np.stack([S.land_mask(g, seed=s) for s in (1, 2, 3)])
    u, v = S.sphere_fields(g, seed=4, lmax=89)
    ub = np.stack([u, 0.5 * u, -u])
    vb = np.stack([v, v, 0.25 * v])
    k = cg.GaussianKernel(4.0)
    p = cg.plan_filter(g, k, 6e5)
    spec, direct = _evaluate(p, lambda: cg.compute_Pi_fields(ub, vb, g, k, 6e5, filter_plan=p, slice_masks=masks))
    for s in range(3):
        ref = oracle_plan(g, k, 6e5, mask=masks[s]).compute_pi(ub[s], vb[s], NTH)
        assert rel_l2(spec["Pi"][s], ref["Pi"]) < PI_FP64
    assert rel_l2(spec["Pi"], direct["Pi"]) < PI_FP64


def test_unavailable_where_rows_are_asymmetric_on_a_bounded_axis():
    # a bounded x axis whose window is capped at Nx/2 closes with asymmetric rows: a correlation
    # with an asymmetric kernel, which the real kernel spectra cannot express, so the plan sums
    # directly and refuses the spectral evaluation
    nx, ny = 48, 40
    dx = 0.5 * math.pi / 180
    g = cg.StructuredGrid(cg.SphericalGeometry(), cg.axis(dx / 2, dx, nx),
                          cg.axis(-math.pi / 2 + math.pi / ny / 2, math.pi / ny, ny), periodic=(False, False))
    p = cg.plan_filter(g, cg.GaussianKernel(4.0), 8e5, engine="banded")
    di, dj, w, ptr = p.footprint()
    if np.max(di) == -np.min(di):
        pytest.skip("this grid's rows are all symmetric")
    assert p.row_spectral == (False, False, 0)
    with pytest.raises(cg.ArgumentError):
        p.set_row_spectral(True)
    f = np.random.default_rng(9).standard_normal(g.shape)
    ref = oracle_plan(g, cg.GaussianKernel(4.0), 8e5, engine=O.ENGINE_BANDED).filter(f)
    assert max_rel(cg.filter_apply(None, f, p), ref) < FIELD_TOL


def test_autotune_keeps_the_faster_evaluation_and_the_results():
    g = _sphere(seed=8)
    u, v = S.sphere_fields(g, seed=12, lmax=89)
    k = cg.GaussianKernel(4.0)
    p = cg.plan_filter(g, k, 1e6)
    p.autotune(1)
    avail, on, _ = p.row_spectral
    assert avail
    r = cg.compute_Pi_fields(u, v, g, k, 1e6, filter_plan=p)
    ref = oracle_plan(g, k, 1e6).compute_pi(u, v, NTH)
    assert rel_l2(r["Pi"], ref["Pi"]) < PI_FP64


@pytest.mark.parametrize("mixed", [False, True])
def test_sweep_sharing_source_spectra_equals_per_scale_flux(mixed):
    # a sweep transforms the source rows once and every row-spectral scale of that FFT length starts
    # from those spectra; each scale's flux must equal the same plan's own compute_Pi bit for bit,
    # also when a direct-gather scale sits between the spectral ones
    g = _sphere(seed=6)
    us, vs = zip(*[S.sphere_fields(g, seed=30 + t, lmax=89) for t in range(2)])
    U, V = np.stack(us), np.stack(vs)
    k = cg.GaussianKernel(4.0)
    scales = [3e5, 6e5, 1.2e6, 2.4e6]
    plans = [cg.plan_filter(g, k, s) for s in scales]
    for p in plans:
        assert p.row_spectral[1]
    if mixed:
        plans[1].set_row_spectral(False)
    res = cg.coarse_grain_batch(U, V, g, scales=scales, kernel=k, filter_plans=plans)
    for si, (s, p) in enumerate(zip(scales, plans)):
        one = cg.compute_Pi(None, U, V, None, g, k, s, filter_plan=p)
        assert np.array_equal(res.Pi[:, si], one), s
        ref = oracle_plan(g, k, s).compute_pi(us[0], vs[0], NTH)
        assert rel_l2(res.Pi[0, si], ref["Pi"]) < PI_FP64
