"""compute_Π! with the vertical velocity w (the 2.5-D path, Diagnostics.jl:254-260, 483-681) against the
FP64 oracle's restatement (orc_compute_pi_w), through every filter engine.

Bounds as for the 2-D flux: the device computes in FP64 like the oracle, differing only in summation
order, so Pi agrees to 1e-9 relative L2 and the filtered/local fields to 1e-10; FP32 inputs are held to
the path's 1e-5 relative L2 on Pi.
"""
import os

import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import synthetic as S
import oracle as O
from helpers import oracle_plan, rel_l2

pytestmark = pytest.mark.gpu

NTH = max(1, os.cpu_count() or 1)
FIELDS = ["ubar", "vbar", "wbar", "tau_xx", "tau_xy", "tau_yy", "tau_xz", "tau_yz", "tau_zz",
          "S_xx", "S_xy", "S_yy", "S_xz", "S_yz"]


def _w_field(g, seed):
    rng = np.random.default_rng(seed)
    # a smooth vertical velocity two orders below the horizontal one, plus a little noise
    y, x = np.meshgrid(np.linspace(0, 2 * np.pi, g.ny), np.linspace(0, 2 * np.pi, g.nx), indexing="ij")
    return 1e-2 * (np.sin(3 * x) * np.cos(2 * y) + 0.1 * rng.standard_normal(g.shape))


_OENG = {"banded": O.ENGINE_BANDED, "separable": O.ENGINE_SEPARABLE, "prefixsum": O.ENGINE_PREFIXSUM}


def _check(g, kernel, scale, strat, u, v, w, plan=None, pi_tol=1e-9, field_tol=1e-10):
    r = cg.compute_Pi_fields(u, v, g, kernel, scale, mask_strategy=strat, filter_plan=plan, w=w)
    eng = _OENG.get(plan.engine, O.ENGINE_AUTO) if plan is not None else O.ENGINE_AUTO
    o = oracle_plan(g, kernel, scale, strat, eng)
    ref = o.compute_pi_w(u, v, w, NTH)
    sel = g.mask
    assert rel_l2(r["Pi"], ref["Pi"], sel) < pi_tol
    for k in FIELDS:
        assert rel_l2(r[k], ref[k], sel) < field_tol, k
    # E = 1/2 <|ubar|^2> over the active area, wbar^2 included when w is given (Diagnostics.jl:1125-1134)
    e = o.energy_from_filtered(ref["ubar"], ref["vbar"]) + o.energy_from_filtered(ref["wbar"], np.zeros_like(u))
    assert abs(float(r["energy"][0]) - e) <= 1e-12 * abs(e)
    if g.mask is not None:
        assert np.all(np.asarray(r["Pi"])[~g.mask] == 0)
    return r


@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
def test_sphere_banded_matches_oracle(strat):
    g = S.sphere_grid(180, 90)
    g = g.with_mask(S.land_mask(g, seed=3))
    u, v = S.sphere_fields(g, seed=11, lmax=60)
    w = _w_field(g, 1)
    p = cg.plan_filter(g, cg.GaussianKernel(4.0), 6e5, mask_strategy=strat)
    assert p.engine == "banded"
    for spectral in (False, True):
        p.set_row_spectral(spectral)
        _check(g, cg.GaussianKernel(4.0), 6e5, strat, u, v, w, plan=p)


def test_sphere_tophat_matches_oracle():
    g = S.sphere_grid(180, 90)
    g = g.with_mask(S.land_mask(g, seed=4))
    u, v = S.sphere_fields(g, seed=12, lmax=60)
    _check(g, cg.TopHatKernel(), 8e5, cg.ZeroFill(), u, v, _w_field(g, 2))


def _cart(n=96, periodic=(True, True), mask=True):
    m = None
    if mask:
        m = np.ones((n, n), bool)
        m[30:50, 40:70] = False
    return cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0, 1000.0, n), cg.axis(0, 1500.0, n), m, periodic)


@pytest.mark.parametrize("periodic", [(True, True), (False, False)])
@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
@pytest.mark.parametrize("kernel,engine", [(cg.GaussianKernel(4.0), "separable"), (cg.GaussianKernel(4.0), "banded"),
                                           (cg.TopHatKernel(), "prefixsum")],
                         ids=["separable", "banded", "prefixsum"])
def test_cartesian_engines_match_oracle(periodic, strat, kernel, engine):
    g = _cart(periodic=periodic)
    rng = np.random.default_rng(5)
    u, v = rng.standard_normal(g.shape), rng.standard_normal(g.shape)
    w = _w_field(g, 3)
    p = cg.plan_filter(g, kernel, 8000.0, mask_strategy=strat, engine=engine)
    assert p.engine == engine
    _check(g, kernel, 8000.0, strat, u, v, w, plan=p)


def test_cartesian_zero_w_is_the_2d_flux():
    """With w = 0 on the plane every extra term vanishes (wbar = 0, tau_iz = 0, S_iz = 0), so Pi and the
    2-D fields are the 2-D path's."""
    g = _cart()
    rng = np.random.default_rng(6)
    u, v = rng.standard_normal(g.shape), rng.standard_normal(g.shape)
    p = cg.plan_filter(g, cg.GaussianKernel(4.0), 6000.0)
    r3 = cg.compute_Pi_fields(u, v, g, cg.GaussianKernel(4.0), 6000.0, filter_plan=p, w=np.zeros(g.shape))
    r2 = cg.compute_Pi_fields(u, v, g, cg.GaussianKernel(4.0), 6000.0, filter_plan=p)
    assert rel_l2(r3["Pi"], r2["Pi"]) < 1e-13
    for k in ("ubar", "vbar", "tau_xx", "tau_xy", "tau_yy", "S_xx", "S_xy", "S_yy"):
        assert rel_l2(r3[k], r2[k]) < 1e-13, k
    for k in ("wbar", "tau_xz", "tau_yz", "tau_zz", "S_xz", "S_yz"):
        assert np.all(np.asarray(r3[k]) == 0), k
    assert abs(float(r3["energy"][0]) - float(r2["energy"][0])) <= 1e-14 * abs(float(r2["energy"][0]))


def test_batched_equals_per_slice_and_slice_masks():
    g = S.sphere_grid(120, 60)
    m = S.land_mask(g, seed=1)
    g = g.with_mask(m)
    nb = 3
    rng = np.random.default_rng(9)
    U = np.stack([S.sphere_fields(g, seed=20 + t, lmax=40)[0] for t in range(nb)])
    V = np.stack([S.sphere_fields(g, seed=40 + t, lmax=40)[1] for t in range(nb)])
    Wv = 1e-2 * rng.standard_normal((nb,) + g.shape)
    k = cg.GaussianKernel(4.0)
    p = cg.plan_filter(g, k, 7e5)
    rb = cg.compute_Pi_fields(U, V, g, k, 7e5, filter_plan=p, w=Wv)
    for t in range(nb):
        r1 = cg.compute_Pi_fields(U[t], V[t], g, k, 7e5, filter_plan=p, w=Wv[t])
        assert np.array_equal(rb["Pi"][t], r1["Pi"])
        assert rb["energy"][t] == r1["energy"][0]
    # one mask per slice: slice t under mask t equals a grid carrying mask t
    sm = np.stack([m, np.roll(m, 7, axis=1), np.roll(m, -5, axis=0)])
    base = g.with_mask(None)
    pb = cg.plan_filter(base, k, 7e5)
    rs = cg.compute_Pi_fields(U, V, base, k, 7e5, filter_plan=pb, w=Wv, slice_masks=sm)
    for t in range(nb):
        gt = base.with_mask(sm[t])
        ref = oracle_plan(gt, k, 7e5).compute_pi_w(U[t], V[t], Wv[t], NTH)
        assert rel_l2(rs["Pi"][t], ref["Pi"], sm[t]) < 1e-9


def test_fp32_inputs():
    g = S.sphere_grid(180, 90)
    g = g.with_mask(S.land_mask(g, seed=3))
    u, v = S.sphere_fields(g, seed=11, lmax=60)
    w = _w_field(g, 1)
    k = cg.GaussianKernel(4.0)
    r = cg.compute_Pi_fields(u.astype(np.float32), v.astype(np.float32), g, k, 6e5, w=w.astype(np.float32))
    assert r["Pi"].dtype == np.float32
    ref = oracle_plan(g, k, 6e5).compute_pi_w(u.astype(np.float32), v.astype(np.float32), w.astype(np.float32), NTH)
    assert rel_l2(r["Pi"], ref["Pi"], g.mask) < 1e-5
    assert rel_l2(r["wbar"], ref["wbar"], g.mask) < 1e-6


def test_device_tensors_equal_host_arrays():
    import torch

    g = S.sphere_grid(180, 90)
    g = g.with_mask(S.land_mask(g, seed=3))
    u, v = S.sphere_fields(g, seed=11, lmax=60)
    w = _w_field(g, 1)
    k = cg.GaussianKernel(4.0)
    p = cg.plan_filter(g, k, 6e5)
    rh = cg.compute_Pi_fields(u, v, g, k, 6e5, filter_plan=p, w=w)
    ud, vd, wd = (torch.from_numpy(x).cuda() for x in (u, v, w))
    rd = cg.compute_Pi_fields(ud, vd, g, k, 6e5, filter_plan=p, w=wd)
    torch.cuda.synchronize()
    assert np.array_equal(rd["Pi"].cpu().numpy(), rh["Pi"])
    for f in FIELDS:
        assert np.array_equal(rd[f].cpu().numpy(), rh[f]), f
