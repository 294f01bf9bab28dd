"""The banded engine's schedule autotuner: it picks one of its candidate split granularities, and
the flux computed under any schedule stays the oracle's to FP64 rounding."""
import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import synthetic as S
from helpers import oracle_plan, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    g = S.sphere_grid(360, 180)
    g = g.with_mask(S.land_mask(g, seed=2))
    u, v = S.sphere_fields(g, seed=8, lmax=120)
    return g, u, v


def test_autotune_picks_a_candidate_and_keeps_parity(case):
    g, u, v = case
    plan = cg.plan_filter(g, cg.GaussianKernel(4.0), 7e5)
    w = plan.autotune(nbatch=1)
    assert w in (2.0, 4.0, 8.0, 16.0)
    Pi = cg.compute_Pi(None, u, v, None, g, plan.kernel, plan.scale, filter_plan=plan)
    ref = oracle_plan(g, cg.GaussianKernel(4.0), 7e5).compute_pi(u, v)["Pi"]
    assert rel_l2(Pi, ref) < 1e-9
    again = cg.compute_Pi(None, u, v, None, g, plan.kernel, plan.scale, filter_plan=plan)
    assert np.array_equal(Pi, again)


def test_every_schedule_gives_the_same_flux(case):
    g, u, v = case
    plan = cg.plan_filter(g, cg.GaussianKernel(4.0), 1.2e6)
    out = []
    for w in (1.0, 2.0, 16.0, 64.0):
        plan.set_split_waves(w)
        out.append(cg.compute_Pi(None, u, v, None, g, plan.kernel, plan.scale, filter_plan=plan))
    for o in out[1:]:
        assert rel_l2(o, out[0]) < 1e-13


def test_autotune_is_a_no_op_off_the_banded_engine():
    g = S.cartesian_grid(n=64)
    plan = cg.plan_filter(g, cg.GaussianKernel(4.0), 8e3)
    assert plan.engine == "separable"
    assert plan.autotune() == 0.0


def test_captured_sweep_graph_replays_the_eager_sweep_exactly(case):
    import ctypes as C

    import torch

    from cgef_b200 import _lib
    g, u, v = case
    L = _lib.load()
    plans = [cg.plan_filter(g, cg.GaussianKernel(4.0), s) for s in (2e5, 6e5)]
    du = torch.from_numpy(np.stack([u, -u])).cuda()
    dv = torch.from_numpy(np.stack([v, 0.5 * v])).cuda()
    parr = (C.c_void_p * 2)(*[p.handle.value for p in plans])
    st = torch.cuda.Stream()
    Pi = torch.empty((2, 2) + g.shape, dtype=torch.float64, device="cuda")
    E = torch.empty((2, 2), dtype=torch.float64, device="cuda")
    _lib.check(L.cgef_sweep_device(parr, 2, _lib.F64, du.data_ptr(), dv.data_ptr(), 2, None, Pi.data_ptr(),
                                   E.data_ptr(), st.cuda_stream))
    torch.cuda.synchronize()
    eager_pi, eager_e = Pi.clone(), E.clone()
    Pi.zero_()
    E.zero_()
    gh = C.c_void_p()
    _lib.check(L.cgef_sweep_graph_create(C.byref(gh), parr, 2, _lib.F64, du.data_ptr(), dv.data_ptr(), 2, None,
                                         Pi.data_ptr(), E.data_ptr(), st.cuda_stream))
    Pi.zero_()
    E.zero_()
    torch.cuda.synchronize()
    L.cgef_reset_launch_count()
    _lib.check(L.cgef_graph_launch(gh, st.cuda_stream))
    torch.cuda.synchronize()
    assert L.cgef_launch_count() > 0
    _lib.check(L.cgef_graph_destroy(gh))
    assert torch.equal(Pi, eager_pi) and torch.equal(E, eager_e)
    # the null (legacy) stream cannot be captured: refused, not attempted
    with pytest.raises(cg.CgefError):
        _lib.check(L.cgef_sweep_graph_create(C.byref(gh), parr, 2, _lib.F64, du.data_ptr(), dv.data_ptr(), 2, None,
                                             Pi.data_ptr(), E.data_ptr(), None))


@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
def test_tall_filter_tiles_match_the_oracle(case, strat):
    g, u, v = case
    plan = cg.plan_filter(g, cg.GaussianKernel(4.0), 9e5, mask_strategy=strat)
    op = oracle_plan(g, cg.GaussianKernel(4.0), 9e5, strat)
    rng = np.random.default_rng(3)
    fields = [rng.standard_normal(g.shape) for _ in range(4)]
    ref = [op.filter(f) for f in fields]
    for rows in (8, 4):
        plan.set_filter_rows(rows)
        assert plan.schedule()[1] == rows
        # 1, 2, 3 and 4 fields per pass (3 with the mask and 4 fall back to 4-row tiles)
        for k in (1, 2, 3, 4):
            outs = cg.filter_apply_batch(None, fields[:k], plan)
            for o, r in zip(outs, ref):
                assert rel_l2(o, r) < 1e-10, (rows, k)
        got = cg.filter_apply_batched(None, np.stack(fields[:3]), plan)
        for t in range(3):
            assert rel_l2(got[t], ref[t]) < 1e-10


def test_autotune_reports_a_filter_tile_height(case):
    g, _, _ = case
    plan = cg.plan_filter(g, cg.GaussianKernel(4.0), 1.5e6)
    plan.autotune()
    w, rows = plan.schedule()
    assert w in (2.0, 4.0, 8.0, 16.0) and rows in (4, 8)
