"""Failure paths, driven by host-side injection (no kernel is made to fault, trap or wait).

- The closure's tensor-core steps wait on mbarriers with an iteration limit; when one runs out the
  kernel sets the closure's device error word, releases its tensor memory and returns.  Here the
  host writes that word before an ordinary call (cgef_debug_inject), and the call must report
  CGEF_ETIMEOUT, clear the word, and leave the closure usable.
- The direct gather hands out work items from a per-plan queue that its last warp zeroes.  Here the
  host leaves the queue as a launch that stopped part-way would, and the next call must still sum
  every item (each launch zeroes the queue first); cgef_plan_reset_queue zeroes it on demand.
"""
import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import _lib
from cgef_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def test_closure_wait_timeout_maps_to_etimeout_and_clears():
    torch = pytest.importorskip("torch")
    from cgef_b200 import closure as CL
    L = _lib.load()
    c = CL.Closure(seed=2)
    x = torch.from_numpy(np.random.default_rng(0).standard_normal((512, 5)).astype(np.float32)).cuda()
    y0 = c.forward(x).cpu().numpy()
    _lib.check(L.cgef_debug_inject(c.handle, _lib.INJECT_CLOSURE_TIMEOUT))
    y = torch.empty((512, 3), dtype=torch.float32, device="cuda")
    rc = L.cgef_closure_forward_device(c.handle, x.data_ptr(), 512, y.data_ptr(),
                                       torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.CGEF_ETIMEOUT
    assert b"wait limit" in L.cgef_last_error()
    # the word was cleared: the next call succeeds and computes the same outputs
    assert np.array_equal(c.forward(x).cpu().numpy(), y0)


@pytest.mark.parametrize("row_spectral", [False, True])
def test_stale_work_queue_does_not_reach_the_next_launch(row_spectral):
    g = S.sphere_grid(360, 180)
    g = g.with_mask(S.land_mask(g, seed=3))
    u, v = S.sphere_fields(g, seed=5, lmax=120)
    k4 = cg.GaussianKernel(4.0)
    plan = cg.plan_filter(g, k4, 4e5)
    plan.set_row_spectral(row_spectral)
    clean = cg.compute_Pi(None, u, v, None, g, k4, 4e5, filter_plan=plan)
    f = cg.filter_apply(None, u, plan)
    L = _lib.load()
    _lib.check(L.cgef_debug_inject(plan.handle, _lib.INJECT_STALE_QUEUE))
    assert np.array_equal(cg.compute_Pi(None, u, v, None, g, k4, 4e5, filter_plan=plan), clean)
    _lib.check(L.cgef_debug_inject(plan.handle, _lib.INJECT_STALE_QUEUE))
    _lib.check(L.cgef_plan_reset_queue(plan.handle))
    assert np.array_equal(cg.filter_apply(None, u, plan), f)
    # a NaN slice takes the zero-weight-skipping gather, which uses the same queue
    un = u.copy()
    un[90, np.flatnonzero(g.mask[90])[0]] = np.nan
    _lib.check(L.cgef_debug_inject(plan.handle, _lib.INJECT_STALE_QUEUE))
    a = cg.compute_Pi(None, un, v, None, g, k4, 4e5, filter_plan=plan)
    assert np.isnan(a).any() and np.isfinite(a).sum() > 0.5 * a.size * g.mask.mean()
    assert np.array_equal(np.isfinite(a), np.isfinite(cg.compute_Pi(None, un, v, None, g, k4, 4e5, filter_plan=plan)))


def test_plan_of_another_engine_has_no_queue_to_inject():
    L = _lib.load()
    plan = cg.plan_filter(S.cartesian_grid(64, 1000.0), cg.GaussianKernel(4.0), 8000.0)
    assert plan.engine == "separable"
    assert L.cgef_debug_inject(plan.handle, _lib.INJECT_STALE_QUEUE) == _lib.CGEF_EINVAL
    _lib.check(L.cgef_plan_reset_queue(plan.handle))
