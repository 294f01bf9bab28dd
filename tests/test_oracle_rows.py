"""The oracle's row-subset form (CPU): a plan that evaluates only some target rows returns, on rows
whose strain-stencil neighbourhood it evaluated, exactly the full plan's Pi and intermediates.  The
full-size GPU parity tests rely on this to keep 1000-2000 km footprints on the 0.25-degree sphere
within seconds of CPU time."""
import math

import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import synthetic as S
import oracle as O
from helpers import oracle_grid


@pytest.mark.parametrize("strategy", [O.ZEROFILL, O.DEFORMABLE])
def test_row_subset_pi_equals_full_plan_on_the_rows(strategy):
    g = S.sphere_grid(180, 90)
    g = g.with_mask(S.land_mask(g, seed=5))
    u, v = S.sphere_fields(g, seed=3, lmax=60)
    og = oracle_grid(g)
    full = O.Plan(og, O.GAUSSIAN, 4.0, 8e5, strategy).compute_pi(u, v, 4)
    rows = [0, 1, 10, 44, 45, 88, 89]
    sub = O.Plan(og, O.GAUSSIAN, 4.0, 8e5, strategy, rows=O.rows_for_pi(rows, g.ny)).compute_pi(u, v, 4)
    for k in full:
        assert np.array_equal(full[k][rows], sub[k][rows]), k


def test_row_subset_builds_only_the_flagged_bands():
    g = S.sphere_grid(120, 60)
    og = oracle_grid(g)
    full = O.Plan(og, O.GAUSSIAN, 4.0, 1e6)
    sub = O.Plan(og, O.GAUSSIAN, 4.0, 1e6, rows=[3, 30])
    _, _, _, pf = full.footprint()
    di, dj, w, ps = sub.footprint()
    counts_f, counts_s = np.diff(pf), np.diff(ps)
    assert np.array_equal(counts_s[[3, 30]], counts_f[[3, 30]])
    assert counts_s.sum() == counts_f[3] + counts_f[30]
    # the flagged bands' entries are the full plan's
    dif, djf, wf, _ = full.footprint()
    for b in (3, 30):
        assert np.array_equal(w[ps[b]:ps[b + 1]], wf[pf[b]:pf[b + 1]])
        assert np.array_equal(di[ps[b]:ps[b + 1]], dif[pf[b]:pf[b + 1]])
    # unflagged rows of a filter read 0; an empty row set needs no footprint at all
    f = np.random.default_rng(0).standard_normal(g.shape)
    out = sub.filter(f)
    assert not np.any(out[[0, 1, 2, 4, 29, 31]])
    assert np.array_equal(out[[3, 30]], full.filter(f)[[3, 30]])
    assert O.Plan(og, O.GAUSSIAN, 4.0, 1e6, rows=[]).footprint()[0].size == 0


def test_rows_for_pi_widens_by_the_stencil_reach():
    assert list(O.rows_for_pi([0, 10], 20)) == [0, 1, 2, 8, 9, 10, 11, 12]
    assert list(O.rows_for_pi([0], 20, periodic_y=True)) == [0, 1, 2, 18, 19]
