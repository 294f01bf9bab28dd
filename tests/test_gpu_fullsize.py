"""GPU parity at the benchmark's full sizes, against the FP64 oracle.

The oracle's direct sums at 1000-2000 km on the full 0.25-degree sphere cost minutes per scale, so
these tests use its row-subset form (`oracle.Plan(..., rows=...)`): it evaluates only the target
rows a test compares, widened by the strain stencil's reach (`oracle.rows_for_pi`), and its Pi on
those rows is the full plan's bit for bit (`tests/test_oracle_rows.py`).  The rows sampled are both
polar caps (where the footprint closes the ring), the jet latitude (40 S), the equator and a few
mid-latitudes.  The device runs its default evaluation, which on these plans is the row-spectral one.

Tolerances are the ones of the other parity tests: 1e-10 relative L2 on the filtered fields and
tau, 1e-9 on Pi (FP64 storage), 1e-6 on Pi with FP32 storage.
"""
import math
import os

import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import synthetic as S
import oracle as O
from helpers import oracle_grid, rel_l2

pytestmark = pytest.mark.gpu

PI_FP64 = 1e-9
FIELD_TOL = 1e-10
PI_FP32 = 1e-6
NTH = max(1, os.cpu_count() or 1)
# 0-based latitude rows of the 1440 x 720 grid: both polar caps, the jet (40 S is between rows 199
# and 200), the equator, mid-latitudes of either hemisphere
C1_ROWS = [0, 2, 60, 199, 200, 290, 359, 360, 470, 600, 717, 719]
C2_SCALES = 5e4 * 40.0 ** (np.arange(24) / 23.0)  # 50 ... 2000 km, log-spaced


@pytest.fixture(scope="module")
def c1():
    g = S.sphere_grid()
    g = g.with_mask(S.land_mask(g))
    u, v = S.sphere_fields(g, seed=0)
    return g, u, v


def _rows_parity(r, ref, mask, rows, pi_tol, field_tol):
    sel = np.zeros(mask.shape, bool)
    sel[rows] = mask[rows]
    errs = {k: rel_l2(r[k], ref[k], sel) for k in ("Pi", "ubar", "vbar", "tau_xx", "tau_xy", "tau_yy")}
    assert errs["Pi"] < pi_tol, errs
    for k in ("ubar", "vbar", "tau_xx", "tau_xy", "tau_yy"):
        assert errs[k] < field_tol, errs
    # inactive targets are exactly zero on both sides
    off = np.zeros(mask.shape, bool)
    off[rows] = ~mask[rows]
    assert not np.any(np.asarray(r["Pi"])[off])
    return errs


@pytest.mark.parametrize("scale", [1.0e6, 2.0e6])
def test_c2_large_scales_full_sphere_rows_match_oracle(c1, scale):
    """C2's largest scales on the full 1440 x 720 sphere with the C1 mask: the row-spectral
    evaluation (347 row offsets and a 1.5 GB kernel-spectrum table at 2000 km) against the oracle's
    direct sums on the sampled rows."""
    g, u, v = c1
    plan = cg.plan_filter(g, cg.GaussianKernel(4.0), scale)
    avail, enabled, L = plan.row_spectral
    assert avail and enabled and L == 1440
    r = cg.compute_Pi_fields(u, v, g, cg.GaussianKernel(4.0), scale, filter_plan=plan)
    rows = O.rows_for_pi(C1_ROWS, g.ny)
    ref = O.Plan(oracle_grid(g), O.GAUSSIAN, 4.0, scale, rows=rows).compute_pi(u, v, NTH)
    _rows_parity(r, ref, g.mask, C1_ROWS, PI_FP64, FIELD_TOL)


def test_c2_sweep_24_scales_energy_and_spectrum_full_size(c1):
    """The 24-scale sweep (50-2000 km) on one full-size snapshot: E(l) of the sweep equals the FP64
    area-weighted energy of the filtered velocities (the oracle's energy_from_filtered over every
    active cell), those velocities equal the oracle's on the sampled rows at the smallest (direct
    gather) and a middle scale, every scale's Pi equals the per-scale compute_Pi! bit for bit, and
    the spectrum is the oracle's spectral density of E(l)."""
    g, u, v = c1
    k4 = cg.GaussianKernel(4.0)
    plans = [cg.plan_filter(g, k4, float(s)) for s in C2_SCALES]
    res = cg.coarse_grain(u, v, g, scales=C2_SCALES, kernel=k4, filter_plans=plans)
    og = oracle_grid(g)
    area_plan = O.Plan(og, O.GAUSSIAN, 4.0, 1e5, rows=[])  # mask and cell areas only; no footprint
    E_host = np.empty(len(C2_SCALES))
    spectral = []
    for s, (scale, p) in enumerate(zip(C2_SCALES, plans)):
        spectral.append(p.row_spectral[1])
        r = cg.compute_Pi_fields(u, v, g, k4, float(scale), filter_plan=p)
        assert np.array_equal(res.Pi[s], r["Pi"]), f"sweep Pi differs from compute_Pi! at {scale:.0f} m"
        E_host[s] = area_plan.energy_from_filtered(r["ubar"], r["vbar"])
        assert r["energy"][0] == pytest.approx(E_host[s], rel=1e-12)
        if s in (0, 12):
            rows = O.rows_for_pi(C1_ROWS, g.ny)
            ref = O.Plan(og, O.GAUSSIAN, 4.0, float(scale), rows=rows).compute_pi(u, v, NTH)
            _rows_parity(r, ref, g.mask, C1_ROWS, PI_FP64, FIELD_TOL)
    assert sum(spectral) >= 12, "most C2 scales run the row-spectral evaluation"
    np.testing.assert_allclose(res.cumulative_energy, E_host, rtol=1e-12)
    k = 1.0 / C2_SCALES
    np.testing.assert_allclose(res.wavenumber, k, rtol=0)
    np.testing.assert_allclose(res.filtering_spectrum, O.spectral_density(E_host, k), rtol=1e-9)


def test_c3_regional_levels_full_shape_fp32(c1):
    """C3 at its real shape: the 400 x 600 regional box, FP32 storage, per-level masks; three levels
    (the surface, a middle one and the deepest, about 20% active) at the row-spectral scales
    132-400 km, against the oracle on sampled rows of each level."""
    grid, U, V, M, _ = S.regional_levels()
    levels = [0, 20, 39]
    assert M[39].mean() < 0.3
    scales = list(2.5e4 * 16.0 ** (np.arange(6) / 5.0))[3:]  # 132, 230, 400 km of the 6-scale set
    grids = [grid.with_mask(M[k]) for k in levels]
    res = cg.coarse_grain_slices([U[k] for k in levels], [V[k] for k in levels], grids, scales=scales,
                                 kernel=cg.GaussianKernel(4.0))
    base = grid.with_mask(None)
    for s in scales:
        assert cg.plan_filter(base, cg.GaussianKernel(4.0), s).row_spectral[1]
    rows_cmp = [0, 1, 100, 199, 200, 330, 398, 399]
    for q, k in enumerate(levels):
        rows = O.rows_for_pi(rows_cmp, grid.ny)
        og = oracle_grid(grid, M[k])
        assert res[q].Pi.dtype == np.float32
        for si, s in enumerate(scales):
            ref = O.Plan(og, O.GAUSSIAN, 4.0, float(s), rows=rows).compute_pi(
                U[k].astype(np.float64), V[k].astype(np.float64), NTH)
            sel = np.zeros(grid.shape, bool)
            sel[rows_cmp] = M[k][rows_cmp]
            err = rel_l2(res[q].Pi[si], ref["Pi"], sel)
            assert err < PI_FP32, (k, s, err)


@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
def test_c1_tophat_full_size_matches_oracle(c1, strat):
    """The package's default kernel on the C1 sphere: the exact top-hat (l = 100 km) by per-row prefix
    sums, the scan taken by warps in 32-column chunks, against the oracle's sequential running sums
    (Filtering.jl:894-1078) over every cell.

    The method itself is ill-conditioned in FP64, whoever sums: an interval's sum is the difference of
    two running sums over the tripled 4320-cell row (the row's magnitude over the window's, ~1e3), and
    tau = (uu)bar - ubar ubar cancels another ~1e3 on this field.  Two summation orders of the same
    terms therefore differ by ~1e-13 in ubar but ~1e-10 in tau and ~1e-9 in Pi (Deformable adds the
    mask's running sum to the denominator).  The bounds are those, with a margin: four orders inside
    the path's 1e-5 contract for Pi."""
    g, u, v = c1
    k = cg.TopHatKernel()
    plan = cg.plan_filter(g, k, 1e5, mask_strategy=strat)
    assert plan.engine == "prefixsum"
    r = cg.compute_Pi_fields(u, v, g, k, 1e5, filter_plan=plan, mask_strategy=strat)
    st = O.DEFORMABLE if isinstance(strat, cg.Deformable) else O.ZEROFILL
    ref = O.Plan(oracle_grid(g), O.TOPHAT, 0.0, 1e5, st).compute_pi(u, v, NTH)
    errs = {key: rel_l2(r[key], ref[key], g.mask) for key in ("Pi", "ubar", "vbar", "tau_xx", "tau_xy", "tau_yy")}
    assert errs["Pi"] < 1e-8, errs
    for key in ("ubar", "vbar"):
        assert errs[key] < 1e-12, errs
    for key in ("tau_xx", "tau_xy", "tau_yy"):
        assert errs[key] < 2e-9, errs
