"""GPU parity against the committed golden fixtures (tests/golden/), through the public API and the
C ABI, with no oracle call at run time: every seeded case the FP64 oracle wrote (filters, compute_Pi
with its intermediates and E, cumulative energy; banded, separable and prefix-sum engines; ZeroFill
and Deformable; sphere and plane), and the reference's own coast known-answer values
(test/test_filtering.jl:918-961).

Tolerances are those of the oracle parity tests: 1e-10 (max, relative to the field's largest value)
on filtered fields, 1e-9 relative L2 on Pi and its intermediates, 1e-12 relative on energies.  The
banded cases run with both evaluations of the footprint sums, direct and row-spectral, where the
plan offers the latter.
"""
import numpy as np
import pytest

import cgef_b200 as cg
from golden_cases import arrays, coast_fields, coast_moments, manifest, reference_kats
from helpers import max_rel, rel_l2

pytestmark = pytest.mark.gpu

CASES = manifest()
FIELD_TOL = 1e-10
PI_TOL = 1e-9


def _grid(g, mask):
    geo = cg.SphericalGeometry(g["R"]) if g["geometry"] == "sphere" else cg.CartesianGeometry()
    return cg.StructuredGrid(geo, cg.axis(g["x0"], g["dx"], g["nx"]), cg.axis(g["y0"], g["dy"], g["ny"]), mask,
                             tuple(g["periodic"]))


def _kernel(case):
    return cg.GaussianKernel(case["alpha"]) if case["kernel"] == "gaussian" else cg.TopHatKernel()


def _strategy(case):
    return cg.Deformable() if case["strategy"] == "deformable" else cg.ZeroFill()


def _evaluations(plan):
    """The plan under each evaluation of its sums it offers (the direct gather always)."""
    if plan.engine != "banded":
        yield "direct"
        return
    plan.set_row_spectral(False)
    yield "direct"
    if plan.row_spectral[0]:
        plan.set_row_spectral(True)
        yield "row-spectral"


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_cuda_path_reproduces_golden_case(case):
    a = arrays(case)
    g = _grid(case["grid"], a["mask"])
    if case["op"] == "energy":
        got = cg.cumulative_energy(a["u"], a["v"], None, g, _kernel(case), case["scales"])
        np.testing.assert_allclose(got, a["cumulative_energy"], rtol=1e-12)
        return
    plan = cg.plan_filter(g, _kernel(case), case["scale"], mask_strategy=_strategy(case), engine=case["engine"])
    assert plan.engine == case["expect_engine"]
    for ev in _evaluations(plan):
        if case["op"] == "filter":
            outs = cg.filter_apply_batch(None, list(a["fields"]), plan)
            for got, ref in zip(outs, a["filtered"]):
                assert max_rel(got, ref) < FIELD_TOL, ev
        else:
            r = cg.compute_Pi_fields(a["u"], a["v"], g, _kernel(case), case["scale"], mask_strategy=_strategy(case),
                                     filter_plan=plan)
            for k in ("Pi", "ubar", "vbar", "tau_xy", "S_xy"):
                assert rel_l2(r[k], a[k]) < PI_TOL, (ev, k)
            assert float(r["energy"][0]) == pytest.approx(float(a["energy"][0]), rel=1e-12), ev


def test_cuda_path_meets_the_reference_coast_known_answers():
    kats = reference_kats()
    n, ic, mask, fields = coast_fields(kats)
    dx = kats["grid"]["dx"]
    g = cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0.0, dx, n), cg.axis(0.0, dx, n), mask)
    res = {}
    for name, st in (("zerofill", cg.ZeroFill()), ("deformable", cg.Deformable())):
        p = cg.plan_filter(g, cg.GaussianKernel(kats["kernel"]["alpha"]), kats["kernel"]["scale"], mask_strategy=st)
        res[name] = coast_moments(kats, *cg.filter_apply_batch(None, fields, p))
    (mz, cz, wz), (md, cd, wd) = res["zerofill"], res["deformable"]
    np.testing.assert_allclose(cz, kats["centroid_over_scale"]["values"], atol=kats["centroid_over_scale"]["atol"])
    np.testing.assert_allclose(wz, kats["width_ratio"]["values"], atol=kats["width_ratio"]["atol"])
    np.testing.assert_allclose(mz, kats["mass_zerofill"]["values"], atol=kats["mass_zerofill"]["atol"])
    np.testing.assert_allclose(md, kats["mass_deformable"]["value"], atol=kats["mass_deformable"]["atol"])
    np.testing.assert_allclose(cz, cd, rtol=kats["strategies_agree_rtol"], atol=1e-15)
    np.testing.assert_allclose(wz, wd, rtol=kats["strategies_agree_rtol"])
