"""The committed golden fixtures (tests/golden/) on the CPU: the FP64 oracle still reproduces every
seeded case it wrote, and it meets the reference's own known-answer values as they are copied into
reference_kats.json (test/test_filtering.jl:918-961).  No GPU is needed."""
import numpy as np
import pytest

import oracle as O
from golden_cases import arrays, coast_fields, coast_moments, manifest, reference_kats

CASES = manifest()
PI_KEYS = ("Pi", "ubar", "vbar", "tau_xy", "S_xy")


def _grid(g, mask):
    geo = O.SPHERE if g["geometry"] == "sphere" else O.CART
    return O.Grid(geo, g["nx"], g["ny"], g["x0"], g["dx"], g["y0"], g["dy"], g["R"], g["periodic"][0],
                  g["periodic"][1], mask)


def _plan(case, mask):
    k = O.GAUSSIAN if case["kernel"] == "gaussian" else O.TOPHAT
    st = O.DEFORMABLE if case["strategy"] == "deformable" else O.ZEROFILL
    eng = O.ENGINE_BANDED if case["engine"] == "banded" else O.ENGINE_AUTO
    return O.Plan(_grid(case["grid"], mask), k, case["alpha"], case["scale"], st, eng)


def _close(got, ref, rtol=1e-13):
    scale = max(float(np.max(np.abs(ref))), 1e-300)
    assert float(np.max(np.abs(np.asarray(got) - ref))) <= rtol * scale


def test_fixture_set_covers_every_engine_operation_and_strategy():
    names = {c["name"] for c in CASES}
    assert len(names) == len(CASES) == 8
    assert {c.get("expect_engine") for c in CASES} >= {"banded", "separable", "prefixsum"}
    assert {c["op"] for c in CASES} == {"filter", "pi", "energy"}
    assert {c["strategy"] for c in CASES} == {"zerofill", "deformable"}
    assert {c["grid"]["geometry"] for c in CASES} == {"sphere", "cartesian"}


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_reproduces_golden_case(case):
    a = arrays(case)
    if case["op"] == "energy":
        k = O.GAUSSIAN if case["kernel"] == "gaussian" else O.TOPHAT
        got = O.cumulative_energy(_grid(case["grid"], a["mask"]), a["u"], a["v"], k, case["alpha"], case["scales"],
                                  O.ZEROFILL, 2)
        _close(got, a["cumulative_energy"])
        return
    plan = _plan(case, a["mask"])
    assert {O.ENGINE_BANDED: "banded", O.ENGINE_SEPARABLE: "separable",
            O.ENGINE_PREFIXSUM: "prefixsum"}[plan.engine] == case["expect_engine"]
    if case["op"] == "filter":
        for got, ref in zip(plan.filter_batch(list(a["fields"]), 2), a["filtered"]):
            _close(got, ref)
    else:
        out = plan.compute_pi(a["u"], a["v"], 2)
        for k in PI_KEYS:
            _close(out[k], a[k])
        assert plan.energy_from_filtered(out["ubar"], out["vbar"]) == pytest.approx(a["energy"][0], rel=1e-13)


def test_oracle_meets_the_reference_coast_known_answers():
    kats = reference_kats()
    assert kats["source"] == "test/test_filtering.jl:918-961"
    n, ic, mask, fields = coast_fields(kats)
    g = O.Grid(O.CART, n, n, 0.0, kats["grid"]["dx"], 0.0, kats["grid"]["dx"], mask=mask)
    res = {}
    for st in (O.ZEROFILL, O.DEFORMABLE):
        p = O.Plan(g, O.GAUSSIAN, kats["kernel"]["alpha"], kats["kernel"]["scale"], st)
        res[st] = coast_moments(kats, *p.filter_batch(fields, 2))
    (mz, cz, wz), (md, cd, wd) = res[O.ZEROFILL], res[O.DEFORMABLE]
    np.testing.assert_allclose(cz, kats["centroid_over_scale"]["values"], atol=kats["centroid_over_scale"]["atol"])
    np.testing.assert_allclose(wz, kats["width_ratio"]["values"], atol=kats["width_ratio"]["atol"])
    np.testing.assert_allclose(mz, kats["mass_zerofill"]["values"], atol=kats["mass_zerofill"]["atol"])
    np.testing.assert_allclose(md, kats["mass_deformable"]["value"], atol=kats["mass_deformable"]["atol"])
    np.testing.assert_allclose(cz, cd, rtol=kats["strategies_agree_rtol"], atol=1e-15)
    np.testing.assert_allclose(wz, wd, rtol=kats["strategies_agree_rtol"])
