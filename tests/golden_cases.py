"""Loads the committed golden fixtures of tests/golden/ (made by tests/golden/make_golden.py)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def manifest():
    with open(os.path.join(GOLDEN, "oracle_cases.json")) as f:
        return json.load(f)["cases"]


def arrays(case):
    """The case's stored arrays, keyed without the case-name prefix; `mask` is bool or None."""
    pre = case["name"] + "/"
    with np.load(os.path.join(GOLDEN, "oracle_cases.npz")) as z:
        out = {k[len(pre):]: z[k] for k in z.files if k.startswith(pre)}
    out["mask"] = out["mask"].astype(bool) if "mask" in out else None
    return out


def reference_kats():
    with open(os.path.join(GOLDEN, "reference_kats.json")) as f:
        return json.load(f)


def coast_fields(kats):
    """The coast test's grid size, mask (ny, nx) and the filtered inputs 1, x and x^2, where x is the
    column offset from the coast (test/test_filtering.jl:918-932, 0-based here)."""
    n = kats["grid"]["n"]
    ic = kats["grid"]["coast_column_1based"] - 1
    mask = np.ones((n, n), bool)
    mask[:, ic:] = False
    xs = np.arange(n) * kats["grid"]["dx"]
    xc = np.ascontiguousarray(np.broadcast_to(xs - xs[ic], (n, n)))
    return n, ic, mask, [np.ones((n, n)), xc, np.ascontiguousarray(xc ** 2)]


def coast_moments(kats, f1, fx, fx2):
    """Mass, centroid / l and width ratio at the test's points from the filtered 1, x, x^2."""
    ic = kats["grid"]["coast_column_1based"] - 1
    jm = kats["grid"]["row_1based"] - 1
    i_in = kats["grid"]["interior_column_1based"] - 1
    ell = kats["kernel"]["scale"]
    x0 = (np.arange(f1.shape[1]) - ic) * kats["grid"]["dx"]
    sig = np.sqrt(fx2[jm, i_in] / f1[jm, i_in] - (fx[jm, i_in] / f1[jm, i_in]) ** 2)
    pts = [ic - d for d in kats["distances"]]
    mass = np.array([f1[jm, i] for i in pts])
    cent = np.array([fx[jm, i] / f1[jm, i] - x0[i] for i in pts]) / ell
    wid = np.array([np.sqrt(fx2[jm, i] / f1[jm, i] - (fx[jm, i] / f1[jm, i]) ** 2) for i in pts]) / sig
    return mass, cent, wid
