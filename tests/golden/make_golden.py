"""Writes the golden fixtures of this directory.

    python tests/golden/make_golden.py

The reference is a Julia package that cannot run here, so these fixtures come from two sources:

* ``reference_kats.json`` holds the numeric known-answer values that the reference's own test
  suite asserts for this path, copied from its test file with file:line (the coast artifacts of
  test/test_filtering.jl:918-961, literals at :951, :952 and :955).
* ``oracle_cases.npz`` + ``oracle_cases.json`` hold small seeded cases: the inputs (fields and masks)
  and the FP64 CPU oracle's outputs. ``oracle/`` is itself pinned against the reference's tests
  (tests/test_oracle_pinning.py). The fixtures let the GPU parity tests run against committed
  numbers without the oracle. ``tests/test_golden.py`` checks on the CPU that the oracle still
  reproduces them.

Each case names its grid, kernel, scale, mask strategy, engine and operation. The inputs are smooth
seeded fields (a few Fourier modes) and seeded land masks, made here with numpy.
"""
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

R_EARTH = 6.371e6
PI_KEYS = ("Pi", "ubar", "vbar", "tau_xy", "S_xy")


def sphere_axes(nlon, nlat):
    d, dl = 2 * math.pi / nlon, math.pi / nlat
    return dict(geometry="sphere", nx=nlon, ny=nlat, x0=d / 2, dx=d, y0=-math.pi / 2 + dl / 2, dy=dl, R=R_EARTH,
                periodic=[True, False])


def cart_axes(nx, ny, dx, dy, periodic):
    return dict(geometry="cartesian", nx=nx, ny=ny, x0=0.0, dx=dx, y0=0.0, dy=dy, R=R_EARTH, periodic=list(periodic))


def smooth_field(g, rng, modes=6):
    """Sum of a few seeded Fourier modes in the two index directions (periodic in x)."""
    i = np.arange(g["nx"])[None, :] / g["nx"]
    j = (np.arange(g["ny"])[:, None] + 0.5) / g["ny"]
    f = np.zeros((g["ny"], g["nx"]))
    for m in range(1, modes + 1):
        for n in range(1, modes):
            a, p, q = rng.standard_normal(), rng.uniform(0, 2 * np.pi), rng.uniform(0, 2 * np.pi)
            f += a / (m * n) * np.cos(2 * np.pi * m * i + p) * np.cos(np.pi * n * j + q)
    return np.ascontiguousarray(f)


def land_mask(g, rng, land=0.3):
    """Active (True) where a smoothed seeded noise is above its `land` quantile."""
    noise = rng.standard_normal((g["ny"], g["nx"]))
    ky = np.fft.fftfreq(g["ny"])[:, None]
    kx = np.fft.fftfreq(g["nx"])[None, :]
    sm = np.real(np.fft.ifft2(np.fft.fft2(noise) * np.exp(-(kx ** 2 + ky ** 2) * 60.0)))
    return np.ascontiguousarray(sm > np.quantile(sm, land))


def oracle_grid(g, mask):
    geo = O.SPHERE if g["geometry"] == "sphere" else O.CART
    return O.Grid(geo, g["nx"], g["ny"], g["x0"], g["dx"], g["y0"], g["dy"], g["R"], g["periodic"][0],
                  g["periodic"][1], mask)


def oracle_plan(case, mask):
    k = O.GAUSSIAN if case["kernel"] == "gaussian" else O.TOPHAT
    st = O.DEFORMABLE if case["strategy"] == "deformable" else O.ZEROFILL
    eng = {"auto": O.ENGINE_AUTO, "banded": O.ENGINE_BANDED}[case["engine"]]
    return O.Plan(oracle_grid(case["grid"], mask), k, case["alpha"], case["scale"], st, eng)


ENGINE_NAMES = {O.ENGINE_BANDED: "banded", O.ENGINE_SEPARABLE: "separable", O.ENGINE_PREFIXSUM: "prefixsum"}


def cases():
    """The case specifications, each with the seed of its inputs."""
    s72 = sphere_axes(72, 36)
    return [
        dict(name="sphere_banded_zerofill_pi", grid=s72, kernel="gaussian", alpha=4.0, scale=1.5e6,
             strategy="zerofill", engine="auto", op="pi", masked=True, seed=11),
        dict(name="sphere_banded_deformable_pi", grid=s72, kernel="gaussian", alpha=4.0, scale=1.0e6,
             strategy="deformable", engine="auto", op="pi", masked=True, seed=12),
        dict(name="sphere_banded_deformable_filter3", grid=s72, kernel="gaussian", alpha=6.0, scale=2.0e6,
             strategy="deformable", engine="auto", op="filter", nfields=3, masked=True, seed=13),
        dict(name="sphere_tophat_prefixsum_filter2", grid=s72, kernel="tophat", alpha=0.0, scale=1.2e6,
             strategy="zerofill", engine="auto", op="filter", nfields=2, masked=True, seed=14),
        dict(name="sphere_cumulative_energy", grid=s72, kernel="gaussian", alpha=4.0, scale=0.0,
             scales=[8e5, 1.5e6, 3e6], strategy="zerofill", engine="auto", op="energy", masked=True, seed=15),
        dict(name="cart_separable_periodic_pi", grid=cart_axes(40, 32, 1000.0, 1250.0, (True, True)),
             kernel="gaussian", alpha=4.0, scale=6000.0, strategy="zerofill", engine="auto", op="pi", masked=False,
             seed=21),
        dict(name="cart_tophat_prefixsum_masked_pi", grid=cart_axes(40, 32, 1000.0, 1000.0, (True, False)),
             kernel="tophat", alpha=0.0, scale=7000.0, strategy="zerofill", engine="auto", op="pi", masked=True,
             seed=22),
        dict(name="cart_banded_bounded_deformable_filter2", grid=cart_axes(40, 32, 1000.0, 1000.0, (False, False)),
             kernel="gaussian", alpha=6.0, scale=5000.0, strategy="deformable", engine="banded", op="filter",
             nfields=2, masked=True, seed=23),
    ]


def run_case(case, arrays):
    """Fills `arrays` with the case's inputs and the oracle's outputs; returns the manifest entry."""
    g = case["grid"]
    rng = np.random.default_rng(case["seed"])
    mask = land_mask(g, rng) if case["masked"] else None
    entry = {k: v for k, v in case.items() if k != "seed"}
    pre = case["name"] + "/"
    if mask is not None:
        arrays[pre + "mask"] = mask.astype(np.uint8)
    if case["op"] == "filter":
        fields = np.stack([smooth_field(g, rng) for _ in range(case["nfields"])])
        plan = oracle_plan(case, mask)
        arrays[pre + "fields"] = fields
        arrays[pre + "filtered"] = np.stack(plan.filter_batch(list(fields)))
        entry["expect_engine"] = ENGINE_NAMES[plan.engine]
    elif case["op"] == "pi":
        u, v = smooth_field(g, rng), smooth_field(g, rng)
        plan = oracle_plan(case, mask)
        out = plan.compute_pi(u, v)
        arrays[pre + "u"], arrays[pre + "v"] = u, v
        for k in PI_KEYS:
            arrays[pre + k] = out[k]
        arrays[pre + "energy"] = np.array([plan.energy_from_filtered(out["ubar"], out["vbar"])])
        entry["expect_engine"] = ENGINE_NAMES[plan.engine]
    else:
        u, v = smooth_field(g, rng), smooth_field(g, rng)
        k = O.GAUSSIAN if case["kernel"] == "gaussian" else O.TOPHAT
        arrays[pre + "u"], arrays[pre + "v"] = u, v
        arrays[pre + "cumulative_energy"] = np.asarray(
            O.cumulative_energy(oracle_grid(g, mask), u, v, k, case["alpha"], case["scales"], O.ZEROFILL, 1))
    return entry


# test/test_filtering.jl:918-961: a 200 x 200 unit-cell Cartesian grid, coast at column 101 (1-based;
# active to its west), Gaussian kernel with the package default alpha = 6, l = 16 cells; at distances
# d = 1, 4, 8, 16 cells west of the coast, on row N/2, the footprint's centroid / l (:951), width
# relative to the interior width (:952) and the ZeroFill mass (:955), each asserted at atol 5e-3; the
# Deformable mass is 1 to 1e-12 (:956) and both strategies share centroid and width to rtol 1e-12 (:949-950).
REFERENCE_KATS = {
    "source": "test/test_filtering.jl:918-961",
    "grid": {"n": 200, "dx": 1.0, "coast_column_1based": 101, "row_1based": 100, "interior_column_1based": 50},
    "kernel": {"name": "gaussian", "alpha": 6.0, "scale": 16.0},
    "distances": [1, 4, 8, 16],
    "centroid_over_scale": {"values": [-0.211, -0.111, -0.032, 0.0], "atol": 5e-3, "line": 951},
    "width_ratio": {"values": [0.621, 0.747, 0.897, 0.998], "atol": 5e-3, "line": 952},
    "mass_zerofill": {"values": [0.543, 0.776, 0.948, 0.9996], "atol": 5e-3, "line": 955},
    "mass_deformable": {"value": 1.0, "atol": 1e-12, "line": 956},
    "strategies_agree_rtol": 1e-12,
}


def main():
    arrays, manifest = {}, []
    for case in cases():
        manifest.append(run_case(case, arrays))
    np.savez_compressed(os.path.join(HERE, "oracle_cases.npz"), **arrays)
    with open(os.path.join(HERE, "oracle_cases.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": manifest}, f, indent=1)
        f.write("\n")
    with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
        json.dump(REFERENCE_KATS, f, indent=1)
        f.write("\n")
    print(f"{len(manifest)} oracle cases, {sum(a.nbytes for a in arrays.values()) / 1e3:.0f} kB of arrays")


if __name__ == "__main__":
    main()
