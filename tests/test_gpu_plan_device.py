"""The device build of large spherical footprints (cgef_set_footprint_build), against the host build,
an all-pairs brute force and the FP64 oracle.

The host decides every entry in both builds; the device computes the weights and the ZeroFill
denominators.  So the entry sets and the reference's CSR offsets must be identical, the weights equal
to a few ulps (CUDA's asin and exp against the host's libm: 1e-15 of the footprint's largest weight),
and the flux unchanged at the parity tests' tolerances.
"""
import math
import os
import time

import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import synthetic as S
import oracle as O
from helpers import oracle_grid, rel_l2

pytestmark = pytest.mark.gpu
NTH = max(1, os.cpu_count() or 1)


def _haversine(R, lon1, lat1, lon2, lat2):
    h = np.sin((lat2 - lat1) / 2) ** 2 + np.cos(lat1) * np.cos(lat2) * np.sin((lon2 - lon1) / 2) ** 2
    return 2 * R * np.arcsin(np.sqrt(np.minimum(h, 1.0)))


def _plans(g, kernel, scale, strat=cg.ZeroFill()):
    try:
        cg.set_footprint_build("host")
        ph = cg.plan_filter(g, kernel, scale, mask_strategy=strat, engine="banded")
        cg.set_footprint_build("device")
        pd = cg.plan_filter(g, kernel, scale, mask_strategy=strat, engine="banded")
    finally:
        cg.set_footprint_build("auto")
    assert ph.footprint_build == "host" and pd.footprint_build == "device"
    return ph, pd


def _grid_pole(nlat=60, nlon=120):
    # the reference's high-latitude configuration (test/test_filtering.jl:733-768): rings close
    return cg.StructuredGrid(cg.SphericalGeometry(), cg.axis(0.0, 2 * math.pi / nlon, nlon),
                             cg.axis(-math.pi / 2 + 1e-6, (math.pi - 2e-6) / (nlat - 1), nlat), periodic=(True, False))


CASES = [
    ("quarter-degree 300 km", lambda: S.sphere_grid(), cg.GaussianKernel(4.0), 3e5),
    ("quarter-degree 1000 km", lambda: S.sphere_grid(), cg.GaussianKernel(4.0), 1e6),
    ("one-degree 2000 km", lambda: S.sphere_grid(360, 180), cg.GaussianKernel(4.0), 2e6),
    ("one-degree 3000 km alpha 6", lambda: S.sphere_grid(360, 180), cg.GaussianKernel(6.0), 3e6),
    ("over the pole", _grid_pole, cg.GaussianKernel(6.0), 3e6),
    ("odd ring top-hat", lambda: S.sphere_grid(361, 181), cg.TopHatKernel(), 1.5e6),
]


@pytest.mark.parametrize("name,make,kernel,scale", CASES, ids=[c[0] for c in CASES])
def test_device_build_equals_host_build(name, make, kernel, scale):
    g = make()
    ph, pd = _plans(g, kernel, scale)
    dih, djh, wh, ptrh = ph.footprint()
    did, djd, wd, ptrd = pd.footprint()
    assert np.array_equal(ptrh, ptrd)
    assert np.array_equal(dih, did) and np.array_equal(djh, djd)
    assert np.max(np.abs(wd - wh)) <= 1e-15 * np.max(np.abs(wh))
    nz = wh != 0
    assert np.array_equal(wd != 0, nz)
    assert np.max(np.abs(wd[nz] - wh[nz]) / np.abs(wh[nz])) < 1e-13
    # the filter through either plan
    f = np.random.default_rng(1).standard_normal(g.shape)
    ph.set_row_spectral(False)
    pd.set_row_spectral(False)
    a, b = cg.filter_apply(None, f, ph), cg.filter_apply(None, f, pd)
    assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(a))


def test_device_build_entry_sets_match_an_all_pairs_brute_force():
    """The entry set of sampled bands straight against all pairs of cells: a cell is an entry of band j
    (as the offset from column 0 of row j) exactly when its haversine distance is within the radius.
    Pairs within 1e-12 of the radius are left out (numpy's transcendentals against the host's)."""
    g = S.sphere_grid(360, 180)
    alpha, scale = 4.0, 1.5e6
    _, pd = _plans(g, cg.GaussianKernel(alpha), scale)
    rad = cg.kernel_radius(cg.GaussianKernel(alpha), scale)
    di, dj, w, ptr = pd.footprint()
    lon, lat = g.coords()
    LON, LAT = np.meshgrid(lon, lat)
    R = g.geometry.R
    for j in (0, 1, 20, 89, 90, 150, 178, 179):
        d = _haversine(R, lon[0], lat[j], LON, LAT)
        sure_in = d <= rad * (1 - 1e-12)
        sure_out = d > rad * (1 + 1e-12)
        got = np.zeros(g.shape, bool)
        sl = slice(ptr[j], ptr[j + 1])
        got[j + dj[sl], di[sl] % g.nx] = True
        assert not np.any(sure_in & ~got), j
        assert not np.any(sure_out & got), j


@pytest.mark.parametrize("strat", [cg.ZeroFill(), cg.Deformable()])
def test_device_built_plan_flux_matches_oracle(strat):
    g = S.sphere_grid(360, 180)
    g = g.with_mask(S.land_mask(g, seed=2))
    u, v = S.sphere_fields(g, seed=7, lmax=150)
    _, pd = _plans(g, cg.GaussianKernel(4.0), 1.2e6, strat)
    r = cg.compute_Pi_fields(u, v, g, cg.GaussianKernel(4.0), 1.2e6, filter_plan=pd, mask_strategy=strat)
    st = O.DEFORMABLE if isinstance(strat, cg.Deformable) else O.ZEROFILL
    ref = O.Plan(oracle_grid(g), O.GAUSSIAN, 4.0, 1.2e6, st).compute_pi(u, v, NTH)
    assert rel_l2(r["Pi"], ref["Pi"], g.mask) < 1e-9
    for k in ("ubar", "vbar", "tau_xx", "tau_xy", "tau_yy"):
        assert rel_l2(r[k], ref[k], g.mask) < 1e-10, k


def test_c2_plans_build_fast_on_the_device():
    """C2's 24 scales on the 0.25-degree sphere: the automatic choice takes the device build for the
    large scales, and the 24 plans build in well under the host build's seconds."""
    g = S.sphere_grid()
    g = g.with_mask(S.land_mask(g))
    scales = 5e4 * 40.0 ** (np.arange(24) / 23.0)
    cg.plan_filter(g, cg.GaussianKernel(4.0), 1e5)  # device context and kernels loaded
    t0 = time.perf_counter()
    plans = [cg.plan_filter(g, cg.GaussianKernel(4.0), float(s)) for s in scales]
    dt = time.perf_counter() - t0
    where = [p.footprint_build for p in plans]
    assert where[-1] == "device" and where.count("device") >= 12
    print(f"24 C2 plans in {dt:.3f} s; device-built: {where.count('device')}")
    assert dt < 2.0
