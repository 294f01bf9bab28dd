"""The benchmark's roofline arithmetic on the CPU: the row-spectral evaluation's compulsory bytes per
launch at the 0.25 degree, 100 km workload, and where the committed ncu traffic applies.  No GPU."""
import importlib.util
import math
import os
import types

import pytest

import cgef_b200 as cg
from cgef_b200 import synthetic as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_row_spectral_compulsory_bytes_at_quarter_degree_100_km(bench):
    g = S.sphere_grid()
    p = cg.plan_filter(g, cg.GaussianKernel(4.0), 1e5)
    D = p.info.dj_lim
    # 100 km, alpha 4: radius 239.9 km over 27.8 km rows
    assert D == math.ceil(1e5 * math.sqrt(-math.log(1e-10) / 4.0) / (6.371e6 * math.pi / 720))
    assert D == 9
    # the plan as the device builds it: a 1440-point ring, so 721 bins per row
    stub = types.SimpleNamespace(row_spectral=(True, True, 1440), info=p.info)
    N, nk, na = 1440 * 720, 721, 9
    kspec = 720 * (2 * D + 1) * nk * 8      # kernel spectra
    # the flux: the strain pass finishes the unnormalised sums, so the launch writes them once
    want = (3 * N * 8                       # staged planes (3 planetary velocities)
            + 4 * 720 * na * nk * 16        # source and summed spectra, each written and read
            + kspec
            + na * N * 8)                   # unnormalised sums, written
    assert want == 477_452_160
    assert bench.rowspec_bytes(stub, g.with_mask(S.land_mask(g)), 1, na, 3, 0, True, raw=True) == want
    # eight snapshots per launch move eight times the per-snapshot bytes; the kernel spectra are read
    # once per launch whatever the snapshot count
    assert bench.rowspec_bytes(stub, g, 8, na, 3, 0, False, raw=True) == 8 * (want - kspec) + kspec
    # a filter of three fields: the sums written and read, the outputs written, the mask read
    f3 = bench.rowspec_bytes(stub, g.with_mask(S.land_mask(g)), 1, 3, 3, 3, True)
    assert f3 == 3 * N * 8 + 4 * 720 * 3 * nk * 16 + kspec + 2 * 3 * N * 8 + 3 * N * 8 + N


def test_committed_traffic_only_where_a_capture_exists(bench):
    t1, basis1, one = bench.committed_traffic("sphere1:rowspec", 1)
    assert t1 is not None and 3e8 < t1 < 6e8 and "one launch" in basis1 and one == t1
    # several snapshots per launch: no capture of that launch, the one-snapshot figure beside it
    t8, basis8, one8 = bench.committed_traffic("sphere1:rowspec", 8)
    assert t8 is None and "8 snapshots" in basis8 and one8 == t1
    assert bench.committed_traffic("sphere1:rowspec", 1, 500.0) == (None, None, None)
    assert bench.committed_traffic("no-such-workload:rowspec", 1) == (None, None, None)
