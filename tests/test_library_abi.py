"""The C-ABI library: builds, loads, exports every declared symbol, builds host-side plans that
match the oracle, validates its arguments, and refuses to compute without a device (no CPU
fallback).  No GPU is needed."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import _lib
import oracle as O
from helpers import oracle_grid

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "cgef_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cgef_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), f"libcgef_b200.so does not export {n}"
    assert sorted(_lib.EXPORTED) == names
    assert L.cgef_version() == 1


def test_library_is_built_for_sm100a():
    # every .cu file refuses to compile device code for any target but sm_100a (cgef_internal.h)
    assert _lib.load().cgef_build_arch() == 1000


def test_failure_entry_points_refuse_null_objects():
    L = _lib.load()
    assert L.cgef_plan_reset_queue(None) == _lib.CGEF_EINVAL
    assert L.cgef_debug_inject(None, _lib.INJECT_STALE_QUEUE) == _lib.CGEF_EINVAL
    assert L.cgef_debug_inject(None, _lib.INJECT_CLOSURE_TIMEOUT) == _lib.CGEF_EINVAL


@pytest.mark.parametrize("scale,alpha", [(1e5, 4.0), (3e5, 6.0), (1.2e6, 4.0)])
def test_host_plan_footprint_equals_oracle_sphere(scale, alpha):
    d = math.radians(1.0)
    g = cg.StructuredGrid(cg.SphericalGeometry(), cg.axis(d / 2, d, 360), cg.axis(-math.pi / 2 + d / 2, d, 180))
    p = cg.plan_filter(g, cg.GaussianKernel(alpha), scale)
    assert p.engine == "banded"
    got = p.footprint()
    ref = O.Plan(oracle_grid(g), O.GAUSSIAN, alpha, scale).footprint()
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


SPHERE_GRIDS = [  # nx, ny, first latitude (deg, None = pole-to-pole centres), spacing (deg), longitude span (deg)
    (72, 36, None, None, 360), (73, 37, None, None, 360), (120, 60, None, None, 360), (45, 30, -40.0, 2.0, 90),
    (31, 15, -40.0, 5.0, 93), (90, 45, None, None, 360), (100, 40, 10.0, 2.0, 360), (64, 90, None, None, 360)]
KERNEL_SCALES = [(4.0, 3e5), (6.0, 8e5), (4.0, 2.5e6), (0.0, 1.2e6), (4.0, 6e6)]  # alpha 0: top-hat


@pytest.mark.parametrize("grid", SPHERE_GRIDS, ids=[f"{c[0]}x{c[1]}" for c in SPHERE_GRIDS])
def test_host_banded_footprints_equal_oracle_across_grids(grid):
    """Odd and even rings, rings that close at high latitude or at large scales, regional boxes that do
    not wrap, Gaussian and top-hat: the exported CSR equals the oracle's, which visits every offset of
    both signs as the reference does (Filtering.jl:675-731)."""
    nx, ny, lat0, dlat, span = grid
    d = math.radians(span / nx)
    if lat0 is None:
        dl = math.pi / ny
        y0 = -math.pi / 2 + dl / 2
    else:
        dl, y0 = math.radians(dlat), math.radians(lat0)
    g = cg.StructuredGrid(cg.SphericalGeometry(), cg.axis(d / 2, d, nx), cg.axis(y0, dl, ny), periodic=(span == 360, False))
    for alpha, scale in KERNEL_SCALES:
        k = cg.TopHatKernel() if alpha == 0.0 else cg.GaussianKernel(alpha)
        got = cg.plan_filter(g, k, scale, engine="banded").footprint()
        ref = O.Plan(oracle_grid(g), O.TOPHAT if alpha == 0.0 else O.GAUSSIAN, alpha, scale, O.ZEROFILL,
                     O.ENGINE_BANDED).footprint()
        for a, b in zip(got, ref):
            assert np.array_equal(a, b), (alpha, scale)


def test_host_plan_footprint_equals_oracle_cartesian_banded():
    g = cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0, 1000.0, 64), cg.axis(0, 1500.0, 48), periodic=(True, True))
    p = cg.plan_filter(g, cg.GaussianKernel(6.0), 8000.0, engine="banded")
    ref = O.Plan(oracle_grid(g), O.GAUSSIAN, 6.0, 8000.0, O.ZEROFILL, O.ENGINE_BANDED).footprint()
    for a, b in zip(p.footprint(), ref):
        assert np.array_equal(a, b)


def test_engine_dispatch_matches_reference():
    gc = cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0, 1.0, 32), cg.axis(0, 1.0, 32))
    gs = cg.StructuredGrid(cg.SphericalGeometry(), cg.axis(0, math.radians(2), 180), cg.axis(-1.5, math.radians(2), 60))
    assert cg.plan_filter(gc, cg.GaussianKernel(), 4.0).engine == "separable"
    assert cg.plan_filter(gc, cg.TopHatKernel(), 4.0).engine == "prefixsum"
    assert cg.plan_filter(gs, cg.GaussianKernel(), 4e5).engine == "banded"
    assert cg.plan_filter(gs, cg.TopHatKernel(), 4e5).engine == "prefixsum"


def test_argument_validation():
    g = cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0, 1.0, 16), cg.axis(0, 1.0, 16))
    for bad in (0.0, -1.0, float("inf"), float("nan")):
        with pytest.raises(cg.ArgumentError):
            cg.plan_filter(g, cg.GaussianKernel(), bad)
    with pytest.raises(cg.CgefError) as e:
        cg.plan_filter(g, cg.TopHatKernel(), 4.0, engine="separable")
    assert e.value.code == _lib.CGEF_EUNSUPPORTED
    gs = cg.StructuredGrid(cg.SphericalGeometry(), cg.axis(0, 0.1, 16), cg.axis(-0.5, 0.1, 8))
    with pytest.raises(cg.CgefError):
        cg.plan_filter(gs, cg.GaussianKernel(), 1e5, engine="separable")
    with pytest.raises(ValueError):
        cg.StructuredGrid(cg.CartesianGeometry(), [0.0, 1.0, 3.0], cg.axis(0, 1.0, 4))
    # the raw ABI rejects bad descriptors
    L = _lib.load()
    h = C.c_void_p()
    d = _lib.GridDesc()
    d.geometry, d.nx, d.ny, d.dx, d.dy = 0, 0, 4, 1.0, 1.0
    assert L.cgef_plan_create(C.byref(h), C.byref(d), 1, 6.0, 1.0, 0, 0) == _lib.CGEF_EINVAL
    assert b"grid size" in L.cgef_last_error()


@pytest.mark.skipif(_lib.device_count() > 0, reason="checks the no-device path")
def test_no_device_means_an_error_not_a_cpu_fallback():
    g = cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0, 1.0, 16), cg.axis(0, 1.0, 16))
    p = cg.plan_filter(g, cg.GaussianKernel(), 4.0)
    with pytest.raises(cg.CgefError) as e:
        cg.filter_apply(None, np.ones((16, 16)), p)
    assert e.value.code == _lib.CGEF_ENODEVICE


def test_plan_info_active_area():
    d = math.radians(2.0)
    m = np.ones((90, 180), bool)
    m[:, :30] = False
    g = cg.StructuredGrid(cg.SphericalGeometry(), cg.axis(d / 2, d, 180), cg.axis(-math.pi / 2 + d / 2, d, 90), m)
    p = cg.plan_filter(g, cg.GaussianKernel(4.0), 5e5)
    ref = O.Plan(oracle_grid(g), O.GAUSSIAN, 4.0, 5e5).active_area()
    assert p.info.active_area == pytest.approx(ref, rel=1e-14)
    assert cg.active_area(g) == pytest.approx(ref, rel=1e-12)


@pytest.mark.skipif(_lib.device_count() > 0, reason="checks the no-device path")
def test_row_spectral_needs_a_device_and_refuses_to_be_forced():
    # the kernel spectra are built on the device with the plan; a host-only plan keeps the direct
    # gather's tables and reports the spectral evaluation unavailable
    d = math.radians(2.0)
    g = cg.StructuredGrid(cg.SphericalGeometry(), cg.axis(d / 2, d, 180), cg.axis(-math.pi / 2 + d / 2, d, 90))
    p = cg.plan_filter(g, cg.GaussianKernel(4.0), 5e5)
    assert p.engine == "banded"
    assert p.row_spectral == (False, False, 0)
    with pytest.raises(cg.ArgumentError):
        p.set_row_spectral(True)
    # through the C ABI a plan without a device refuses either setting with its own status
    assert _lib.load().cgef_plan_set_row_spectral(p.handle, 1) == _lib.CGEF_ENODEVICE
    assert _lib.load().cgef_plan_set_row_spectral(p.handle, 0) == _lib.CGEF_ENODEVICE
