"""The spectral method's host side (no GPU needed): method resolution as the reference does it, the
refusals, and the plan's transfer function against the oracle's."""
import math

import numpy as np
import pytest

import cgef_b200 as cg
import oracle_spectral as SP


def cart(nx=32, ny=None, periodic=(True, True), dx=1.0, dy=None, mask=None):
    ny = nx if ny is None else ny
    dy = dx if dy is None else dy
    return cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0, dx, nx), cg.axis(0, dy, ny), mask, periodic)


def test_auto_method_resolves_as_the_reference():
    # test_spectral.jl:411-423 (Filtering._resolve_method)
    g = cg.GaussianKernel()
    assert isinstance(cg.resolve_method(cart(), g, cg.AutoMethod()), cg.Spectral)
    assert isinstance(cg.resolve_method(cart(periodic=(False, False)), g, cg.AutoMethod()), cg.RealSpace)
    assert isinstance(cg.resolve_method(cart(periodic=(True, False)), g, cg.AutoMethod()), cg.RealSpace)
    assert isinstance(cg.resolve_method(cart(periodic=(False, False)), g, cg.RealSpace()), cg.RealSpace)
    assert isinstance(cg.resolve_method(cart(), g, None), cg.RealSpace)
    assert isinstance(cg.resolve_method(cart(), g, "spectral"), cg.Spectral)
    sph = cg.StructuredGrid(cg.SphericalGeometry(), cg.axis(0.0, 2 * math.pi / 64, 64),
                            cg.axis(-1.0, 2.0 / 31, 32), periodic=(True, False))
    assert isinstance(cg.resolve_method(sph, g, cg.AutoMethod()), cg.RealSpace)
    # a length the transforms do not cover stays in real space under AutoMethod
    assert isinstance(cg.resolve_method(cart(31), g, cg.AutoMethod()), cg.RealSpace)
    with pytest.raises(cg.ArgumentError):
        cg.resolve_method(cart(), g, "fourier")


def test_spectral_plan_refusals():
    # test_spectral.jl:52-54: a non-periodic grid refuses the spectral method
    with pytest.raises(cg.ArgumentError):
        cg.plan_filter(cart(periodic=(False, False)), cg.GaussianKernel(), 4.0, method=cg.Spectral())
    with pytest.raises(cg.ArgumentError):
        cg.plan_filter(cart(periodic=(True, False)), cg.GaussianKernel(), 4.0, method=cg.Spectral())
    with pytest.raises(cg.ArgumentError):
        cg.plan_filter(cart(), cg.GaussianKernel(), 4.0, method=cg.Spectral(), engine="banded")
    with pytest.raises(cg.ArgumentError):
        cg.plan_filter(cart(), cg.GaussianKernel(), -4.0, method=cg.Spectral())
    # odd nx, or a prime factor above 5: outside the transforms' lengths
    for g in (cart(31), cart(32, 14)):
        with pytest.raises(cg.CgefError) as e:
            cg.plan_filter(g, cg.GaussianKernel(), 4.0, method=cg.Spectral())
        assert e.value.code == cg._lib.CGEF_EUNSUPPORTED


@pytest.mark.parametrize("kernel", [cg.GaussianKernel(4.0), cg.TopHatKernel()], ids=["gaussian", "tophat"])
def test_plan_transfer_matches_the_oracle(kernel):
    g = cart(48, 30, dx=2.0, dy=3.0)
    p = cg.plan_filter(g, kernel, 11.0, method=cg.Spectral())
    assert p.engine == "spectral" and isinstance(p, cg.SpectralFilterPlan)
    k = SP.GAUSSIAN if isinstance(kernel, cg.GaussianKernel) else SP.TOPHAT
    ref = SP.transfer(k, float(kernel.alpha), 11.0, 48, 30, 2.0, 3.0)
    got = p.transfer()
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) < 1e-15
    assert got[0, 0] == 1.0
