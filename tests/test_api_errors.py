"""The reference's error contract on the public API, restated (no GPU needed: every check runs before
any device work).  Shape disagreements are DimensionMismatch, unsupported or inadmissible requests
ArgumentError, a spectrum policy of the wrong type TypeError."""
import warnings

import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import diagnostics as D


def cart(n=16, ny=None, periodic=(True, True)):
    ny = n if ny is None else ny
    return cg.StructuredGrid(cg.CartesianGeometry(), cg.axis(0, 1000.0, n), cg.axis(0, 1000.0, ny), None, periodic)


SCALES = [4e3, 8e3]
NOSPEC = cg.NoSpectrum()


def test_coarse_grain_batch_shape_errors():
    # test/test_backends.jl:476-480: the grid fixes the spatial rank, everything before it is batch
    g = cart(12)
    N, Nt = 12, 3
    v = np.zeros((Nt, N, N))
    with pytest.raises(cg.DimensionMismatch):
        cg.coarse_grain_batch(np.zeros((Nt + 1, N, N)), v, g, scales=SCALES, spectrum=NOSPEC)
    with pytest.raises(cg.DimensionMismatch):
        cg.coarse_grain_batch(np.zeros((Nt, N, N + 1)), v, g, scales=SCALES, spectrum=NOSPEC)
    with pytest.raises(cg.DimensionMismatch):
        cg.coarse_grain_batch(np.zeros((N, N)), np.zeros((N, N)), g, scales=SCALES, spectrum=NOSPEC)
    with pytest.raises(cg.DimensionMismatch):
        cg.coarse_grain(np.zeros((N, N + 1)), np.zeros((N, N + 1)), g, scales=SCALES, spectrum=NOSPEC)
    with pytest.raises(cg.DimensionMismatch):
        cg.coarse_grain_slices([np.zeros((N, N))], [np.zeros((N, N))] * 2, [g], scales=SCALES, spectrum=NOSPEC)


def test_filter_apply_batched_shape_errors():
    # test/test_backends.jl:594-597 (grid 64 x 32 in Julia's (Nx, Ny) = numpy (32, 64))
    g = cart(64, 32)
    p = cg.plan_filter(g, cg.TopHatKernel(), 8e3)
    with pytest.raises(cg.DimensionMismatch):
        cg.filter_apply_batched(np.zeros((2, 8, 8)), np.zeros((2, 8, 8)), p)
    with pytest.raises(cg.DimensionMismatch):
        cg.filter_apply_batched(np.zeros((32, 64)), np.zeros((32, 64)), p)
    with pytest.raises(cg.DimensionMismatch):
        cg.filter_apply_batched(np.zeros((3, 32, 64)), np.zeros((2, 32, 64)), p)
    with pytest.raises(cg.DimensionMismatch):
        cg.filter_apply(np.zeros((32, 64)), np.zeros((64, 32)), p)
    with pytest.raises(cg.ArgumentError):
        cg.filter_apply_batched(np.zeros((2, 32, 64), np.float32), np.zeros((2, 32, 64)), p)
    with pytest.raises(cg.DimensionMismatch):
        cg.filter_apply_batch([np.zeros((32, 64))], [np.zeros((32, 64))] * 2, p)


def test_compute_pi_batch_errors():
    # test/test_backends.jl:754-766: every field must agree on the batch, and energy on its length
    g = cart(10)
    N, Nb = 10, 3
    k = cg.TopHatKernel()
    with pytest.raises(cg.DimensionMismatch):
        cg.compute_Pi(np.zeros((Nb, N, N)), np.zeros((Nb, N, N)), np.zeros((Nb + 2, N, N)), None, g, k, 4e3)
    with pytest.raises(cg.DimensionMismatch):
        cg.compute_Pi(np.zeros((Nb, N, N)), np.zeros((Nb, N + 1, N)), np.zeros((Nb, N + 1, N)), None, g, k, 4e3)
    with pytest.raises(cg.DimensionMismatch):
        cg.compute_Pi(np.zeros((Nb + 1, N, N)), np.zeros((Nb, N, N)), np.zeros((Nb, N, N)), None, g, k, 4e3)
    with pytest.raises(cg.DimensionMismatch):
        cg.compute_Pi(None, np.zeros((Nb, N, N)), np.zeros((Nb, N, N)), None, g, k, 4e3, energy=np.zeros(Nb + 1))
    with pytest.raises(cg.DimensionMismatch):
        cg.compute_Pi(None, np.zeros((Nb, N, N)), np.zeros((Nb, N, N)), None, g, k, 4e3,
                      slice_masks=np.ones((Nb + 1, N, N), bool))
    # the vertical velocity (2.5-D path) must match u's batch and dtype too
    with pytest.raises(cg.DimensionMismatch):
        cg.compute_Pi(None, np.zeros((Nb, N, N)), np.zeros((Nb, N, N)), np.zeros((Nb + 1, N, N)), g, k, 4e3)
    with pytest.raises(cg.ArgumentError):
        cg.compute_Pi(None, np.zeros((N, N)), np.zeros((N, N)), np.zeros((N, N), np.float32), g, k, 4e3)
    with pytest.raises(cg.ArgumentError):
        cg.compute_Pi(None, np.zeros((N, N)), np.zeros((N, N)), np.zeros((N, N)), g, k, 4e3,
                      outputs={"tau_ww": np.zeros((N, N))})
    with pytest.raises(cg.ArgumentError):
        cg.compute_Pi(None, np.zeros((N, N)), np.zeros((N, N), np.float32), None, g, k, 4e3)
    with pytest.raises(cg.ArgumentError):
        cg.compute_Pi(None, np.zeros((N, N)), np.zeros((N, N)), None, g, k, 4e3, outputs={"nope": np.zeros((N, N))})


def test_scale_and_kernel_validation():
    # src/Filtering.jl:2917-2922: a non-finite or non-positive scale is refused at the API edge
    g = cart(8)
    for s in (0.0, -1.0, float("nan"), float("inf")):
        with pytest.raises(cg.ArgumentError):
            cg.plan_filter(g, cg.GaussianKernel(4.0), s)
    with pytest.raises(cg.ArgumentError):
        cg.plan_filter(g, cg.GaussianKernel(4.0), 4e3, engine="spectral")


def test_spectrum_policy_gate():
    # test/test_diagnostics.jl:706-735
    th, ga = cg.TopHatKernel(), cg.GaussianKernel()
    assert D.gate_spectrum(ga, cg.StrictSpectrum())
    with pytest.raises(cg.ArgumentError):
        D.gate_spectrum(th, cg.StrictSpectrum())
    assert not D.gate_spectrum(th, NOSPEC)
    assert not D.gate_spectrum(ga, NOSPEC)
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        assert D.gate_spectrum(th, cg.ForceSpectrum())
    assert any("not monotone" in str(x.message) for x in w)
    with pytest.raises(cg.ArgumentError) as e:
        D.gate_spectrum(th, cg.StrictSpectrum())
    for recourse in ("ForceSpectrum", "NoSpectrum", "GaussianKernel", "cumulative_energy", "TopHatKernel",
                     "monotone"):
        assert recourse in str(e.value)


def test_pipeline_is_gated_before_any_work():
    # test/test_diagnostics.jl:671-680: the default kernel (top-hat) under the default StrictSpectrum
    g = cart(12)
    u = np.zeros((12, 12))
    with pytest.raises(cg.ArgumentError):
        cg.coarse_grain(u, u, g, scales=SCALES)
    with pytest.raises(cg.ArgumentError):
        cg.coarse_grain(u, u, g, scales=SCALES, kernel=cg.TopHatKernel())
    with pytest.raises(cg.ArgumentError):
        cg.coarse_grain_batch(np.zeros((2, 12, 12)), np.zeros((2, 12, 12)), g, scales=SCALES)
    with pytest.raises(cg.ArgumentError):
        cg.coarse_grain_slices([u], [u], [g], scales=SCALES)
    with pytest.raises(cg.ArgumentError):
        cg.filtering_spectrum(u, u, None, g, cg.TopHatKernel(), SCALES)
    for bad in (False, "force", None):
        with pytest.raises(TypeError):
            cg.coarse_grain(u, u, g, scales=SCALES, spectrum=bad)
