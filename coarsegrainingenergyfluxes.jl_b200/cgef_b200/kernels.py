"""Filter kernels (Kernels.jl).  The filter scale l is the FULL width (Kernels.jl:11-15)."""
from __future__ import annotations

import math
from dataclasses import dataclass

from . import _lib

# Kernels.jl:307
GAUSSIAN_TRUNCATION_TOL = 1e-10


class AbstractFilterKernel:
    code = -1


@dataclass(frozen=True)
class TopHatKernel(AbstractFilterKernel):
    """Unit weight for d <= l/2 (Kernels.jl:28, 318-320)."""

    code = _lib.TOPHAT
    alpha = 0.0


@dataclass(frozen=True)
class GaussianKernel(AbstractFilterKernel):
    """exp(-alpha (d/l)^2) (Kernels.jl:59-62, 322-324); alpha = 6 by default, 4 = FlowSieve's."""

    alpha: float = 6.0
    code = _lib.GAUSSIAN


def kernel_weight(kernel: AbstractFilterKernel, d: float, ell: float) -> float:
    if isinstance(kernel, TopHatKernel):
        return 1.0 if d <= ell / 2 else 0.0
    q = d / ell
    return math.exp(-kernel.alpha * (q * q))


def kernel_radius(kernel: AbstractFilterKernel, ell: float) -> float:
    """Truncation radius (Kernels.jl:354-359): l/2 for the top-hat, l sqrt(-ln(1e-10)/alpha)."""
    if isinstance(kernel, TopHatKernel):
        return ell / 2
    return ell * math.sqrt(-math.log(GAUSSIAN_TRUNCATION_TOL) / kernel.alpha)


def transfer_monotone(kernel: AbstractFilterKernel) -> bool:
    """d|G(k)|^2/dk <= 0 (Kernels.jl:509-518): true for the Gaussian, false for the top-hat."""
    if isinstance(kernel, GaussianKernel):
        return True
    if isinstance(kernel, TopHatKernel):
        return False
    raise TypeError(f"no monotonicity rule for {type(kernel).__name__}")


def check_spectrum_kernel(kernel: AbstractFilterKernel) -> None:
    """Kernels.jl:527-543: refuse a kernel whose |G|^2 is not monotone."""
    from .errors import ArgumentError
    if not transfer_monotone(kernel):
        raise ArgumentError(
            f"{type(kernel).__name__} cannot produce a guaranteed non-negative filtering spectral density: "
            "its |G(k)|^2 is not monotone decreasing.  Use spectrum=ForceSpectrum() to compute it anyway, "
            "NoSpectrum() to skip it, a GaussianKernel, or cumulative_energy.")
