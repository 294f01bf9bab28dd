"""cgef_b200 -- the coarse-graining hot path of CoarseGrainingEnergyFluxes.jl on NVIDIA B200.

The host API mirrors the reference's Julia names (plan_filter, filter_apply!, compute_Π!,
cumulative_energy, filtering_spectrum, coarse_grain, ...); every compute call runs the CUDA
kernels of libcgef_b200.so through its C ABI (include/cgef_b200.h).  Fields are numpy arrays of
shape (ny, nx) -- the reference's column-major (Nx, Ny) -- or CUDA tensors of that shape.
"""
from ._lib import CgefError, device_count, library_path, load
from .diagnostics import (AbstractSpectrumPolicy, ForceSpectrum, NoSpectrum, StrictSpectrum, active_area,
                          compute_Pi, compute_Pi_fields, compute_Pi_strain_convergence, compute_Π,
                          compute_Π_strain_convergence, cumulative_energy, ddx, ddy, filtering_spectrum,
                          gate_spectrum, spectral_density, tau_decomposition)
from .errors import ArgumentError, DimensionMismatch
from .filtering import (AbstractFilterMethod, AbstractMaskStrategy, AutoMethod, Deformable, PhysicalFilterPlan,
                        RealSpace, Spectral, SpectralFilterPlan, ZeroFill, filter_apply, filter_apply_batch,
                        filter_apply_batched, filter_field, filter_fields, plan_filter, resolve_method,
                        set_footprint_build)
from .grids import Axis, CartesianGeometry, SphericalGeometry, StructuredGrid, axis
from .kernels import (GaussianKernel, TopHatKernel, check_spectrum_kernel, kernel_radius, kernel_weight,
                      transfer_monotone)
from .pipeline import (CoarseGrainBatchResult, CoarseGrainResult, coarse_grain, coarse_grain_batch,
                       coarse_grain_profile, coarse_grain_slices, SnapshotStream)

__all__ = [n for n in dir() if not n.startswith("_")]
