"""ctypes binding of libcgef_b200.so (the C ABI of include/cgef_b200.h).

The library is the product: every compute call below runs CUDA kernels.  There is no CPU
fallback -- a missing library or device raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

from . import build as _build

CGEF_OK = 0
CGEF_EINVAL = -1
CGEF_ENOMEM = -2
CGEF_ECUDA = -3
CGEF_ESTRATEGY = -4
CGEF_EUNSUPPORTED = -5
CGEF_ENODEVICE = -6
CGEF_ETIMEOUT = -7
INJECT_CLOSURE_TIMEOUT, INJECT_STALE_QUEUE = 1, 2
BUILD_AUTO, BUILD_HOST, BUILD_DEVICE = 0, 1, 2

CARTESIAN, SPHERICAL = 0, 1
TOPHAT, GAUSSIAN = 0, 1
ZEROFILL, DEFORMABLE = 0, 1
ENGINE_AUTO, ENGINE_BANDED, ENGINE_SEPARABLE, ENGINE_PREFIXSUM, ENGINE_SPECTRAL = 0, 1, 2, 3, 4
F64, F32 = 0, 1

# Every symbol include/cgef_b200.h declares.
EXPORTED = [
    "cgef_version", "cgef_last_error", "cgef_device_count", "cgef_plan_create", "cgef_plan_destroy",
    "cgef_plan_get_info", "cgef_plan_get_footprint", "cgef_filter", "cgef_filter_batch", "cgef_compute_pi",
    "cgef_cumulative_energy", "cgef_sweep", "cgef_ddx", "cgef_ddy", "cgef_filter_device",
    "cgef_compute_pi_device", "cgef_sweep_device", "cgef_launch_count", "cgef_reset_launch_count",
    "cgef_profile_enable", "cgef_profile_read", "cgef_profile_reset", "cgef_filter_device_noalloc",
    "cgef_closure_create", "cgef_closure_destroy", "cgef_closure_get_params", "cgef_closure_set_params",
    "cgef_closure_pairs_device", "cgef_closure_train_device", "cgef_closure_forward_device",
    "cgef_closure_grad_device", "cgef_closure_pi_device", "cgef_plan_autotune", "cgef_plan_set_split_waves",
    "cgef_sweep_graph_create", "cgef_graph_launch", "cgef_graph_destroy", "cgef_tau_decomposition",
    "cgef_tau_decomposition_device", "cgef_pi_strain_convergence", "cgef_pi_strain_convergence_device",
    "cgef_pipeline_create", "cgef_pipeline_submit", "cgef_pipeline_drain", "cgef_pipeline_destroy",
    "cgef_plan_set_filter_rows", "cgef_plan_get_schedule", "cgef_plan_set_row_spectral",
    "cgef_plan_get_row_spectral", "cgef_build_arch", "cgef_plan_reset_queue", "cgef_debug_inject",
    "cgef_set_footprint_build", "cgef_plan_get_build", "cgef_compute_pi_w", "cgef_compute_pi_w_device",
    "cgef_plan_get_transfer",
]
KERNEL_STAGE, KERNEL_BANDED, KERNEL_SEPARABLE, KERNEL_PREFIX, KERNEL_STRAIN, KERNEL_CLOSURE, KERNEL_ROWSPEC = (
    0, 1, 2, 3, 4, 5, 6)
CLOSURE_NPARAM = 8899


class GridDesc(C.Structure):
    _fields_ = [
        ("geometry", C.c_int32), ("periodic_x", C.c_int32), ("periodic_y", C.c_int32), ("reserved", C.c_int32),
        ("nx", C.c_int64), ("ny", C.c_int64),
        ("x0", C.c_double), ("dx", C.c_double), ("y0", C.c_double), ("dy", C.c_double),
        ("radius", C.c_double), ("mask", C.c_void_p),
    ]


class PlanInfo(C.Structure):
    _fields_ = [
        ("engine", C.c_int32), ("nbands", C.c_int32), ("nentries", C.c_int64), ("dj_lim", C.c_int32),
        ("di_max", C.c_int32), ("kernel_radius", C.c_double), ("active_area", C.c_double),
    ]


class PiWOutputs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in
                ("pi", "ubar", "vbar", "wbar", "tau_xx", "tau_xy", "tau_yy", "tau_xz", "tau_yz", "tau_zz",
                 "s_xx", "s_xy", "s_yy", "s_xz", "s_yz", "energy")]


class PiOutputs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in
                ("pi", "ubar", "vbar", "tau_xx", "tau_xy", "tau_yy", "s_xx", "s_xy", "s_yy", "energy")]


class AdamW(C.Structure):
    _fields_ = [("lr", C.c_double), ("beta1", C.c_double), ("beta2", C.c_double), ("eps", C.c_double),
                ("weight_decay", C.c_double)]


class ClosureReport(C.Structure):
    _fields_ = [("judged_tiles", C.c_int64), ("failed_tiles", C.c_int64), ("est_rel_l2", C.c_double),
                ("fallbacks", C.c_int32), ("reserved", C.c_int32)]


class TauParts(C.Structure):
    _fields_ = [("leonard", C.c_void_p * 3), ("cross", C.c_void_p * 3), ("reynolds", C.c_void_p * 3)]


class StrainConvOutputs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("total", "strain", "convergence", "divergence", "strain_magnitude")]


class CgefError(RuntimeError):
    """A failed library call; `code` is the negative CGEF status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"cgef status {code}: {msg}")
        self.code = code


_lib: Optional[C.CDLL] = None


def library_path() -> str:
    return _build.LIB_PATH


def load(build_if_missing: bool = True) -> C.CDLL:
    """Loads (building first, if needed and possible) libcgef_b200.so."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB_PATH
    if not os.path.exists(path):
        if not build_if_missing:
            raise RuntimeError(f"libcgef_b200.so is not built ({path}); run `python -m cgef_b200.build`")
        _build.build()
    L = C.CDLL(path)
    vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    L.cgef_version.restype = i32
    L.cgef_last_error.restype = C.c_char_p
    L.cgef_device_count.restype = i32
    L.cgef_build_arch.restype = i32
    L.cgef_plan_reset_queue.argtypes = [vp]
    L.cgef_plan_reset_queue.restype = i32
    L.cgef_debug_inject.argtypes = [vp, i32]
    L.cgef_debug_inject.restype = i32
    L.cgef_compute_pi_w.argtypes = [vp, i32, vp, vp, vp, i64, vp, C.POINTER(PiWOutputs)]
    L.cgef_compute_pi_w.restype = i32
    L.cgef_compute_pi_w_device.argtypes = [vp, i32, vp, vp, vp, i64, vp, C.POINTER(PiWOutputs), vp]
    L.cgef_compute_pi_w_device.restype = i32
    L.cgef_set_footprint_build.argtypes = [i32]
    L.cgef_set_footprint_build.restype = i32
    L.cgef_plan_get_build.argtypes = [vp, C.POINTER(i32)]
    L.cgef_plan_get_build.restype = i32
    L.cgef_plan_create.argtypes = [C.POINTER(vp), C.POINTER(GridDesc), i32, dbl, dbl, i32, i32]
    L.cgef_plan_create.restype = i32
    L.cgef_plan_destroy.argtypes = [vp]
    L.cgef_plan_destroy.restype = i32
    L.cgef_plan_get_info.argtypes = [vp, C.POINTER(PlanInfo)]
    L.cgef_plan_get_info.restype = i32
    L.cgef_plan_get_footprint.argtypes = [vp, vp, vp, vp, vp]
    L.cgef_plan_get_footprint.restype = i32
    L.cgef_filter.argtypes = [vp, i32, vp, vp, i64]
    L.cgef_filter.restype = i32
    L.cgef_filter_batch.argtypes = [vp, i32, vp, vp, i32]
    L.cgef_filter_batch.restype = i32
    L.cgef_compute_pi.argtypes = [vp, i32, vp, vp, i64, vp, C.POINTER(PiOutputs)]
    L.cgef_compute_pi.restype = i32
    L.cgef_cumulative_energy.argtypes = [vp, i32, i32, vp, vp, vp]
    L.cgef_cumulative_energy.restype = i32
    L.cgef_sweep.argtypes = [vp, i32, i32, vp, vp, i64, vp, vp, vp]
    L.cgef_sweep.restype = i32
    L.cgef_ddx.argtypes = [vp, i32, vp, vp]
    L.cgef_ddx.restype = i32
    L.cgef_ddy.argtypes = [vp, i32, vp, vp]
    L.cgef_ddy.restype = i32
    L.cgef_filter_device.argtypes = [vp, i32, vp, vp, i64, vp]
    L.cgef_filter_device.restype = i32
    L.cgef_filter_device_noalloc.argtypes = [vp, i32, vp, vp, i64, vp]
    L.cgef_filter_device_noalloc.restype = i32
    L.cgef_compute_pi_device.argtypes = [vp, i32, vp, vp, i64, vp, C.POINTER(PiOutputs), vp]
    L.cgef_compute_pi_device.restype = i32
    L.cgef_sweep_device.argtypes = [vp, i32, i32, vp, vp, i64, vp, vp, vp, vp]
    L.cgef_sweep_device.restype = i32
    L.cgef_launch_count.restype = i64
    L.cgef_reset_launch_count.restype = None
    L.cgef_profile_enable.argtypes = [i32]
    L.cgef_profile_enable.restype = None
    L.cgef_profile_read.argtypes = [i32, C.POINTER(dbl), C.POINTER(i64)]
    L.cgef_profile_read.restype = i32
    L.cgef_profile_reset.restype = None
    L.cgef_pipeline_create.argtypes = [C.POINTER(vp), vp, i32, i32, i64, vp, i32]
    L.cgef_pipeline_submit.argtypes = [vp, vp, vp, vp, vp]
    L.cgef_pipeline_drain.argtypes = [vp]
    L.cgef_pipeline_destroy.argtypes = [vp]
    for n in ("create", "submit", "drain", "destroy"):
        getattr(L, "cgef_pipeline_" + n).restype = i32
    L.cgef_tau_decomposition.argtypes = [vp, i32, vp, vp, C.POINTER(TauParts)]
    L.cgef_tau_decomposition.restype = i32
    L.cgef_tau_decomposition_device.argtypes = [vp, i32, vp, vp, C.POINTER(TauParts), vp]
    L.cgef_tau_decomposition_device.restype = i32
    L.cgef_pi_strain_convergence.argtypes = [vp, i32, vp, vp, i64, C.POINTER(StrainConvOutputs)]
    L.cgef_pi_strain_convergence.restype = i32
    L.cgef_pi_strain_convergence_device.argtypes = [vp, i32, vp, vp, i64, vp, C.POINTER(StrainConvOutputs), vp]
    L.cgef_pi_strain_convergence_device.restype = i32
    L.cgef_sweep_graph_create.argtypes = [C.POINTER(vp), vp, i32, i32, vp, vp, i64, vp, vp, vp, vp]
    L.cgef_sweep_graph_create.restype = i32
    L.cgef_graph_launch.argtypes = [vp, vp]
    L.cgef_graph_launch.restype = i32
    L.cgef_graph_destroy.argtypes = [vp]
    L.cgef_graph_destroy.restype = i32
    L.cgef_plan_autotune.argtypes = [vp, i32, C.POINTER(dbl)]
    L.cgef_plan_autotune.restype = i32
    L.cgef_plan_set_split_waves.argtypes = [vp, dbl]
    L.cgef_plan_set_split_waves.restype = i32
    L.cgef_plan_set_filter_rows.argtypes = [vp, i32]
    L.cgef_plan_set_filter_rows.restype = i32
    L.cgef_plan_get_schedule.argtypes = [vp, C.POINTER(dbl), C.POINTER(i32)]
    L.cgef_plan_get_schedule.restype = i32
    L.cgef_plan_set_row_spectral.argtypes = [vp, i32]
    L.cgef_plan_set_row_spectral.restype = i32
    L.cgef_plan_get_row_spectral.argtypes = [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]
    L.cgef_plan_get_row_spectral.restype = i32
    L.cgef_plan_get_transfer.argtypes = [vp, vp]
    L.cgef_plan_get_transfer.restype = i32
    L.cgef_closure_create.argtypes = [C.POINTER(vp), C.c_uint64]
    L.cgef_closure_destroy.argtypes = [vp]
    L.cgef_closure_get_params.argtypes = [vp, vp]
    L.cgef_closure_set_params.argtypes = [vp, vp]
    L.cgef_closure_pairs_device.argtypes = [vp, i32, vp, vp, i64, vp, vp, vp, vp]
    L.cgef_closure_train_device.argtypes = [vp, vp, vp, i64, i64, i32, C.POINTER(AdamW), vp, vp]
    L.cgef_closure_forward_device.argtypes = [vp, vp, i64, vp, vp]
    L.cgef_closure_grad_device.argtypes = [vp, vp, vp, i64, vp, vp, vp]
    L.cgef_closure_pi_device.argtypes = [vp, vp, i32, vp, vp, i64, vp, dbl, C.c_uint64, dbl, vp,
                                         C.POINTER(ClosureReport), vp]
    for n in ("create", "destroy", "get_params", "set_params", "pairs_device", "train_device", "forward_device",
              "grad_device", "pi_device"):
        getattr(L, "cgef_closure_" + n).restype = i32
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != CGEF_OK:
        msg = load().cgef_last_error().decode(errors="replace")
        raise CgefError(rc, msg)


def device_count() -> int:
    return int(load().cgef_device_count())
