"""Learned closure for the subfilter stress (no counterpart in the reference).

A pointwise MLP (5 -> 64 -> 64 -> 64 -> 3, GELU) maps the filtered velocity-gradient tensor scaled
by ell^2, and log ell, to tau; the flux is -S:tau with S from the same gradients.  Training and
inference run on the tensor cores (tcgen05, BF16 operands, FP32 accumulation) inside
libcgef_b200.so; the exact flux path (compute_Pi) makes the training pairs and judges a seeded
fraction of every result, tile by tile, falling back to itself for a slice whose judged error is
above the tolerance.  All buffers are CUDA tensors (torch); there is no host path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np

from . import _arrays as A
from . import _lib
from .errors import ArgumentError, DimensionMismatch
from .filtering import PhysicalFilterPlan

NPARAM = _lib.CLOSURE_NPARAM
NIN, NOUT = 5, 3


@dataclass
class ClosureReport:
    judged_tiles: int
    failed_tiles: int
    est_rel_l2: float
    fallbacks: int


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the closure runs on a CUDA device only")
    return torch


def _f32(a, shape_tail, name):
    torch = _torch()
    if not (A.is_device(a) and a.dtype == torch.float32):
        raise ArgumentError(f"{name} must be a float32 CUDA tensor")
    if a.dim() != len(shape_tail) + 1 or tuple(a.shape[1:]) != tuple(shape_tail):
        raise DimensionMismatch(f"{name} must have shape (n, {', '.join(map(str, shape_tail))})")
    return a.contiguous()


class Closure:
    """The network's parameters live on the GPU (FP32 master copy plus packed BF16 operand tiles)."""

    def __init__(self, seed: int = 0):
        torch = _torch()
        self._torch = torch
        self._h = C.c_void_p()
        _lib.check(_lib.load().cgef_closure_create(C.byref(self._h), C.c_uint64(seed)))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value and _lib._lib is not None:
            _lib._lib.cgef_closure_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        if self._h is None:
            raise ArgumentError("closure has been closed")
        return self._h

    # ---- parameters ----
    def get_params(self) -> np.ndarray:
        p = np.empty(NPARAM, np.float32)
        _lib.check(_lib.load().cgef_closure_get_params(self.handle, p.ctypes.data))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.shape != (NPARAM,):
            raise DimensionMismatch(f"params must have {NPARAM} entries")
        _lib.check(_lib.load().cgef_closure_set_params(self.handle, p.ctypes.data))

    # ---- network ----
    def forward(self, x):
        """Network outputs y (n, 3) for features x (n, 5)."""
        x = _f32(x, (NIN,), "x")
        y = self._torch.empty((x.shape[0], NOUT), dtype=self._torch.float32, device=x.device)
        _lib.check(_lib.load().cgef_closure_forward_device(self.handle, x.data_ptr(), x.shape[0], y.data_ptr(),
                                                           A.stream_of(x)))
        return y

    def grad(self, x, t) -> Tuple[np.ndarray, float]:
        """Gradient of mean_i sum_o (y_io - t_io)^2 over all points as one batch (no update)."""
        x = _f32(x, (NIN,), "x")
        t = _f32(t, (NOUT,), "t")
        if x.shape[0] != t.shape[0]:
            raise DimensionMismatch("x and t must hold the same points")
        g = self._torch.empty(NPARAM, dtype=self._torch.float32, device=x.device)
        l = self._torch.empty(1, dtype=self._torch.float32, device=x.device)
        _lib.check(_lib.load().cgef_closure_grad_device(self.handle, x.data_ptr(), t.data_ptr(), x.shape[0],
                                                        g.data_ptr(), l.data_ptr(), A.stream_of(x)))
        return g.cpu().numpy(), float(l.item())

    def train(self, x, t, *, batch: int = 8192, steps: int = 1, lr: float = 1e-3, beta1: float = 0.9,
              beta2: float = 0.999, eps: float = 1e-8, weight_decay: float = 1e-4) -> np.ndarray:
        """`steps` AdamW steps over consecutive batches of (x, t) (shuffle beforehand); returns the losses."""
        x = _f32(x, (NIN,), "x")
        t = _f32(t, (NOUT,), "t")
        if x.shape[0] != t.shape[0]:
            raise DimensionMismatch("x and t must hold the same points")
        losses = self._torch.empty(max(1, steps), dtype=self._torch.float32, device=x.device)
        opt = _lib.AdamW(lr, beta1, beta2, eps, weight_decay)
        _lib.check(_lib.load().cgef_closure_train_device(self.handle, x.data_ptr(), t.data_ptr(), x.shape[0], batch,
                                                         steps, C.byref(opt), losses.data_ptr(), A.stream_of(x)))
        return losses[:steps].cpu().numpy()

    # ---- flux ----
    def pi(self, plan: PhysicalFilterPlan, u, v, *, slice_masks=None, judge_fraction: float = 0.02,
           judge_seed: int = 0, tol: float = 0.05, out=None) -> Tuple[object, ClosureReport]:
        """The flux by the closure at the plan's scale for u, v of shape (..., ny, nx) (CUDA tensors).
        A seeded `judge_fraction` of the 32 x 32 tiles is recomputed exactly; a slice whose judged
        relative L2 error exceeds `tol` is recomputed by the exact path."""
        if not A.is_device(u) or not A.is_device(v):
            raise ArgumentError("u and v must be CUDA tensors")
        g = plan.grid
        if tuple(u.shape[-2:]) != g.shape or tuple(v.shape) != tuple(u.shape):
            raise DimensionMismatch("u and v must be (..., ny, nx) and equal")
        nb = int(np.prod(u.shape[:-2])) if u.dim() > 2 else 1
        u = u.contiguous()
        v = v.contiguous()
        dt = A.dtype_code(u)
        if A.dtype_code(v) != dt:
            raise ArgumentError("u and v must share a dtype")
        if out is None:
            out = A.empty_like(u)
        m = None if slice_masks is None else A.mask_bytes(slice_masks, u)
        rep = _lib.ClosureReport()
        _lib.check(_lib.load().cgef_closure_pi_device(self.handle, plan.handle, dt, u.data_ptr(), v.data_ptr(), nb,
                                                      None if m is None else m.data_ptr(), float(judge_fraction),
                                                      C.c_uint64(judge_seed), float(tol), out.data_ptr(),
                                                      C.byref(rep), A.stream_of(u)))
        return out, ClosureReport(int(rep.judged_tiles), int(rep.failed_tiles), float(rep.est_rel_l2),
                                  int(rep.fallbacks))


def training_pairs(plan: PhysicalFilterPlan, u, v, *, slice_masks=None):
    """(features, targets) of every point from the exact path: planar float32 CUDA tensors of shape
    (nbatch, 5, ny*nx) and (nbatch, 3, ny*nx); masked points hold zeros."""
    torch = _torch()
    if not A.is_device(u) or not A.is_device(v):
        raise ArgumentError("u and v must be CUDA tensors")
    g = plan.grid
    if tuple(u.shape[-2:]) != g.shape or tuple(v.shape) != tuple(u.shape):
        raise DimensionMismatch("u and v must be (..., ny, nx) and equal")
    nb = int(np.prod(u.shape[:-2])) if u.dim() > 2 else 1
    u = u.contiguous()
    v = v.contiguous()
    N = g.nx * g.ny
    feat = torch.empty((nb, NIN, N), dtype=torch.float32, device=u.device)
    targ = torch.empty((nb, NOUT, N), dtype=torch.float32, device=u.device)
    m = None if slice_masks is None else A.mask_bytes(slice_masks, u)
    _lib.check(_lib.load().cgef_closure_pairs_device(plan.handle, A.dtype_code(u), u.data_ptr(), v.data_ptr(), nb,
                                                     None if m is None else m.data_ptr(), feat.data_ptr(),
                                                     targ.data_ptr(), A.stream_of(u)))
    return feat, targ


def log_feature(ell: float) -> float:
    """The fifth input: (ln ell - ln 223607 m) / 1.4979 (ell in metres)."""
    return (np.log(ell) - 12.317637) / 1.4978661
