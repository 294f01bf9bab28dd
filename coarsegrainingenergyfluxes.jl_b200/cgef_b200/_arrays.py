"""Host (numpy) and device (torch CUDA tensor) buffers handed to the C ABI."""
from __future__ import annotations

import numpy as np

from ._lib import F32, F64


def is_device(a) -> bool:
    return getattr(a, "is_cuda", False) is True


def dtype_code(a) -> int:
    if is_device(a):
        import torch
        if a.dtype == torch.float64:
            return F64
        if a.dtype == torch.float32:
            return F32
    else:
        if a.dtype == np.float64:
            return F64
        if a.dtype == np.float32:
            return F32
    raise TypeError(f"fields must be float64 or float32, got {a.dtype}")


def ptr(a) -> int:
    if is_device(a) or hasattr(a, "data_ptr"):  # CUDA tensors, and host (e.g. pinned) torch tensors
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return a.data_ptr()
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("host arrays must be C-contiguous ((ny, nx) with x fastest)")
    return a.ctypes.data


def host(a, dtype=None) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype if dtype is not None else (a.dtype if a.dtype in (np.float32, np.float64) else np.float64))


def empty_like(a, shape=None):
    shape = tuple(a.shape) if shape is None else tuple(shape)
    if is_device(a):
        import torch
        return torch.empty(shape, dtype=a.dtype, device=a.device)
    return np.empty(shape, dtype=a.dtype)


def stream_of(a) -> int:
    import torch
    return torch.cuda.current_stream(a.device).cuda_stream


def mask_bytes(m, device_like=None):
    """uint8 mask buffer (1 = active) on the host, or on the device of `device_like`."""
    if m is None:
        return None
    if device_like is not None and is_device(device_like):
        import torch
        if is_device(m):
            return m.to(torch.uint8).contiguous()
        return torch.as_tensor(np.ascontiguousarray(m, dtype=np.uint8), device=device_like.device)
    if is_device(m):
        m = m.cpu().numpy()
    return np.ascontiguousarray(m, dtype=np.uint8)
