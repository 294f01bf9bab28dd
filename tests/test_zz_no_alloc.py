"""The allocation-free filter entry point (cgef_filter_device_noalloc).

Some callers cannot let a library allocate device memory during a call -- a host whose device
memory belongs to its own pool allocator, or a loop with a fixed memory budget.  For them the
library offers the footprint filter with its scratch in a fixed 64 MiB array compiled into the
library.  This test calls it through the C ABI twice in a row, on different fields, and checks
each result against the allocating entry point cgef_filter_device within the tolerance the other
parity tests use, and one case against the FP64 oracle; it checks that the device's free memory does
not move across calls of the entry point on a fresh plan (while the allocating entry point's first
call on that plan does move it), and that a grid too large for the array is refused.  The file sorts
last so a failure here comes after every other test has run; it needs nothing from them.
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import _lib
from cgef_b200 import synthetic as S
from helpers import oracle_plan

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-10  # the filtered-field tolerance of tests/test_gpu_parity.py


def _max_rel(x, ref):
    scale = float(np.max(np.abs(ref)))
    return float(np.max(np.abs(x - ref))) / (scale if scale > 0 else 1.0)


@pytest.mark.parametrize("strategy", [cg.ZeroFill(), cg.Deformable()])
def test_noalloc_filter_matches_allocating_filter_twice(strategy):
    torch = pytest.importorskip("torch")
    L = _lib.load()
    g = S.sphere_grid(180, 90)
    g = g.with_mask(S.land_mask(g, seed=4))
    plan = cg.plan_filter(g, cg.GaussianKernel(4.0), 6e5, mask_strategy=strategy)
    rng = np.random.default_rng(42)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        f = torch.from_numpy(rng.standard_normal((2,) + g.shape)).cuda()
        ref = torch.empty_like(f)
        got = torch.full_like(f, float("nan"))
        _lib.check(L.cgef_filter_device(plan.handle, _lib.F64, f.data_ptr(), ref.data_ptr(), 2, stream))
        _lib.check(L.cgef_filter_device_noalloc(plan.handle, _lib.F64, f.data_ptr(), got.data_ptr(), 2, stream))
        torch.cuda.synchronize()
        assert _max_rel(got.cpu().numpy(), ref.cpu().numpy()) < FIELD_TOL, f"call {call}"


def test_noalloc_filter_float32_and_other_engines():
    torch = pytest.importorskip("torch")
    L = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    cases = [
        (S.cartesian_grid(128, 1000.0), cg.GaussianKernel(4.0), 8000.0),   # separable
        (S.sphere_grid(180, 90), cg.TopHatKernel(), 9e5),                   # prefix sum
    ]
    rng = np.random.default_rng(7)
    for g, k, scale in cases:
        plan = cg.plan_filter(g, k, scale)
        for call in range(2):
            f = torch.from_numpy(rng.standard_normal((1,) + g.shape).astype(np.float32)).cuda()
            ref = torch.empty_like(f)
            got = torch.empty_like(f)
            _lib.check(L.cgef_filter_device(plan.handle, _lib.F32, f.data_ptr(), ref.data_ptr(), 1, stream))
            _lib.check(L.cgef_filter_device_noalloc(plan.handle, _lib.F32, f.data_ptr(), got.data_ptr(), 1, stream))
            torch.cuda.synchronize()
            assert _max_rel(got.cpu().numpy(), ref.cpu().numpy()) < FIELD_TOL, (plan.engine, call)


def test_noalloc_filter_rejects_grids_beyond_its_array():
    torch = pytest.importorskip("torch")
    L = _lib.load()
    g = S.sphere_grid(1440, 720)
    plan = cg.plan_filter(g, cg.GaussianKernel(4.0), 1e5)
    f = torch.zeros((8,) + g.shape, dtype=torch.float64, device="cuda")
    out = torch.empty_like(f)
    rc = L.cgef_filter_device_noalloc(plan.handle, _lib.F64, f.data_ptr(), out.data_ptr(), 8,
                                      torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.CGEF_EINVAL
    assert b"fixed" in L.cgef_last_error()


def test_noalloc_filter_allocates_nothing_and_matches_the_oracle():
    torch = pytest.importorskip("torch")
    L = _lib.load()
    g = S.sphere_grid(240, 120)
    g = g.with_mask(S.land_mask(g, seed=6))
    rng = np.random.default_rng(11)
    fields = [rng.standard_normal((1,) + g.shape) for _ in range(3)]
    dev = [torch.from_numpy(f).cuda() for f in fields]
    outs = [torch.empty_like(d) for d in dev]
    stream = torch.cuda.current_stream().cuda_stream
    plan = cg.plan_filter(g, cg.GaussianKernel(4.0), 7e5)  # a fresh plan: its workspace is empty
    # the first call may load kernel modules (lazy loading); it must not need the plan's workspace
    _lib.check(L.cgef_filter_device_noalloc(plan.handle, _lib.F64, dev[0].data_ptr(), outs[0].data_ptr(), 1, stream))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for k in (1, 2, 0):
        _lib.check(L.cgef_filter_device_noalloc(plan.handle, _lib.F64, dev[k].data_ptr(), outs[k].data_ptr(), 1,
                                                stream))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0, "the allocation-free entry point changed free device memory"
    ref = oracle_plan(g, cg.GaussianKernel(4.0), 7e5).filter(fields[1][0], max(1, os.cpu_count() or 1))
    assert _max_rel(outs[1].cpu().numpy()[0], ref) < FIELD_TOL
    # the measurement can see an allocation: the allocating entry point's first call grows the workspace
    alloc = torch.empty_like(dev[0])
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    _lib.check(L.cgef_filter_device(plan.handle, _lib.F64, dev[2].data_ptr(), alloc.data_ptr(), 1, stream))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] < free1
    assert _max_rel(outs[2].cpu().numpy(), alloc.cpu().numpy()) < FIELD_TOL
