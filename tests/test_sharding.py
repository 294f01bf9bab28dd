"""Multi-rank sweeps without a data-path collective (cgef_b200.sharding), on CPU.

The assignment and result assembly run as world-size-2 `gloo` ranks with an injected compute
function standing in for the GPU sweep; the checks are that every (slice, scale) unit is computed
exactly once, that the loads balance on the cost of the evaluation each scale runs, and that the
assembled result (sent to rank 0 as tensors) equals one rank's.
"""
import math
import os
import socket

import numpy as np
import pytest

from cgef_b200 import sharding as SH


def fake_compute(ny=3, nx=4):
    def compute(slices, scales):
        E = np.array([[1000.0 * t + s for s in scales] for t in slices])
        Pi = np.stack([np.stack([np.full((ny, nx), 10.0 * t + s) for s in scales]) for t in slices])
        return E, Pi
    return compute


@pytest.mark.parametrize("nslices,nscales,world", [(8, 24, 2), (8, 24, 8), (1, 24, 4), (40, 6, 8), (3, 5, 4)])
def test_assignment_covers_every_unit_once_and_balances(nslices, nscales, world):
    rng = np.random.default_rng(nslices * 100 + world)
    sc = list(rng.uniform(1, 100, nscales))
    tc = list(rng.uniform(0.2, 1.0, nslices))
    a = SH.assign(sc, tc, world)
    seen = [u for part in a.units for u in part]
    assert sorted(seen) == [(t, s) for t in range(nslices) for s in range(nscales)]
    assert len(set(seen)) == len(seen)
    if (a.mode == "slices" and nslices >= 2 * world) or (a.mode == "scales" and nscales >= 2 * world):
        costs = [c * sum(sc) for c in tc] if a.mode == "slices" else [c * sum(tc) for c in sc]
        # LPT bound: max load <= average + largest item
        assert max(a.loads) <= sum(a.loads) / world + max(costs) + 1e-9


def test_single_rank_assembly():
    a = SH.assign([1.0, 2.0, 3.0], [1.0, 1.0], 1)
    E, Pi = SH.run_sharded(0, 1, 2, 3, a, fake_compute())
    assert E.shape == (2, 3) and Pi.shape == (2, 3, 3, 4)
    assert E[1, 2] == 1002.0 and Pi[1, 2, 0, 0] == 12.0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, nslices, nscales, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = [float(1 + (s * 7) % 5) for s in range(nscales)]
        tc = [float(1 + (t * 3) % 4) for t in range(nslices)]
        a = SH.assign(sc, tc, world)
        calls = []

        base = fake_compute()

        def compute(sl, scl):
            calls.append((tuple(sl), tuple(scl)))
            return base(sl, scl)

        out = SH.run_sharded(rank, world, nslices, nscales, a, compute, SH.torch_collect(a, (3, 4)))
        q.put((rank, calls, None if out is None else (out[0].tolist(), out[1].shape)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nslices,nscales", [(8, 6), (1, 6)])
def test_two_gloo_ranks_assemble_the_single_rank_result(nslices, nscales):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, nslices, nscales, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    by_rank = {r: (calls, out) for r, calls, out in got}
    # each rank ran exactly one batched sweep of its own units; together they cover the grid once
    units = set()
    for r in (0, 1):
        for sl, scl in by_rank[r][0]:
            for t in sl:
                for s in scl:
                    assert (t, s) not in units
                    units.add((t, s))
    assert len(units) == nslices * nscales
    assert by_rank[1][1] is None
    E, pishape = by_rank[0][1]
    ref, _ = SH.run_sharded(0, 1, nslices, nscales, SH.assign([1.0] * nscales, [1.0] * nslices, 1), fake_compute())
    assert np.array_equal(np.array(E), ref)
    assert tuple(pishape) == (nslices, nscales, 3, 4)


def test_cost_model_follows_the_evaluation_each_scale_runs():
    # 0.25 degree sphere: 2000 km has 168k entries per target and 347 row offsets; 100 km 873 and 19
    nx = 1440
    direct_2000 = SH.scale_cost("banded", nx=nx, entries_per_target=168_388.0, dj_lim=173)
    spectral_2000 = SH.scale_cost("banded", nx=nx, entries_per_target=168_388.0, dj_lim=173, fft_length=1440)
    direct_100 = SH.scale_cost("banded", nx=nx, entries_per_target=873.0, dj_lim=9)
    spectral_100 = SH.scale_cost("banded", nx=nx, entries_per_target=873.0, dj_lim=9, fft_length=1440)
    assert direct_2000 / spectral_2000 > 50           # measured on the device: ~109 (one snapshot)
    assert 0.5 < direct_100 / spectral_100 < 5       # comparable near the autotuner's switch (~80 km)
    assert SH.scale_cost("banded", nx=nx, dj_lim=173, fft_length=1440) < 2 * SH.scale_cost(
        "banded", nx=nx, dj_lim=9, fft_length=1440) * 173 / 9


def test_scales_mode_balances_a_mixed_direct_and_spectral_set():
    # C2's 24 scales on 2 ranks with one snapshot ("scales" mode): the small ones direct, the rest
    # row-spectral, costed by what they run
    nx = 1440
    ells = [50e3 * 40.0 ** (s / 23.0) for s in range(24)]
    costs = []
    for ell in ells:
        dj = math.ceil(ell * 2.399 / 27_798.0)
        entries = 873.0 * (ell / 1e5) ** 2
        costs.append(SH.scale_cost("banded", nx=nx, entries_per_target=entries, dj_lim=dj,
                                   fft_length=0 if ell < 80e3 else 1440))
    a = SH.assign(costs, [1.0], 2)
    assert a.mode == "scales"
    per = [c * 1.0 for c in costs]
    assert max(a.loads) <= sum(per) / 2 + max(per) + 1e-9
    # the direct-sum model (entries per target) balances its own numbers, not the device's: under the
    # costs of what each scale runs, its split is further from even
    naive = SH.assign([873.0 * (ell / 1e5) ** 2 for ell in ells], [1.0], 2)
    true_loads = [sum(per[s] for _, s in part) for part in naive.units]
    assert max(a.loads) / (sum(per) / 2) < 1.1
    assert max(a.loads) <= max(true_loads)
