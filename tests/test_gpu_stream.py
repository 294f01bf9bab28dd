"""The streaming sweep (cgef_pipeline_*): snapshots submitted back to back from pinned host memory
give exactly the synchronous sweep's Pi and E, snapshot by snapshot."""
import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def test_stream_equals_the_synchronous_sweep():
    import torch
    g = S.sphere_grid(180, 90)
    g = g.with_mask(S.land_mask(g, seed=4))
    plans = [cg.plan_filter(g, cg.GaussianKernel(4.0), s) for s in (3e5, 9e5)]
    snaps = [S.sphere_fields(g, seed=40 + k, lmax=60) for k in range(5)]
    ref = [cg.coarse_grain_batch(u[None], v[None], g, scales=[3e5, 9e5], kernel=cg.GaussianKernel(4.0),
                                 filter_plans=plans) for u, v in snaps]
    st = cg.SnapshotStream(plans, nbatch=1)
    outs = []
    for u, v in snaps:
        hu = torch.from_numpy(u[None].copy()).pin_memory()
        hv = torch.from_numpy(v[None].copy()).pin_memory()
        pi = torch.empty((1, 2) + g.shape, dtype=torch.float64).pin_memory()
        e = torch.empty((1, 2), dtype=torch.float64).pin_memory()
        st.submit(hu, hv, pi, e)
        outs.append((pi, e))
    st.drain()
    for (pi, e), r in zip(outs, ref):
        assert np.array_equal(pi.numpy()[0], r.Pi[0])
        assert np.array_equal(e.numpy()[0], r.cumulative_energy[0])
    # pageable numpy buffers work too (without overlap); shapes and types are checked
    u, v = snaps[0]
    pi = np.empty((1, 2) + g.shape)
    st.submit(u[None].copy(), v[None].copy(), pi)
    st.drain()
    assert np.array_equal(pi[0], ref[0].Pi[0])
    with pytest.raises(cg.DimensionMismatch):
        st.submit(u, v, pi)
    with pytest.raises(cg.ArgumentError):
        st.submit(u[None].astype(np.float32), v[None].astype(np.float32), pi)
    st.close()


def test_sharded_sweep_on_one_rank_equals_the_batch_sweep():
    """coarse_grain_sharded with no process group (one rank, one GPU) runs every unit itself and
    assembles exactly the batch sweep's E and Pi."""
    from cgef_b200 import sharding as SH
    g = S.sphere_grid(144, 72)
    g = g.with_mask(S.land_mask(g, seed=6))
    scales = [3e5, 6e5, 1.2e6]
    U, V = zip(*[S.sphere_fields(g, seed=60 + k, lmax=50) for k in range(3)])
    U, V = np.stack(U), np.stack(V)
    E, Pi = SH.coarse_grain_sharded(U, V, g, scales=scales, kernel=cg.GaussianKernel(4.0))
    ref = cg.coarse_grain_batch(U, V, g, scales=scales, kernel=cg.GaussianKernel(4.0))
    assert np.array_equal(E, ref.cumulative_energy)
    assert np.array_equal(Pi, ref.Pi)
