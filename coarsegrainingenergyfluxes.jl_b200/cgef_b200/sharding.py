"""Multi-GPU sweeps: independent (slice, scale) units shared out across ranks.

A coarse-graining sweep is a grid of independent units -- one Pi field and one E(l) per (slice,
scale) -- that share only read-only plans (the reference parallelises the same axis over threads,
Pipeline.jl:686-717 and ext/CoarseGrainingEnergyFluxesOhMyThreadsExt.jl:248-286).  So ranks take
disjoint units with no data-path collective: every rank runs its own units on its own GPU, and the
results meet once at the end (a gather of Pi slabs and E values to rank 0).

Units are assigned longest-processing-time first by a cost model (footprint entries x active
targets), deterministically, so every rank computes the same assignment without communicating.
When there are at least as many slices as ranks, whole slices are dealt out (each rank runs all
scales of its slices in one batched sweep); otherwise scales are dealt out.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np


@dataclass(frozen=True)
class Assignment:
    """units[r] = the (slice, scale) pairs rank r computes; mode is "slices" or "scales"."""

    mode: str
    units: Tuple[Tuple[Tuple[int, int], ...], ...]
    loads: Tuple[float, ...]


def lpt(costs: Sequence[float], world: int) -> List[List[int]]:
    """Longest-processing-time-first greedy: item indices per rank (deterministic ties)."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    loads = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (loads[q], q))
        out[r].append(i)
        loads[r] += float(costs[i])
    for r in range(world):
        out[r].sort()
    return out


def assign(scale_costs: Sequence[float], slice_costs: Sequence[float], world: int) -> Assignment:
    """Shares the (slice, scale) grid out over `world` ranks.

    scale_costs[s]: relative cost of one slice at scale s (footprint entries per target);
    slice_costs[t]: relative cost of slice t (its active targets)."""
    ns, nt = len(scale_costs), len(slice_costs)
    if world < 1:
        raise ValueError("world must be >= 1")
    if nt >= world:
        per = [float(c) * float(sum(scale_costs)) for c in slice_costs]
        parts = lpt(per, world)
        units = tuple(tuple((t, s) for t in part for s in range(ns)) for part in parts)
        loads = tuple(sum(per[t] for t in part) for part in parts)
        return Assignment("slices", units, loads)
    per = [float(c) * float(sum(slice_costs)) for c in scale_costs]
    parts = lpt(per, world)
    units = tuple(tuple((t, s) for t in range(nt) for s in part) for part in parts)
    loads = tuple(sum(per[s] for s in part) for part in parts)
    return Assignment("scales", units, loads)


def plan_costs(plans, grid, slice_masks=None, nslices: int = 1) -> Tuple[List[float], List[float]]:
    """Cost model: entries per active target for each scale's plan, active targets per slice."""
    sc = []
    for p in plans:
        if p.engine == "banded":
            sc.append(float(p.info.nentries) / max(1, int(p.info.nbands)))
        elif p.engine == "separable":
            sc.append(float(2 * p.info.di_max + 2 * p.info.dj_lim + 2))
        else:
            sc.append(float(2 * p.info.dj_lim + 1))
    if slice_masks is not None:
        m = np.asarray(slice_masks).reshape(-1, grid.ny * grid.nx)
        tc = [float(x) for x in m.sum(axis=1)]
    else:
        act = float(grid.nx * grid.ny if grid.mask is None else grid.mask.sum())
        tc = [act] * nslices
    return sc, tc


def run_sharded(rank: int, world: int, nslices: int, nscales: int, assignment: Assignment,
                compute: Callable[[List[int], List[int]], Tuple[np.ndarray, Optional[np.ndarray]]],
                gather: Optional[Callable[[object], Optional[List[object]]]] = None):
    """Runs this rank's units and assembles the full sweep on rank 0.

    compute(slices, scales) -> (E[len(slices), len(scales)], Pi[len(slices), len(scales), ny, nx] or None)
    runs one batched sweep on this rank's GPU.  gather(obj) returns the list of every rank's obj on
    rank 0 (None elsewhere); with one rank it may be omitted.  Returns (E, Pi) on rank 0, else None.
    """
    mine = assignment.units[rank]
    results: Dict[Tuple[int, int], Tuple[float, Optional[np.ndarray]]] = {}
    if mine:
        if assignment.mode == "slices":
            slices = sorted({t for t, _ in mine})
            scales = list(range(nscales))
            batches = [(slices, scales)]
        else:
            slices = list(range(nslices))
            scales = sorted({s for _, s in mine})
            batches = [(slices, scales)]
        for sl, sc in batches:
            E, Pi = compute(sl, sc)
            for a, t in enumerate(sl):
                for b, s in enumerate(sc):
                    results[(t, s)] = (float(E[a, b]), None if Pi is None else np.asarray(Pi[a, b]))
    everything = [results] if gather is None else gather(results)
    if everything is None:
        return None
    E = np.full((nslices, nscales), np.nan)
    Pi_parts: Dict[Tuple[int, int], np.ndarray] = {}
    for part in everything:
        for (t, s), (e, pi) in part.items():
            if not np.isnan(E[t, s]):
                raise RuntimeError(f"unit ({t}, {s}) computed twice")
            E[t, s] = e
            if pi is not None:
                Pi_parts[(t, s)] = pi
    if np.isnan(E).any():
        raise RuntimeError("some units were not computed")
    Pi = None
    if Pi_parts:
        shape = next(iter(Pi_parts.values())).shape
        Pi = np.empty((nslices, nscales) + shape, dtype=next(iter(Pi_parts.values())).dtype)
        for (t, s), pi in Pi_parts.items():
            Pi[t, s] = pi
    return E, Pi


def torch_gather(group=None) -> Callable[[object], Optional[List[object]]]:
    """Gather of picklable objects to rank 0 over torch.distributed (gloo or nccl)."""
    import torch.distributed as dist

    def g(obj):
        world = dist.get_world_size(group)
        rank = dist.get_rank(group)
        out = [None] * world if rank == 0 else None
        dist.gather_object(obj, out, dst=0, group=group)
        return out

    return g


def coarse_grain_sharded(u, v, grid, *, scales, kernel, mask_strategy=None, slice_masks=None,
                         want_pi: bool = True, group=None):
    """coarse_grain_batch over all ranks of torch.distributed's default (or given) group: every rank
    plans the scales, computes its units on its own GPU, and rank 0 receives (E, Pi) for the whole
    (slice, scale) grid.  u, v: (nslices, ny, nx) host arrays, identical on every rank."""
    import torch.distributed as dist

    from . import _arrays as A  # noqa: F401
    from .filtering import ZeroFill, plan_filter
    from .pipeline import _sweep

    strat = mask_strategy if mask_strategy is not None else ZeroFill()
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    nsl = int(u.shape[0])
    base = grid.with_mask(None) if slice_masks is not None else grid
    plans = [plan_filter(base, kernel, float(s), mask_strategy=strat) for s in scales]
    sc, tc = plan_costs(plans, grid, slice_masks, nsl)
    asg = assign(sc, tc, world)

    def compute(sl, scl):
        m = None if slice_masks is None else np.ascontiguousarray(np.asarray(slice_masks)[sl])
        Pi, E = _sweep(np.ascontiguousarray(u[sl]), np.ascontiguousarray(v[sl]), base, [plans[s] for s in scl],
                       len(sl), m, want_pi)
        return E, Pi

    return run_sharded(rank, world, nsl, len(scales), asg, compute, torch_gather(group) if world > 1 else None)
