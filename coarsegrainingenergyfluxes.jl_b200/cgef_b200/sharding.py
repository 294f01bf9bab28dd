"""Multi-GPU sweeps: independent (slice, scale) units shared out across ranks.

A coarse-graining sweep is a grid of independent units -- one Pi field and one E(l) per (slice,
scale) -- that share only read-only plans (the reference parallelises the same axis over threads,
Pipeline.jl:686-717 and ext/CoarseGrainingEnergyFluxesOhMyThreadsExt.jl:248-286).  So ranks take
disjoint units with no data-path collective: every rank runs its own units on its own GPU, and the
results meet once at the end (every rank's Pi slabs and E values sent to rank 0).

Units are assigned longest-processing-time first by a cost model (the device time per target of the
evaluation each scale's plan runs, times active targets), deterministically, so every rank computes the
same assignment without communicating.  When there are at least as many slices as ranks, whole slices
are dealt out (each rank runs all scales of its slices in one batched sweep); otherwise scales are dealt
out.  Results travel as tensors, rank by rank to rank 0 (each rank's units are known to every rank from
the assignment, so nothing but the values is sent).
"""
from __future__ import annotations

import math
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

    scale_costs[s]: relative cost of one slice at scale s (scale_cost: device time per target);
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


# Device time per target, calibrated on a B200 (the flux of the 0.25-degree sphere, one snapshot): the
# direct gather takes 0.40 ms for 0.73e6 active targets x 873 entries; the row-spectral evaluation's two
# FFT kernels 0.11 ms for 720 rows of 1440 points and its accumulation 0.065 ms for 19 row offsets.
DIRECT_S_PER_ENTRY = 0.40e-3 / (0.73e6 * 873)
SPECTRAL_FFT_S_PER_ROW = 0.11e-3 / 720      # both transforms of a 1440-point row, all quantities
SPECTRAL_ACC_S_PER_ROW_OFFSET = 0.065e-3 / (720 * 19)  # one row offset of a 1440-point row's 721 bins


def scale_cost(engine: str, *, nx: int, entries_per_target: float = 0.0, dj_lim: int = 0, di_max: int = 0,
               fft_length: int = 0, periodic_x: bool = True) -> float:
    """Device seconds per target of one scale, for the evaluation its plan runs (calibrated above).

    - banded, direct gather: per footprint entry;
    - banded, row-spectral: per target row, the two FFTs (L log L, scaled from 1440 points) and the
      accumulation over 2 dj_lim + 1 row offsets of L/2 + 1 bins, shared by the row's nx targets;
    - separable: both passes' taps, at the direct gather's rate per tap;
    - prefix sum: a running sum over the (tripled, periodic) row plus two prefix reads per row offset.
    Only ratios matter to the assignment.
    """
    if engine == "banded":
        if fft_length > 0:
            L = fft_length
            fft = SPECTRAL_FFT_S_PER_ROW * (L * math.log2(max(L, 2))) / (1440 * math.log2(1440))
            acc = SPECTRAL_ACC_S_PER_ROW_OFFSET * (2 * dj_lim + 1) * (L // 2 + 1) / 721
            return (fft + acc) / max(nx, 1)
        return DIRECT_S_PER_ENTRY * float(entries_per_target)
    if engine == "separable":
        return DIRECT_S_PER_ENTRY * float(2 * di_max + 2 * dj_lim + 2)
    return DIRECT_S_PER_ENTRY * ((3.0 if periodic_x else 1.0) + 2.0 * (2 * dj_lim + 1))


def plan_scale_cost(p) -> float:
    """scale_cost of a PhysicalFilterPlan, with the evaluation it is set to run."""
    info = p.info
    L = 0
    if p.engine == "banded":
        _, enabled, length = p.row_spectral
        L = length if enabled else 0
    return scale_cost(p.engine, nx=p.grid.nx, entries_per_target=float(info.nentries) / max(1, int(info.nbands)),
                      dj_lim=int(info.dj_lim), di_max=int(info.di_max), fft_length=L,
                      periodic_x=bool(p.grid.periodic[0]))


def plan_costs(plans, grid, slice_masks=None, nslices: int = 1) -> Tuple[List[float], List[float]]:
    """Cost model: each scale's plan_scale_cost, and the active targets of each slice."""
    sc = [plan_scale_cost(p) for p in plans]
    if slice_masks is not None:
        m = np.asarray(slice_masks).reshape(-1, grid.ny * grid.nx)
        tc = [float(x) for x in m.sum(axis=1)]
    else:
        act = float(grid.nx * grid.ny if grid.mask is None else grid.mask.sum())
        tc = [act] * nslices
    return sc, tc


def run_sharded(rank: int, world: int, nslices: int, nscales: int, assignment: Assignment,
                compute: Callable[[List[int], List[int]], Tuple[np.ndarray, Optional[np.ndarray]]],
                collect: Optional[Callable] = None):
    """Runs this rank's units and assembles the full sweep on rank 0.

    compute(slices, scales) -> (E[len(slices), len(scales)], Pi[len(slices), len(scales), ny, nx] or None)
    runs one batched sweep on this rank's GPU.  collect(E_units, Pi_units) moves every rank's results
    to rank 0 -- E_units[n] and Pi_units[n, ny, nx] in the order of assignment.units[rank] -- and returns
    the list of every rank's (E_units, Pi_units) there (None elsewhere); with one rank it may be omitted.
    Returns (E, Pi) on rank 0, else None.
    """
    mine = assignment.units[rank]
    E_units = np.zeros(len(mine))
    Pi_units = None
    if mine:
        if assignment.mode == "slices":
            slices = sorted({t for t, _ in mine})
            scales = list(range(nscales))
        else:
            slices = list(range(nslices))
            scales = sorted({s for _, s in mine})
        E, Pi = compute(slices, scales)
        at = {(t, s): (a, b) for a, t in enumerate(slices) for b, s in enumerate(scales)}
        for n, u in enumerate(mine):
            a, b = at[u]
            E_units[n] = E[a, b]
            if Pi is not None:
                if Pi_units is None:
                    Pi_units = np.empty((len(mine),) + tuple(np.asarray(Pi).shape[2:]), dtype=np.asarray(Pi).dtype)
                Pi_units[n] = Pi[a, b]
    parts = [(E_units, Pi_units)] if collect is None else collect(E_units, Pi_units)
    if parts is None:
        return None
    E = np.full((nslices, nscales), np.nan)
    Pi = None
    for r, (Er, Pr) in enumerate(parts):
        for n, (t, s) in enumerate(assignment.units[r]):
            if not np.isnan(E[t, s]):
                raise RuntimeError(f"unit ({t}, {s}) computed twice")
            E[t, s] = Er[n]
            if Pr is not None:
                if Pi is None:
                    Pi = np.empty((nslices, nscales) + tuple(Pr.shape[1:]), dtype=Pr.dtype)
                Pi[t, s] = Pr[n]
    if np.isnan(E).any():
        raise RuntimeError("some units were not computed")
    return E, Pi


def torch_collect(assignment: Assignment, field_shape: Optional[Tuple[int, ...]], dtype=np.float64, group=None):
    """collect() for run_sharded over torch.distributed: each rank > 0 sends its E and Pi units to rank 0
    as tensors (CUDA tensors over NCCL, host tensors over gloo), and rank 0 receives rank by rank into
    buffers sized from the assignment -- no sizes, no pickles.  field_shape: (ny, nx), or None without Pi."""
    import torch
    import torch.distributed as dist

    tdt = torch.float32 if np.dtype(dtype) == np.float32 else torch.float64

    def on_device():
        return dist.get_backend(group) == "nccl"

    def to_t(a, dt):
        t = torch.from_numpy(np.ascontiguousarray(a)).to(dt)
        return t.cuda() if on_device() else t

    def c(E_units, Pi_units):
        rank = dist.get_rank(group)
        world = dist.get_world_size(group)
        dev = "cuda" if on_device() else "cpu"
        if rank != 0:
            if len(assignment.units[rank]):
                dist.send(to_t(E_units, torch.float64), dst=0, group=group)
                if field_shape is not None:
                    dist.send(to_t(Pi_units, tdt), dst=0, group=group)
            return None
        parts = [(E_units, Pi_units)]
        for r in range(1, world):
            n = len(assignment.units[r])
            if n == 0:
                parts.append((np.zeros(0), None))
                continue
            Er = torch.empty(n, dtype=torch.float64, device=dev)
            dist.recv(Er, src=r, group=group)
            Pr = None
            if field_shape is not None:
                Pr = torch.empty((n,) + tuple(field_shape), dtype=tdt, device=dev)
                dist.recv(Pr, src=r, group=group)
                Pr = Pr.cpu().numpy()
            parts.append((Er.cpu().numpy(), Pr))
        return parts

    return c


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

    collect = None
    if world > 1:
        collect = torch_collect(asg, grid.shape if want_pi else None, np.asarray(u).dtype, group)
    return run_sharded(rank, world, nsl, len(scales), asg, compute, collect)
