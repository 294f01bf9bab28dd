#!/usr/bin/env python3
"""Benchmark: Pi grid-points x scales per second on one or more B200s.

Default workload (one step): compute_Π! on the 0.25-degree global sphere, 1440 x 720 cells,
Gaussian alpha = 4, l = 100 km, ZeroFill, ~30% land -- one scale x one snapshot per GPU per step
(weak scaling: every rank takes its own seeded snapshot).  Other workloads (--workload):
  sweep24x8 : 24 scales (50-2000 km, log-spaced) x 8 snapshots per step, Pi and E(l)
  cart256   : 256^2 doubly periodic Cartesian, dx = 1 km, l = 8 km (separable engine)
  levels40  : regional 400 x 600 x 40 levels, FP32 storage, 6 scales 25-400 km, one mask per level
  tophat    : the sphere1 grid and mask with the package's default kernel, the exact top-hat at
              l = 100 km (the prefix-sum engine)
  closure8  : the learned closure: trained on exact-path pairs of two snapshots at 8 scales
              (50-1000 km, 10^7 points), then Pi of a fresh snapshot at the 8 scales by the closure
              (2% of tiles judged exactly, per-slice fallback above the tolerance) against the plain
              sweep of the same scales

`value` times the device-resident path (inputs already in HBM, an L2 flush between steps inside
the timed region); `e2e` times the host C-ABI call (pinned host inputs copied in, Pi copied out)
every step.  The default run (sphere1, one rank) adds sub-records to its line: the metric's "plain vs
batched/closure" -- `batched` (the sweep24x8 workload, measured the same way) and `closure` (the
closure8 workload) -- and `tophat` (the tophat workload).  `--impl reference` times the CPU FP64 oracle -- the restated threaded
reference path -- on the host's cores instead, with the same `config`.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "coarsegrainingenergyfluxes.jl_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "Π grid-points×scales/s, 0.25° sphere; plain vs batched/closure; rel-L2 vs FP64"
UNIT = "grid-points*scales/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sphere1", choices=["sphere1", "sweep24x8", "cart256", "levels40", "closure8", "tophat"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--snapshots", type=int, default=1, help="snapshots per step of the sphere1 workload")
    ap.add_argument("--scale-km", type=float, default=None, help="filter scale of the sphere1 workload (km)")
    ap.add_argument("--closure-tol", type=float, default=0.05,
                    help="closure8: judged Pi rel-L2 above which a slice falls back to the exact path")
    ap.add_argument("--closure-epochs", type=float, default=3.0, help="closure8: training epochs over 10^7 points")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default banded schedules")
    ap.add_argument("--evaluation", choices=("auto", "direct", "spectral"), default="auto",
                    help="footprint sums of the banded engine: the autotuner's choice per scale (default), the "
                         "direct gather, or the row-spectral evaluation")
    ap.add_argument("--no-subrecords", action="store_true",
                    help="sphere1: time the headline only, without the batched (24 scales x 8 snapshots), "
                         "closure and top-hat sub-records")
    ap.add_argument("--batched-steps", type=int, default=6, help="timed steps of the batched sub-record")
    ap.add_argument("--clocks-out", default=None,
                    help="directory for the nvidia-smi clock samples (default: a temporary directory)")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------------------------
def sweep_scales():
    return [50e3 * 40.0 ** (s / 23.0) for s in range(24)]


def closure_scales():
    return [50e3 * 20.0 ** (s / 7.0) for s in range(8)]


def make_workload(name: str, rank: int, snapshots: int = 1, scale_km=None):
    """Returns dict(grid, u, v, scales, slice_masks, kernel, nslices, desc)."""
    import cgef_b200 as cg
    from cgef_b200 import synthetic as S
    if name == "sphere1":
        g = S.sphere_grid()
        g = g.with_mask(S.land_mask(g, seed=1))
        us, vs = zip(*[S.sphere_fields(g, seed=100 + snapshots * rank + t) for t in range(snapshots)])
        ell = 1e5 if scale_km is None else 1e3 * scale_km
        return dict(grid=g, u=np.stack(us), v=np.stack(vs), scales=[ell], slice_masks=None,
                    kernel=cg.GaussianKernel(4.0),
                    desc=f"sphere-0.25deg-1440x720-gauss-a4-l{ell / 1e3:g}km-zerofill-30pct-land"
                         + ("" if snapshots == 1 else f"-x{snapshots}snapshots"),
                    dtype="f64")
    if name == "sweep24x8":
        g = S.sphere_grid()
        g = g.with_mask(S.land_mask(g, seed=1))
        us, vs = zip(*[S.sphere_fields(g, seed=100 + 8 * rank + t) for t in range(8)])
        return dict(grid=g, u=np.stack(us), v=np.stack(vs), scales=sweep_scales(), slice_masks=None,
                    kernel=cg.GaussianKernel(4.0),
                    desc="sphere-0.25deg-1440x720-gauss-a4-24scales-50to2000km-x8snapshots-zerofill-30pct-land",
                    dtype="f64")
    if name == "tophat":
        g = S.sphere_grid()
        g = g.with_mask(S.land_mask(g, seed=1))
        u, v = S.sphere_fields(g, seed=100 + rank)
        return dict(grid=g, u=u[None], v=v[None], scales=[1e5], slice_masks=None, kernel=cg.TopHatKernel(),
                    desc="sphere-0.25deg-1440x720-tophat-l100km-zerofill-30pct-land", dtype="f64")
    if name == "cart256":
        g = S.cartesian_grid()
        u, v = S.cartesian_fields(seed=rank)
        return dict(grid=g, u=u[None], v=v[None], scales=[8000.0], slice_masks=None, kernel=cg.GaussianKernel(4.0),
                    desc="cartesian-256x256-dx1km-periodic-gauss-a4-l8km-zerofill", dtype="f64")
    if name == "closure8":
        g = S.sphere_grid()
        g = g.with_mask(S.land_mask(g, seed=1))
        u, v = S.sphere_fields(g, seed=4 + rank)
        return dict(grid=g, u=u[None], v=v[None], scales=closure_scales(), slice_masks=None,
                    kernel=cg.GaussianKernel(4.0),
                    desc="closure-sphere-0.25deg-1440x720-gauss-a4-8scales-50to1000km-zerofill-30pct-land",
                    dtype="f64")
    grid, U, V, M, _ = S.regional_levels(seed=2 + rank)
    scales = [25e3 * 16.0 ** (s / 5.0) for s in range(6)]
    return dict(grid=grid, u=U, v=V, scales=scales, slice_masks=M, kernel=cg.GaussianKernel(4.0),
                desc="regional-0.25deg-400x600x40levels-f32-gauss-a4-6scales-25to400km-per-level-masks",
                dtype="f32")


def algorithmic_flops(plans, grid, nslices, slice_masks) -> float:
    """Sum over active targets of footprint entries x K x 2 (K = 9 on the sphere, 5 on the plane)."""
    K = 9 if grid.is_spherical else 5
    total = 0.0
    for p in plans:
        if p.engine == "banded":
            n = p.band_counts().astype(np.float64)
            if slice_masks is not None:
                act = slice_masks.reshape(nslices, grid.ny, grid.nx).sum(axis=(0, 2)).astype(np.float64)
            else:
                m = np.ones(grid.shape) if grid.mask is None else grid.mask
                act = m.sum(axis=1).astype(np.float64) * nslices
            if n.size == 1:
                n = np.full(grid.ny, n[0])
            total += float((act * n).sum()) * K * 2
        elif p.engine == "separable":
            total += grid.nx * grid.ny * nslices * 2 * (2 * p.info.di_max + 1 + 2 * p.info.dj_lim + 1) * K
    return total


def apply_evaluation(plans, how: str) -> None:
    """auto: the autotuner's choice per plan; direct / spectral: forced where the plan allows."""
    for p in plans:
        if how == "direct" and p.engine == "banded":
            p.set_row_spectral(False)
        elif how == "spectral" and p.engine == "banded" and p.row_spectral[0]:
            p.set_row_spectral(True)


def uses_row_spectral(p) -> bool:
    return p.engine == "banded" and p.row_spectral[1]


def rowspec_bytes(p, grid, nslices, na, nplanes, nout, masked, raw=False) -> float:
    """Compulsory DRAM bytes of one row-spectral launch: the staged planes read, the source spectra
    written and read once, the kernel spectra read, the summed spectra written and read, then either
    (raw: the flux, whose strain pass finishes the sums) the unnormalised sums written once, or (a
    filter) the unnormalised sums written and read, the outputs written and the mask read."""
    L = p.row_spectral[2]
    nk = L // 2 + 1
    D = p.info.dj_lim
    nrows = (grid.ny if grid.is_spherical else 1) * (2 * D + 1)
    N = grid.nx * grid.ny
    spec = nslices * grid.ny * na * nk * 16
    base = nslices * nplanes * N * 8 + 4 * spec + nrows * nk * 8
    if raw:
        return float(base + nslices * na * N * 8)
    return float(base + 2 * nslices * na * N * 8 + nslices * nout * N * 8 + (nslices * N if masked else 0))


def prefix_bytes(p, grid, nslices, na, nplanes, nout, masked) -> float:
    """Compulsory DRAM bytes of one prefix-sum launch: the staged planes read, the prefix sums of every
    quantity along the tripled (periodic) or single row written once and read once, the outputs
    written (and the mask read)."""
    N = grid.nx * grid.ny
    ne = (3 if grid.periodic[0] else 1) * grid.nx
    P = nslices * na * grid.ny * (ne + 1) * 8
    return float(nslices * nplanes * N * 8 + 2 * P + nslices * nout * N * 8 + (nslices * N if masked else 0))


def committed_traffic(key: str, nsl: int, scale_km=None):
    """DRAM bytes (read + write) per launch from the committed ncu summary, how they were obtained, and
    the one-snapshot figure.

    The summaries hold one snapshot's traffic at the workload's own scale.  A launch of several
    snapshots has no capture of its own, and its traffic is not that figure times the snapshots (the
    kernel spectra are read once per launch, and L2 holds less of a larger launch), so it reports None
    with the one-snapshot figure beside it.  A scale other than the workload's own has no capture."""
    if scale_km is not None:
        return None, None, None
    try:
        t = json.load(open(os.path.join(ROOT, "profiles", "ncu_traffic.json"))).get(key)
    except Exception:
        t = None
    if t is None:
        return None, None, None
    if nsl == 1:
        return float(t), "ncu capture of one launch (profiles/ncu_traffic.json)", float(t)
    return None, f"no capture of {nsl} snapshots per launch; one-snapshot capture beside it", float(t)


def hbm_peak():
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), \
            "measured: MEASURED_PEAKS.json hbm_gbs (STREAM-style copy on this pool's B200s)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s (earlier measurement on this pool)"


# ---------------------------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int, out_dir=None):
        import tempfile
        d = out_dir if out_dir else tempfile.mkdtemp(prefix="cgef_clocks_")
        self.path = os.path.join(d, f"clocks_rank{device_index}.csv")
        self.proc = None
        self.dev = device_index

    def _smi_index(self):
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.dev)
            return "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
        except Exception:
            return str(self.dev)

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self._smi_index(), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[4:]))
            except ValueError:
                continue
        if not rows:
            return None
        sm = [r[0] for r in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, val in zip(names, r[2][1:]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(r[1] for r in rows), "samples": len(rows),
                "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------------------------
# CPU baseline / reference arm: the FP64 oracle's threaded path
# ---------------------------------------------------------------------------------------------
def oracle_rate(wl, budget_s: float):
    """Rate of the oracle's OpenMP compute_Pi (the restated reference threaded path) on this host.

    A unit is Pi for one (slice, scale).  With one unit it is repeated within the budget; otherwise
    a bounded subset of units is timed and the whole workload's time is extrapolated linearly in
    (active targets x footprint entries), the direct sum's cost.  Also returns the first timed unit's
    FP64 Pi with its (slice, scale index), against which the GPU result is compared."""
    import oracle as O
    g = wl["grid"]
    nthreads = O.max_threads()
    nsl = wl["u"].shape[0]
    scales = list(wl["scales"])
    alpha = float(getattr(wl["kernel"], "alpha", 0.0))
    okernel = O.GAUSSIAN if alpha > 0 else O.TOPHAT
    masks = wl["slice_masks"]

    def ogrid(mask):
        return O.Grid(O.SPHERE if g.is_spherical else O.CART, g.nx, g.ny, g.x.start, g.x.step, g.y.start, g.y.step,
                      g.geometry.R if g.is_spherical else 6.371e6, g.periodic[0], g.periodic[1], mask)

    def mask_of(t):
        return masks[t] if masks is not None else g.mask

    def active(t):
        m = mask_of(t)
        return float(g.nx * g.ny if m is None else np.count_nonzero(m))

    entries = [float(O.count_entries(ogrid(None), okernel, alpha, s)) for s in scales]
    cost = lambda t, s: active(t) * entries[s]
    # subset: scales spread over the range whose estimated time fits the budget
    order = sorted(range(len(scales)), key=lambda s: entries[s])
    plans = {}

    first = {}

    def run(t, s):
        key = (t if masks is not None else -1, s)
        if key not in plans:
            plans[key] = O.Plan(ogrid(mask_of(t)), okernel, alpha, scales[s], O.ZEROFILL)
        p = plans[key]
        u = np.asarray(wl["u"][t], dtype=np.float64)
        v = np.asarray(wl["v"][t], dtype=np.float64)
        t0 = time.perf_counter()
        out = p.compute_pi(u, v, nthreads)
        dt = time.perf_counter() - t0
        if not first:
            first.update(slice=t, scale=s, Pi=out["Pi"])
        return dt

    run(0, order[0])  # warm-up
    timed, spent, ccost = [], 0.0, 0.0
    t0 = run(0, order[0])
    timed.append((0, order[0]))
    spent += t0
    ccost += cost(0, order[0])
    per_cost = t0 / cost(0, order[0])
    picks = [order[len(order) * q // 4] for q in (1, 2, 3)] if len(order) > 1 else []
    for s in picks:
        est = per_cost * cost(0, s)
        if spent + est > budget_s or s in [x[1] for x in timed]:
            continue
        dt = run(0, s)
        timed.append((0, s))
        spent += dt
        ccost += cost(0, s)
    if len(scales) == 1 and nsl == 1:
        while spent < budget_s * 0.5:
            spent += run(0, 0)
            timed.append((0, 0))
            ccost += cost(0, 0)
    per_cost = spent / ccost
    full = sum(cost(t, s) for t in range(nsl) for s in range(len(scales))) * per_cost
    rate = g.nx * g.ny * nsl * len(scales) / full
    if len(scales) == 1 and nsl == 1:
        sample = f"{len(timed)} timed compute_Pi runs of the full {g.nx}x{g.ny} workload ({spent:.1f} s)"
    else:
        sample = (f"{len(timed)} timed (slice, scale) units, scales "
                  f"{sorted({round(scales[s] / 1e3) for _, s in timed})} km of slice 0 ({spent:.1f} s), "
                  f"extrapolated to all {nsl}x{len(scales)} units linearly in active targets x footprint entries")
    return rate, nthreads, len(timed), spent, sample, first


def device_steps_ms(run, steps, stream, flush) -> float:
    """Device time of `steps` steps: an L2 flush (a write larger than L2) before each step, and a pair of
    CUDA events on the launch stream around each step alone; returns the summed milliseconds."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        flush.fill_(1.0)
        ev[k][0].record(stream)
        run(k)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    return float(sum(a.elapsed_time(b) for a, b in ev))


def host_link(h2d_bytes: int, d2h_bytes: int, reps: int = 20) -> dict:
    """The host link's own copy rate for one step's transfers: pinned host -> device and device -> pinned
    host copies of the step's byte counts, each alone and both at once on two streams (the pipelined
    steady state), timed with CUDA events on the copying streams after warm-up; the fastest of five
    turns of each."""
    import torch
    hin = torch.empty(h2d_bytes, dtype=torch.uint8).pin_memory()
    din = torch.empty(h2d_bytes, dtype=torch.uint8, device="cuda")
    hout = torch.empty(d2h_bytes, dtype=torch.uint8).pin_memory()
    dout = torch.empty(d2h_bytes, dtype=torch.uint8, device="cuda")
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()

    def timed(do_in, do_out):
        for _ in range(5):
            with torch.cuda.stream(s_in):
                din.copy_(hin, non_blocking=True)
            with torch.cuda.stream(s_out):
                hout.copy_(dout, non_blocking=True)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s_in)
        s_out.wait_event(a)
        for _ in range(reps):
            if do_in:
                with torch.cuda.stream(s_in):
                    din.copy_(hin, non_blocking=True)
            if do_out:
                with torch.cuda.stream(s_out):
                    hout.copy_(dout, non_blocking=True)
        s_in.wait_stream(s_out)
        b.record(s_in)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    # the three measurements taken in turn five times, the fastest of each kept (the first copies
    # from freshly pinned pages, and a shared host's other traffic, are slower)
    t_in = t_out = t_both = float("inf")
    for _ in range(5):
        t_in = min(t_in, timed(True, False))
        t_out = min(t_out, timed(False, True))
        t_both = min(t_both, timed(True, True))
    return {"h2d_GBps": h2d_bytes / t_in / 1e6, "d2h_GBps": d2h_bytes / t_out / 1e6,
            "h2d_ms": t_in, "d2h_ms": t_out, "both_ms": t_both}


def mlp_flops_per_point() -> float:
    """Multiply-adds x 2 of the closure MLP per point, unpadded (5-64-64-64-3)."""
    return 2.0 * (5 * 64 + 64 * 64 + 64 * 64 + 64 * 3)


def run_closure(args, rank, world, local, dist, steps=None, with_cpu=True):
    """closure8: train the closure on exact pairs, then time closure vs plain Pi at 8 scales.  Returns the
    record (value, ms_per_step, roofline, e2e, cpu_baseline, clocks, the closure's accuracy terms)."""
    import ctypes as C

    import torch

    import cgef_b200 as cg
    from cgef_b200 import _lib
    from cgef_b200 import closure as CL
    from cgef_b200 import synthetic as S

    L = _lib.load()
    wl = make_workload("closure8", rank)
    g = wl["grid"]
    scales = wl["scales"]
    ns = len(scales)
    N = g.nx * g.ny
    plans = [cg.plan_filter(g, wl["kernel"], s) for s in scales]
    waves = [p.autotune(1) if not args.no_autotune else 4.0 for p in plans]
    apply_evaluation(plans, args.evaluation)
    stream = torch.cuda.current_stream()

    # training pairs from two snapshots, 10^7 points sampled (seed 3)
    t0 = time.perf_counter()
    m = torch.from_numpy(g.mask.reshape(-1)).cuda()
    xs, ts = [], []
    for seed in (300 + 2 * rank, 301 + 2 * rank):
        u, v = S.sphere_fields(g, seed=seed)
        du, dv = torch.from_numpy(u).cuda(), torch.from_numpy(v).cuda()
        for p in plans:
            f, t = CL.training_pairs(p, du, dv)
            xs.append(f[0][:, m].T.contiguous())
            ts.append(t[0][:, m].T.contiguous())
    X = torch.cat(xs)
    T = torch.cat(ts)
    del xs, ts
    gen = torch.Generator(device="cuda")
    gen.manual_seed(3)
    idx = torch.randperm(X.shape[0], device="cuda", generator=gen)[:10_000_000]
    X, T = X[idx].contiguous(), T[idx].contiguous()
    torch.cuda.synchronize()
    pairs_s = time.perf_counter() - t0
    c = CL.Closure(seed=3)
    batch = 8192
    nsteps = int(args.closure_epochs * X.shape[0] / batch)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    l1 = c.train(X, T, batch=batch, steps=nsteps * 2 // 3, lr=2e-3, weight_decay=1e-4)
    l2 = c.train(X, T, batch=batch, steps=nsteps - nsteps * 2 // 3, lr=4e-4, weight_decay=1e-4)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    losses = np.concatenate([l1, l2])
    del X, T

    du = torch.from_numpy(np.ascontiguousarray(wl["u"][0])).cuda()
    dv = torch.from_numpy(np.ascontiguousarray(wl["v"][0])).cuda()
    parr = (C.c_void_p * ns)(*[p.handle.value for p in plans])
    dPi = torch.empty((1, ns) + g.shape, dtype=torch.float64, device="cuda")
    dE = torch.empty((1, ns), dtype=torch.float64, device="cuda")
    cPi = torch.empty((ns,) + g.shape, dtype=torch.float64, device="cuda")
    reports = []

    def plain_step():
        _lib.check(L.cgef_sweep_device(parr, ns, _lib.F64, du.data_ptr(), dv.data_ptr(), 1, None, dPi.data_ptr(),
                                       dE.data_ptr(), stream.cuda_stream))

    def closure_step(k, frac=0.02, tol=args.closure_tol):
        reports.clear()
        for s, p in enumerate(plans):
            _, rep = c.pi(p, du, dv, judge_fraction=frac, judge_seed=1000 * k + s, tol=tol, out=cPi[s])
            reports.append(rep)

    # accuracy: raw closure (no judge) and the judged result against the exact flux
    plain_step()
    closure_step(0, frac=0.0, tol=float("inf"))
    torch.cuda.synchronize()
    exact = dPi[0].cpu().numpy()
    msk = g.mask
    raw_err = [float(np.linalg.norm((cPi[s].cpu().numpy() - exact[s])[msk]) / np.linalg.norm(exact[s][msk]))
               for s in range(ns)]
    # the classical nonlinear gradient model on the same snapshot, for comparison: for a Gaussian of
    # second moment l^2 / (2 alpha), tau_ij = l^2 / (2 alpha) A_ik A_jk with A the filtered velocity
    # gradient (curvature terms included); in the closure's normalised units y = x x^T / (2 alpha).
    # Also with its coefficient fitted by least squares to this snapshot's exact tau (an upper bound
    # on what the model can do).
    ngm_err, ngm_fit_err = [], []
    mflat = torch.from_numpy(msk.reshape(-1)).cuda()
    for s_, p in enumerate(plans):
        f, t = CL.training_pairs(p, du, dv)
        x, y = f[0].double(), t[0].double()
        yn = torch.stack([x[0] ** 2 + x[1] ** 2, x[0] * x[2] + x[1] * x[3], x[2] ** 2 + x[3] ** 2])
        # Pi from normalised quantities: S = (x0, (x1 + x2)/2, x3) n / l^2, tau = y n^2 / l^2, so
        # Pi is proportional to -(x0 y0 + (x1 + x2) y1 + x3 y2) with one positive factor per slice
        pi_of = lambda yy: -(x[0] * yy[0] + (x[1] + x[2]) * yy[1] + x[3] * yy[2])
        ex = pi_of(y)[mflat]
        ng = pi_of(yn)[mflat]
        c_th = 1.0 / (2.0 * wl["kernel"].alpha)
        c_fit = float((ng * ex).sum() / (ng * ng).sum())
        ngm_err.append(float(torch.linalg.norm(c_th * ng - ex) / torch.linalg.norm(ex)))
        ngm_fit_err.append(float(torch.linalg.norm(c_fit * ng - ex) / torch.linalg.norm(ex)))
    closure_step(0)
    torch.cuda.synchronize()
    judged_err = [float(np.linalg.norm((cPi[s].cpu().numpy() - exact[s])[msk]) / np.linalg.norm(exact[s][msk]))
                  for s in range(ns)]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed(fn, steps, profile=False):
        for k in range(max(args.warmup, 3)):
            flush.fill_(1.0)
            fn(k)
        torch.cuda.synchronize()
        if profile:
            L.cgef_reset_launch_count()
            L.cgef_profile_reset()
            L.cgef_profile_enable(1)
        return device_steps_ms(lambda k: fn(k + 100), steps, stream, flush)

    steps = steps or args.steps or 3
    sampler = ClockSampler(local, args.clocks_out)
    sampler.start()
    time.sleep(0.3)
    ms_open = timed(lambda k: closure_step(k, tol=float("inf")), steps)
    reports_open = list(reports)
    ms_closure = timed(closure_step, steps, profile=True)
    L.cgef_profile_enable(0)
    launches = int(L.cgef_launch_count())
    prof = {}
    for name, kind in (("banded", _lib.KERNEL_BANDED), ("closure_mlp", _lib.KERNEL_CLOSURE),
                       ("strain", _lib.KERNEL_STRAIN), ("stage", _lib.KERNEL_STAGE), ("rowspec", _lib.KERNEL_ROWSPEC)):
        tot, cnt = C.c_double(), C.c_int64()
        _lib.check(L.cgef_profile_read(kind, C.byref(tot), C.byref(cnt)))
        prof[name] = (tot.value, cnt.value)
    ms_plain = timed(lambda k: plain_step(), steps)
    clocks = sampler.stop()
    fallbacks = sum(r.fallbacks for r in reports)
    units = N * ns
    value = world * units * steps / (ms_closure / 1e3)
    plain_value = world * units * steps / (ms_plain / 1e3)

    # roofline of the dominant kernel (the 3-field FP64 velocity gather) and of the tensor-core MLP
    act = g.mask.sum(axis=1).astype(np.float64)
    vel_flops = sum(float((act * p.band_counts()).sum()) * 3 * 2 for p in plans)
    peak = fp64_peak(local)
    bt, bc = prof["banded"]
    rt, rc_ = prof["rowspec"]
    mt, mc = prof["closure_mlp"]
    mlp_ach = N * ns * mlp_flops_per_point() * steps / (mt * 1e-3) / 1e12 if mt > 0 else None
    bf16, bf16_source = bf16_peak()
    mlp_line = {"bound": "tensor", "achieved": mlp_ach, "peak": bf16, "unit": "TFLOP/s",
                "frac": (mlp_ach / bf16) if (mlp_ach and bf16) else None,
                "per_step_ms": mt / steps, "flops_per_point": mlp_flops_per_point(), "peak_source": bf16_source}
    if rt > bt:
        # the 3-field velocity filter runs through the row-spectral evaluation
        hbm, hbm_source = hbm_peak()
        vb = sum(rowspec_bytes(p, g, 1, 3, 3, 3, True) for p in plans if uses_row_spectral(p))
        ach = vb * steps / (rt * 1e-3) / 1e9
        roofline = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                    "traffic": None,
                    "kernel": "row-spectral filter of the 3 planetary velocity components (rs_forward, rs_accumulate, "
                              "rs_inverse, rs_finish); judged tiles add a direct 9-field gather over 2% of the tiles",
                    "per_step_ms": rt / steps, "algorithmic_bytes_per_step": vb, "direct_gather_ms_per_step": bt / steps,
                    "peak_source": hbm_source, "mlp": mlp_line}
    else:
        ach = vel_flops * steps / (bt * 1e-3) / 1e12 if bt > 0 else None
        roofline = {"bound": "fp64", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                    "frac": (ach / peak) if (ach and peak) else None, "traffic": None,
                    "kernel": "banded_kernel in fields mode (3 planetary velocity components, FP64 FMA); judged "
                              "tiles add a 9-field gather over 2% of the tiles",
                    "per_step_ms": bt / steps, "algorithmic_flops_per_step": vel_flops, "mlp": mlp_line}

    # end to end: pinned host u, v in, Pi of every scale out, each step
    hu = torch.from_numpy(np.ascontiguousarray(wl["u"][0])).pin_memory()
    hv = torch.from_numpy(np.ascontiguousarray(wl["v"][0])).pin_memory()
    hPi = torch.empty((ns,) + g.shape, dtype=torch.float64).pin_memory()

    def e2e_step(k):
        du.copy_(hu, non_blocking=True)
        dv.copy_(hv, non_blocking=True)
        closure_step(k)
        hPi.copy_(cPi, non_blocking=True)
        torch.cuda.synchronize()

    e2e_step(0)
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(steps):
        e2e_step(k + 1)
    el = time.perf_counter() - t0
    el = max_over_ranks(el, dist)
    e2e = {"value": world * units * steps / el, "unit": UNIT, "h2d_bytes_per_step": 2 * N * 8,
           "d2h_bytes_per_step": ns * N * 8, "steps": steps,
           "timing": "wall clock: pinned H2D of u, v, the closure at 8 scales, D2H of Pi"}
    cpu = None
    if rank == 0 and world == 1 and with_cpu and not args.no_cpu_baseline:
        rate, nth, done, el, sample, _ = oracle_rate(wl, budget_s=20.0)
        cpu = {"value": rate, "unit": UNIT, "cores": nth, "kind": "port",
               "sample": sample + f"; CPU {cpu_model()}; restated reference threaded path (plain Pi, FP64 oracle)"}
    return {"value": value, "unit": UNIT, "steps": steps, "ms_per_step": ms_closure / steps,
            "dtype": "f64 flux, bf16 closure (fp32 accumulate)", "config": workload_config(wl),
            "run": {"judge_fraction": 0.02, "tol": args.closure_tol, "schedule_split_waves": waves,
                    "parallelism": f"{world} rank(s), independent snapshots per rank"},
            "plain_value": plain_value, "plain_ms_per_step": ms_plain / steps,
            "speedup_vs_plain": value / plain_value, "fallback_slices_per_step": fallbacks,
            "no_fallback_value": world * units * steps / (ms_open / 1e3),
            "no_fallback_ms_per_step": ms_open / steps,
            "no_fallback_speedup_vs_plain": (world * units * steps / (ms_open / 1e3)) / plain_value,
            "no_fallback_est_rel_l2": [r.est_rel_l2 for r in reports_open],
            "pi_rel_l2_raw": raw_err, "pi_rel_l2_judged": judged_err,
            "gradient_model_pi_rel_l2": ngm_err, "gradient_model_fitted_pi_rel_l2": ngm_fit_err,
            "est_rel_l2_judge": [r.est_rel_l2 for r in reports], "scales_km": [s / 1e3 for s in scales],
            "training": {"points": 10_000_000, "batch": batch, "steps": int(nsteps), "seconds": train_s,
                         "pairs_seconds": pairs_s, "loss_first": float(losses[:10].mean()),
                         "loss_last": float(losses[-50:].mean())},
            "gpu_launches": launches, "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def fp64_peak(local: int):
    """The FP64 FMA peak measured in this run by libcgef_peak.so (a DFMA loop over all SMs)."""
    import ctypes as C
    try:
        pk = C.CDLL(os.path.join(ROOT, "coarsegrainingenergyfluxes.jl_b200", "cgef_b200", "libcgef_peak.so"))
        pk.cgef_peak_fp64_tflops.restype = C.c_double
        pk.cgef_peak_fp64_tflops.argtypes = [C.c_int]
        return float(pk.cgef_peak_fp64_tflops(local))
    except Exception:
        return None


def bf16_peak():
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"]), \
            "measured: MEASURED_PEAKS.json bf16_tflops (cuBLAS burst on this pool's B200s)"
    except Exception:
        return 1590.0, "fallback 1.59 PFLOP/s (earlier cuBLAS bf16 burst measurement on this pool)"


def max_over_ranks(x: float, dist) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


L2_NOTE = ("GPU arm: a 256 MiB write flushes L2 before every timed step, outside the step's own CUDA events; "
           "CPU arm (the oracle on the host cores): no flush")


def workload_config(wl) -> dict:
    """The workload, in the same words from both arms (the GPU's and --impl reference)."""
    g = wl["grid"]
    if wl["slice_masks"] is not None:
        act = float(np.mean(wl["slice_masks"]))
    else:
        act = float(1.0 if g.mask is None else np.mean(g.mask))
    return {"workload": wl["desc"], "nx": g.nx, "ny": g.ny, "scales": len(wl["scales"]),
            "snapshots": int(wl["u"].shape[0]), "active_fraction": act, "storage": wl["dtype"], "l2": L2_NOTE}


def compulsory_bytes(g, nsl: int, ns: int, bsz: int, slice_masks) -> float:
    """Bytes a step must move at least: u, v (and the masks) read once, Pi and E written once."""
    N = g.nx * g.ny
    masks = nsl * N if slice_masks is not None else (N if g.mask is not None else 0)
    return float(2 * nsl * N * bsz + masks + nsl * ns * N * bsz + nsl * ns * 8)


def measure_sweep(args, name, rank, world, local, dist, *, snapshots=1, scale_km=None, steps=None, e2e_steps=None,
                  with_cpu=True, cpu_budget=20.0):
    """Times one sweep workload (Pi and E(l) of every slice at every scale): the step replayed from its
    CUDA graph (the value), launched call by call (eager; its per-kernel events feed the roofline), and
    end to end through the host C ABI; plus the CPU baseline and the accuracy against the FP64 oracle
    (rank 0 of one rank).  Returns the record."""
    import ctypes as C

    import torch

    import cgef_b200 as cg
    from cgef_b200 import _lib

    L = _lib.load()
    wl = make_workload(name, rank, snapshots, scale_km)
    g = wl["grid"]
    nsl = int(wl["u"].shape[0])
    ns = len(wl["scales"])
    t0 = time.perf_counter()
    plans = [cg.plan_filter(g.with_mask(None) if wl["slice_masks"] is not None else g, wl["kernel"], s)
             for s in wl["scales"]]
    # schedule autotuning is plan setup, like building the footprint: outside the timed region
    waves = [p.autotune(nsl) if not args.no_autotune else 4.0 for p in plans]
    apply_evaluation(plans, args.evaluation)
    setup_s = time.perf_counter() - t0
    tdt = torch.float32 if wl["dtype"] == "f32" else torch.float64
    du = torch.from_numpy(np.ascontiguousarray(wl["u"])).to(device="cuda", dtype=tdt)
    dv = torch.from_numpy(np.ascontiguousarray(wl["v"])).to(device="cuda", dtype=tdt)
    dm = None if wl["slice_masks"] is None else torch.from_numpy(wl["slice_masks"].astype(np.uint8)).cuda()
    dt_code = _lib.F32 if tdt == torch.float32 else _lib.F64
    parr = (C.c_void_p * ns)(*[p.handle.value for p in plans])
    dPi = torch.empty((nsl, ns) + g.shape, dtype=tdt, device="cuda")
    dE = torch.empty((nsl, ns), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        _lib.check(L.cgef_sweep_device(parr, ns, dt_code, du.data_ptr(), dv.data_ptr(), nsl,
                                       None if dm is None else dm.data_ptr(), dPi.data_ptr(), dE.data_ptr(),
                                       stream.cuda_stream))

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    if steps is None:
        # about 5 s of timed work (every rank takes the slowest rank's count)
        step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(3):
            step()
        torch.cuda.synchronize()
        per = max_over_ranks((time.perf_counter() - t0) / 3, dist)
        steps = int(max(3, min(5000, 5.0 / max(per, 1e-6))))
    for _ in range(max(args.warmup, 3)):
        flush.fill_(1.0)
        step()
    torch.cuda.synchronize()

    sampler = ClockSampler(local, args.clocks_out)
    sampler.start()
    time.sleep(0.3)
    L.cgef_reset_launch_count()
    L.cgef_profile_reset()
    L.cgef_profile_enable(1)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    elapsed_ms = device_steps_ms(lambda k: step(), steps, stream, flush)
    if dist is not None:
        dist.barrier()
    L.cgef_profile_enable(0)
    launches = int(L.cgef_launch_count())

    # the same step replayed from a captured CUDA graph (cgef_sweep_graph_create / cgef_graph_launch)
    gs = torch.cuda.Stream()  # capture needs a created stream
    torch.cuda.synchronize()
    gh = C.c_void_p()
    _lib.check(L.cgef_sweep_graph_create(C.byref(gh), parr, ns, dt_code, du.data_ptr(), dv.data_ptr(), nsl,
                                         None if dm is None else dm.data_ptr(), dPi.data_ptr(), dE.data_ptr(),
                                         gs.cuda_stream))
    with torch.cuda.stream(gs):
        for _ in range(max(args.warmup, 3)):
            flush.fill_(1.0)
            _lib.check(L.cgef_graph_launch(gh, gs.cuda_stream))
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    L.cgef_reset_launch_count()
    with torch.cuda.stream(gs):
        graph_ms = device_steps_ms(lambda k: _lib.check(L.cgef_graph_launch(gh, gs.cuda_stream)), steps, gs, flush)
    graph_launches = int(L.cgef_launch_count())
    _lib.check(L.cgef_graph_destroy(gh))
    graph_ms = max_over_ranks(graph_ms, dist)
    clocks = sampler.stop()
    elapsed_ms = max_over_ranks(elapsed_ms, dist)
    units_per_step = g.nx * g.ny * ns * nsl
    # the value is the step replayed from the CUDA graph it was captured into once (the library's
    # API for repeated sweeps, cgef_sweep_graph_create / cgef_graph_launch); the same step launched call
    # by call, whose per-kernel events feed the roofline, is reported beside it as "eager"
    value = world * units_per_step * steps / (graph_ms / 1e3)
    eager_line = {"value": world * units_per_step * steps / (elapsed_ms / 1e3), "ms_per_step": elapsed_ms / steps,
                  "gpu_launches": launches,
                  "timing": "the same step launched call by call (cgef_sweep_device); same L2 flush, same events"}

    # dominant kernel timing (CUDA events on the launch stream, inside the timed region): the footprint
    # sums of the direct gather or of the row-spectral evaluation, whichever took longer
    kinds = {"banded": _lib.KERNEL_BANDED, "separable": _lib.KERNEL_SEPARABLE, "prefixsum": _lib.KERNEL_PREFIX}
    prof = {}
    for pname, kind in (("direct", kinds[plans[0].engine]), ("rowspec", _lib.KERNEL_ROWSPEC)):
        tot, cnt = C.c_double(), C.c_int64()
        _lib.check(L.cgef_profile_read(kind, C.byref(tot), C.byref(cnt)))
        prof[pname] = (tot.value, int(cnt.value))
    spec_plans = [p for p in plans if uses_row_spectral(p)]
    direct_plans = [p for p in plans if not uses_row_spectral(p)]
    flops_all = algorithmic_flops(plans, g, nsl, wl["slice_masks"])
    masked = g.mask is not None or wl["slice_masks"] is not None
    if plans[0].engine == "prefixsum":
        tot, cnt = prof["direct"]
        per_launch_ms = tot / max(cnt, 1)
        launches_per_step = max(cnt // steps, 1)
        na, npl = (9, 3) if g.is_spherical else (5, 2)
        if isinstance(plans[0].strategy, cg.Deformable):
            na, npl = na + 1, npl + 1
        bytes_launch = sum(prefix_bytes(p, g, nsl, na, npl, 5, masked) for p in plans) / launches_per_step
        peak, peak_source = hbm_peak()
        achieved = bytes_launch / (per_launch_ms * 1e-3) / 1e9
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": None, "traffic_basis": "no capture of this workload",
                    "kernel": "prefix_scan_kernel + prefix_sweep_kernel (exact top-hat: per-row prefix sums over the "
                              "tripled periodic row, then interval differences per target and row offset)",
                    "per_launch_ms": per_launch_ms, "launches": cnt, "algorithmic_bytes_per_launch": bytes_launch,
                    "peak_source": peak_source}
    elif prof["rowspec"][0] >= prof["direct"][0] and spec_plans:
        tot, cnt = prof["rowspec"]
        per_launch_ms = tot / max(cnt, 1)
        launches_per_step = max(cnt // steps, 1)
        na, npl = (9, 3) if g.is_spherical else (5, 2)
        if isinstance(plans[0].strategy, cg.Deformable):  # the mask is one more quantity and plane
            na, npl = na + 1, npl + 1
        bytes_step = sum(rowspec_bytes(p, g, nsl, na, npl, 0, masked, raw=True) for p in spec_plans)
        # a sweep transforms the source rows once for all row-spectral scales of one FFT length: the
        # other scales read those spectra but neither read the staged planes nor write spectra
        L0 = spec_plans[0].row_spectral[2]
        nshare = sum(1 for p in spec_plans if p.row_spectral[2] == L0)
        if nshare > 1:
            nk = L0 // 2 + 1
            bytes_step -= (nshare - 1) * (nsl * npl * g.nx * g.ny * 8 + nsl * g.ny * na * nk * 16)
        bytes_launch = bytes_step / launches_per_step
        peak, peak_source = hbm_peak()
        achieved = bytes_launch / (per_launch_ms * 1e-3) / 1e9
        traffic, traffic_basis, traffic_one = committed_traffic(f"{name}:rowspec", nsl, scale_km)
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": traffic, "traffic_basis": traffic_basis, "traffic_one_snapshot": traffic_one,
                    "kernel": "rs_forward_kernel + rs_accumulate_tma_kernel (rs_accumulate_kernel off the sphere) + "
                              "rs_inverse_kernel (row-spectral footprint sums: FFTs along x, banded spectral sums, "
                              "inverse FFTs; the epilogue runs in the strain pass)",
                    "per_launch_ms": per_launch_ms, "launches": cnt, "algorithmic_bytes_per_launch": bytes_launch,
                    "direct_sum_equivalent_tflops": flops_all / launches_per_step / (per_launch_ms * 1e-3) / 1e12
                    if not direct_plans else None,
                    "direct_gather_launches": prof["direct"][1], "peak_source": peak_source}
    else:
        tot, cnt = prof["direct"]
        per_launch_ms = tot / max(cnt, 1)
        flops_step = algorithmic_flops(direct_plans, g, nsl, wl["slice_masks"])
        launches_per_step = max(cnt // steps, 1)
        flops_launch = flops_step / launches_per_step
        peak = fp64_peak(local)
        achieved = flops_launch / (per_launch_ms * 1e-3) / 1e12
        traffic, traffic_basis, traffic_one = committed_traffic(f"{name}:{plans[0].engine}", nsl, scale_km)
        roofline = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": (achieved / peak) if peak and peak > 0 else None, "traffic": traffic,
                    "traffic_basis": traffic_basis, "traffic_one_snapshot": traffic_one,
                    "kernel": {"banded": "banded_kernel + banded_combine_kernel (FP64 FMA footprint gather)",
                               "separable": "sep_row_kernel + sep_col_kernel (FP64 separable passes)",
                               "prefixsum": "prefix_scan_kernel + prefix_sweep_kernel"}[plans[0].engine],
                    "per_launch_ms": per_launch_ms, "launches": cnt,
                    "algorithmic_flops_per_launch": flops_launch, "row_spectral_launches": prof["rowspec"][1],
                    "peak_source": "measured: DFMA loop over all SMs on this GPU (libcgef_peak.so), "
                                   "nominal B200 FP64 37 TFLOP/s; MEASURED_PEAKS.json holds no FP64 figure"}
    # second term: the step's compulsory bytes (inputs read once, outputs written once) over the whole
    # step, against HBM -- how far the step is from the problem's own I/O bound
    bsz = 4 if tdt == torch.float32 else 8
    comp = compulsory_bytes(g, nsl, ns, bsz, wl["slice_masks"])
    hbm, hbm_source = hbm_peak()
    comp_ach = comp / (graph_ms / steps * 1e-3) / 1e9
    roofline["compulsory"] = {"bound": "hbm", "bytes_per_step": comp, "achieved": comp_ach, "peak": hbm,
                              "unit": "GB/s", "frac": comp_ach / hbm, "peak_source": hbm_source,
                              "what": "u, v (and masks) read once, Pi and E written once, over the whole step "
                                      "(graph replay) -- the problem's own I/O"}

    # end to end through the host C ABI: pinned inputs in, Pi (and E) out, every step
    hu = torch.from_numpy(np.ascontiguousarray(wl["u"])).to(dtype=tdt).pin_memory()
    hv = torch.from_numpy(np.ascontiguousarray(wl["v"])).to(dtype=tdt).pin_memory()
    hPi = torch.empty((nsl, ns) + g.shape, dtype=tdt).pin_memory()
    hE = torch.empty((nsl, ns), dtype=torch.float64).pin_memory()
    hm = None if wl["slice_masks"] is None else torch.from_numpy(wl["slice_masks"].astype(np.uint8)).pin_memory()

    def host_step():
        _lib.check(L.cgef_sweep(parr, ns, dt_code, hu.data_ptr(), hv.data_ptr(), nsl,
                                None if hm is None else hm.data_ptr(), hPi.data_ptr(), hE.data_ptr()))

    host_step()
    per_step_s = elapsed_ms / 1e3 / steps
    n_e2e = e2e_steps if e2e_steps is not None else (
        args.e2e_steps if args.e2e_steps is not None else max(2, min(steps, 200, int(4.0 / per_step_s))))
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        host_step()
    el = max_over_ranks(time.perf_counter() - t0, dist)
    e2e_sync = {"value": world * units_per_step * n_e2e / el, "unit": UNIT,
                "h2d_bytes_per_step": int(2 * nsl * g.nx * g.ny * bsz + (0 if hm is None else hm.numel())),
                "d2h_bytes_per_step": int(nsl * ns * g.nx * g.ny * bsz + nsl * ns * 8), "steps": n_e2e,
                "timing": "wall clock around synchronous cgef_sweep calls (host buffers, pinned)"}

    # the same steps streamed through cgef_pipeline_*: every step still copies its u, v in and its Pi
    # and E out, but a step's copies overlap its neighbours' sweeps (double-buffered device memory)
    ph = C.c_void_p()
    _lib.check(L.cgef_pipeline_create(C.byref(ph), parr, ns, dt_code, nsl, None if hm is None else hm.data_ptr(), 1))
    outs = [(torch.empty_like(hPi).pin_memory(), torch.empty_like(hE).pin_memory()) for _ in range(2)]

    def submit(k):
        pi_k, e_k = outs[k % 2]
        _lib.check(L.cgef_pipeline_submit(ph, hu.data_ptr(), hv.data_ptr(), pi_k.data_ptr(), e_k.data_ptr()))

    submit(0)
    submit(1)
    _lib.check(L.cgef_pipeline_drain(ph))
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(n_e2e):
        submit(k)
    _lib.check(L.cgef_pipeline_drain(ph))
    el = time.perf_counter() - t0
    _lib.check(L.cgef_pipeline_destroy(ph))
    el = max_over_ranks(el, dist)
    e2e = {"value": world * units_per_step * n_e2e / el, "unit": UNIT,
           "h2d_bytes_per_step": int(2 * nsl * g.nx * g.ny * bsz),
           "d2h_bytes_per_step": int(nsl * ns * g.nx * g.ny * bsz + nsl * ns * 8), "steps": n_e2e,
           "timing": "wall clock from the first cgef_pipeline_submit to cgef_pipeline_drain: pinned u, v "
                     "copied in and Pi, E copied out for every step, overlapping the neighbouring steps' "
                     "sweeps (the per-level masks, if any, are copied once at create); no L2 flush: "
                     "each step's inputs arrive by H2D",
           "synchronous": e2e_sync}
    # what the host link allows: the pipelined steady state can be no faster than the slower of the
    # step's copies (both directions at once) and its device time
    link = host_link(e2e["h2d_bytes_per_step"], e2e["d2h_bytes_per_step"])
    bound_ms = max(link["both_ms"], graph_ms / steps)
    got_ms = el / n_e2e * 1e3
    e2e["link_bound"] = dict(link, bound_ms_per_step=bound_ms, achieved_ms_per_step=got_ms,
                             frac=bound_ms / got_ms,
                             what="one step's H2D and D2H bytes copied alone and both at once (pinned, CUDA "
                                  "events); bound = max(both at once, device ms per step); frac = bound / "
                                  "the streamed e2e's ms per step")

    cpu = None
    accuracy = None
    if rank == 0 and world == 1 and with_cpu and not args.no_cpu_baseline:
        rate, nth, done, el, sample, ref = oracle_rate(wl, budget_s=cpu_budget)
        cpu = {"value": rate, "unit": UNIT, "cores": nth, "kind": "port",
               "sample": sample + f"; CPU {cpu_model()}; restated reference threaded path (FP64 oracle, OpenMP rows)"}
        # the metric's accuracy term: the library's Pi (host C ABI, cgef_sweep) against the FP64 oracle on
        # the oracle's first timed unit; and the streamed output against the synchronous one
        got = hPi[ref["slice"], ref["scale"]].to(torch.float64).numpy()
        den = float(np.linalg.norm(ref["Pi"]))
        streamed = outs[(n_e2e - 1) % 2][0]
        accuracy = {"rel_l2_pi_vs_fp64_oracle": float(np.linalg.norm(got - ref["Pi"])) / (den if den > 0 else 1.0),
                    "unit": f"Pi of snapshot {ref['slice']} at l = {wl['scales'][ref['scale']] / 1e3:g} km, all cells",
                    "streamed_equals_synchronous": bool(torch.equal(streamed, hPi))}

    return {"value": value, "unit": UNIT, "steps": steps, "ms_per_step": graph_ms / steps,
            "dtype": "f64" if wl["dtype"] == "f64" else "f64 (f32 storage)", "config": workload_config(wl),
            "run": {"parallelism": f"{world} rank(s), independent snapshots per rank",
                    "schedule_split_waves": waves, "row_spectral": [uses_row_spectral(p) for p in plans],
                    "plan_setup_seconds": setup_s},
            "timing": "value: K steps replayed from a CUDA graph captured once, each bracketed by CUDA events on "
                      "the replay stream, a 256 MiB L2 flush between steps outside the events, max over ranks",
            "gpu_launches": graph_launches, "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks,
            "eager": eager_line, "accuracy": accuracy}


def headline(args, world, rec) -> dict:
    line = {"metric": METRIC, "value": rec["value"], "unit": UNIT, "n_gpus": world, "steps": rec["steps"],
            "warmup": args.warmup, "ms_per_step": rec["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": rec["dtype"], "data": "synthetic (seeded)", "config": rec["config"]}
    line.update({k: v for k, v in rec.items() if k not in line and k not in ("unit",)})
    return line


# ---------------------------------------------------------------------------------------------
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        wl = make_workload(args.workload, 0, args.snapshots, args.scale_km)
        rate, nth, done, el, sample, _ = oracle_rate(wl, budget_s=120.0)
        line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / max(done, 1),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded)", "config": workload_config(wl),
                "cpu_baseline": {"value": rate, "unit": UNIT, "cores": nth, "kind": "port",
                                 "sample": sample + f"; CPU {cpu_model()}; restated reference threaded path"},
                "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.workload == "closure8":
        line = headline(args, world, run_closure(args, rank, world, local, dist))
    else:
        line = headline(args, world, measure_sweep(args, args.workload, rank, world, local, dist,
                                                   snapshots=args.snapshots, scale_km=args.scale_km,
                                                   steps=args.steps))
        # the metric compares the plain path with the batched sweep and the closure: the default run
        # measures both beside the headline (one rank; a scaling run times the headline only)
        if (args.workload == "sphere1" and args.snapshots == 1 and args.scale_km is None and world == 1
                and not args.no_subrecords):
            b = measure_sweep(args, "sweep24x8", rank, world, local, dist, steps=args.batched_steps, e2e_steps=2,
                              cpu_budget=15.0)
            b["speedup_vs_plain"] = b["value"] / line["value"]
            line["batched"] = b
            line["closure"] = run_closure(args, rank, world, local, dist, steps=3)
            # the package's default kernel (Pipeline.jl:344) on the same grid: the exact top-hat
            line["tophat"] = measure_sweep(args, "tophat", rank, world, local, dist, steps=50, e2e_steps=20,
                                           cpu_budget=15.0)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
