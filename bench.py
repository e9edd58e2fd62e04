"""Benchmark: N-1 solves/s on the 9,241-bus synthetic grid with 500 branch outages, max mismatch 1e-8 pu.

One step = one batch of 500 single-branch outages solved to convergence by the batched Newton-Raphson engine, every
scenario warm-started from the base case.  Prints ONE JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference] [--precision mixed|fp64]

``--impl reference`` times the reference path's CPU arm instead: the C restatement of the reference's Newton-Raphson
(the oracle) on every host core, on a bounded sample of the same outages (the reference's own CPU path, OLF with
KLU in a JVM, does not run here: no JVM, no OLF jars, no network).
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "olf-gpu_b200"))

METRIC = "N-1 solves/s (9k-bus, 500 outages) learned+mixed vs plain FP64 NR at 1e-8 pu"
GRID = "grid9241"
N_OUTAGES = 500
TOL = 1e-8
CHECKPOINT = os.path.join(ROOT, "olf-gpu_b200", "checkpoints", "warmstart_grid9241.npz")
# DRAM bytes (read + write) of one lane's factorization (narrow levels in shared memory), from ncu captures of the
# launches of the first factorization of a 64-outage batch: the dense-front plan on plain minimum degree (89 launches;
# FP64 490.9 MB, FP32 LU 288.3 MB over 64 lanes) and on the shallow-tree order (123 launches; 573.2 MB, 328.6 MB);
# scaled to a launch by the lanes it factorizes
TRAFFIC = {("dense", "fp64"): 7.67e6, ("dense", "mixed"): 4.51e6,
           ("shallow", "fp64"): 8.96e6, ("shallow", "mixed"): 5.13e6}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms during the timed region: ONE looping nvidia-smi
    process (``-lms 100``), started before the region and past its first sample when the region begins, so no process
    start or NVML initialisation falls inside the timed steps."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self._proc = None
        self._t = None
        self._first = threading.Event()

    def _read(self):
        for line in self._proc.stdout:
            vals = [v.strip() for v in line.strip().split(",")]
            if len(vals) == 6:
                self.samples.append(vals)
                self._first.set()

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                           "--format=csv,noheader,nounits", "-lms", "100"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self._proc = None
            return self
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        self._first.wait(10)                    # the first sample is in: the process is up
        self.samples.clear()                    # only samples taken during the region count
        return self

    def __exit__(self, *a):
        if self._proc is not None:
            deadline = time.time() + 0.5          # a region shorter than the period still gets its sample
            while not self.samples and time.time() < deadline:
                time.sleep(0.01)
            self._proc.terminate()
            try:
                self._proc.wait(timeout=10)
            except subprocess.TimeoutExpired:
                self._proc.kill()
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[2 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def plan_flags(plan: str) -> int:
    """Structure ordering flags of a --plan choice: scaled (minimum degree), deferred (deferred-L), dense (minimum
    degree + dense front), shallow (minimum degree relaxed toward a shallow elimination tree + dense front)."""
    from olfgpu import native
    return {"deferred": native.PLAN_DEFERRED_L, "dense": native.PLAN_DENSE_FRONT,
            "shallow": native.PLAN_DENSE_FRONT | native.MIN_DEGREE_SHALLOW}.get(plan, 0)


def dense_front(plan: str) -> bool:
    return plan in ("dense", "shallow")


def workload(rank: int, count: int = N_OUTAGES):
    from olfgpu import packing, synthetic
    g = synthetic.build(GRID)
    p = packing.pack(g)
    # weak scaling: every rank solves its own 500 outages of the same grid
    outs = synthetic.draw_outages(g, count, seed=9241 + rank)
    return g, p, outs


# The engine's launch structure (engine.cu / kernels.cu), used to count the kernels a step launches: narrow levels
# hold <= 48 tasks; the shared-memory factorization region holds <= 110 KB of FP64 blocks (3,520 slots) in levels of
# <= 256 tasks; a shared-memory solve region holds <= 2,048 rows.
NARROW, REGION_SLOTS, REGION_THREADS, SOLVE_REGION_SLOTS = 48, 110 * 1024 // 32, 256, 2048
# kernels of one learned-start prediction: input GEMM, 4 x (edge projection, PQ GEMM, message, update GEMM), output
# GEMM, compact inputs, start composition and scatter
GNN_LAUNCHES = 1 + 4 * 4 + 1 + 1 + 2


def launches_per_solve(s, sched, rounds: int, dense: bool, deferred: bool, mixed: bool, refine_rounds: int) -> int:
    """Kernels one batch solve launches: per factorizing round the factorization (level launches, the range or the
    shared-memory region, the dense front), the solves, step and advance; per round the start, fill, test and lane
    count; per solve the install and result gathers (6).  Matches the ncu launch lists: 802 per FP64 solve of the
    9,241-bus / 500-outage batch under schedule 4, 782 under the level schedule with 2-lane tiles (scaled plan)."""
    schedule, lanes = int(sched[0]), int(sched[1])
    f, _, fw, bw = s.levels()
    wf, wfw, wbw = np.diff(f), np.diff(fw), np.diff(bw)
    nl, nf, nb = len(wf), len(wfw), len(wbw)
    factor_to = nl - 1 if dense else nl
    factor_from = factor_to
    while factor_from > 0 and wf[factor_from - 1] <= NARROW:
        factor_from -= 1
    # the shared-memory region: the narrow levels from the top of the tree down while a level holds <=
    # REGION_THREADS tasks and the blocks fit REGION_SLOTS
    region_from = factor_to
    if not deferred:
        while (region_from > factor_from and wf[region_from - 1] <= REGION_THREADS
               and f[factor_to] - f[region_from - 1] <= REGION_SLOTS):
            region_from -= 1
    fwd_from = nf
    while fwd_from > 0 and wfw[fwd_from - 1] <= NARROW:
        fwd_from -= 1
    bwd_until = 0
    while bwd_until < nb and wbw[bwd_until] <= NARROW:
        bwd_until += 1
    fwd_region = 0 < fw[nf] - fw[fwd_from] <= SOLVE_REGION_SLOTS
    bwd_region = 0 < bw[bwd_until] <= SOLVE_REGION_SLOTS
    front = 1 if dense else 0
    if schedule == 1:                       # the whole Newton loop in one persistent launch
        return 1 + 6
    if schedule == 2:                       # cooperative sweeps: one launch per factorization and per sweep
        factor, solve = 1 + 1 + front, 2 + front + 2
    else:
        if schedule in (3, 4) and f[factor_to] - f[region_from] > 0:
            factor = region_from + 2 + (nl - factor_to)
        elif lanes > 0:
            factor = factor_from + 1 + (nl - factor_to)
        else:
            factor = nl
        factor += 1 + front                 # lane trouble flags, dense front
        solve = 2 + front                   # right-hand side, scatter, dense front rows
        if schedule == 4 and fwd_region:
            solve += fwd_from + 2
        elif schedule == 4 or lanes <= 0:
            solve += nf
        else:
            solve += fwd_from + 1
        if schedule == 4 and bwd_region:
            solve += 1 + (nb - bwd_until)
        elif schedule == 4 or lanes <= 0:
            solve += nb
        else:
            solve += 1 + (nb - bwd_until)
    per_round = factor + solve + 2 + (1 if mixed else 0)   # step, advance, (mixed) FP64-refactor lane count
    return int(rounds * per_round + (rounds + 1) * 4 + 6 + refine_rounds * 3)


def algorithmic_bytes(s, p, iterations_total: int, precision_bytes: int, refinement: int):
    """Bytes one scenario-iteration must move (J once, LU written and read once, six n-vectors), summed."""
    nnz_lu = s.n_lu_blocks * 4
    b_it = 8 * s.nnz + precision_bytes * 2 * nnz_lu + 8 * 6 * p.n
    b_it += refinement * (precision_bytes * nnz_lu + 8 * s.nnz)
    return b_it * iterations_total, b_it


def run_engine(args, rank: int, world: int):
    import torch
    from olfgpu import native
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    g, p, outs = workload(rank, args.outages)
    precision = native.MIXED if args.precision == "mixed" else native.FP64
    refinement = args.refinement if precision == native.MIXED else 0
    s = native.Structure(p, plan_flags(args.plan))
    ns = outs.shape[0]
    ctx = native.BatchContext(s, ns)
    ctx.set_linear_solver_settings(precision, max(refinement, 0))
    policy = native.MIXED_FP64_NEAR if args.mixed_policy == "fp64near" else native.MIXED_REFINE
    ctx.set_mixed_precision_policy(policy)
    ctx.set_device_loop(args.device_loop)
    if args.schedule == "auto":
        ctx.set_schedule(native.AUTOTUNE)           # the first (warm-up) solve times the candidates
    elif args.schedule == "coop":
        ctx.set_schedule(native.COOPERATIVE, 0, 512)
    elif args.schedule == "shared":
        ctx.set_schedule(native.LEVELS_SHARED, 2, 256)
    elif args.schedule == "shared-all":
        ctx.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
    # host inputs in pinned memory (e2e copies them every step); results read back to pinned memory
    dis = torch.from_numpy(p.outage_masks(outs)).pin_memory().numpy()
    out = torch.empty((ns, p.n + 3), dtype=torch.float64).pin_memory().numpy()
    x0 = torch.from_numpy(p.x_base.copy()).pin_memory().numpy()
    tgt = torch.from_numpy(p.target.copy()).pin_memory().numpy()
    mode = torch.from_numpy(p.base_row_mode.astype(np.int32)).pin_memory().numpy()

    learned = None
    if args.start == "learned":
        from olfgpu.learned_start import LearnedStart
        learned = LearnedStart.load(args.checkpoint, g)
        x0_dev = torch.empty((ns, p.n), dtype=torch.float64, device="cuda")
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctx.set_fallback_start(True)           # per lane: the better start by initial mismatch, restart on failure
        ctx.set_device_start(x0_dev)

    # concurrent parts: the batch split into lane ranges solved as concurrent device loops in one graph launch
    cb = None
    part_schedule = None
    part_tuning = []
    if args.parts > 1:
        from olfgpu.security_analysis import ConcurrentBatch
        if learned is not None:
            learned.predict_device(p, x0, outs, out=x0_dev)
        ctx.solve(x0, tgt, mode, dis, max_iter=15, tol=TOL, out=out)      # the single context's autotune
        part_schedule = tuple(ctx.schedule()[0])
        if part_schedule[0] in (native.PERSISTENT, native.COOPERATIVE):
            part_schedule = (native.LEVELS_SHARED_ALL, 0, 256)
        cb = ConcurrentBatch(s, ns, args.parts, precision, max(refinement, 0), policy, part_schedule)
        if learned is not None:
            cb.set_device_start(x0_dev)
        if args.schedule == "auto":
            # the parts interleave their level kernels: the single batch's pick and the shared-memory level
            # schedules are timed again as concurrent parts
            part_tuning = cb.autotune(x0, tgt, mode, dis, [part_schedule, (native.LEVELS_SHARED_ALL, 0, 256),
                                                           (native.SUBTREES, 0, 256)], max_iter=15, tol=TOL, out=out)
            part_schedule = cb.schedule

    def solve_once(c_single, c_parts, xs):
        """One solve of the batch: device ms and per-scenario total iterations."""
        if c_parts is not None:
            _, ms = c_parts.solve(xs, tgt, mode, dis, max_iter=15, tol=TOL, out=out)
            return ms, np.concatenate([c.last_stats()[2] for c in c_parts.contexts])
        c_single.solve(xs, tgt, mode, dis, max_iter=15, tol=TOL, out=out)
        ms, _, tot = c_single.last_stats()
        return ms, tot

    last = {}

    def step():
        """One batch: the learned-start prediction (on the device), then the solve; returns the prediction's device
        milliseconds (0 with the base start)."""
        pred_ms = 0.0
        if learned is not None:
            ev0.record()
            learned.predict_device(p, x0, outs, out=x0_dev)
            ev1.record()
            ev1.synchronize()
            pred_ms = ev0.elapsed_time(ev1)
        last["ms"], last["tot"] = solve_once(ctx, cb, x0)
        return pred_ms

    for _ in range(args.warmup):
        step()
    statuses = out[:, p.n + 2].astype(int).copy()
    iters_last = out[:, p.n].astype(int).copy()
    # device-resident timing: the library's CUDA events around the device work of each step (no host copies); with
    # the learned start, the device span of the whole pipelined loop
    dev_ms, wall_ms, tot_iters = [], [], 0
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", 0)))
    pred_total = 0.0
    gc.collect()
    gc.disable()                                # no collector pause inside the timed steps
    with sampler:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            t0 = time.perf_counter()
            pred_ms = step()
            wall_ms.append((time.perf_counter() - t0) * 1e3)
            ms, tot = last["ms"], last["tot"]
            dev_ms.append(ms + pred_ms)
            pred_total += pred_ms
            tot_iters += int(tot.sum())
    gc.enable()
    solver = cb if cb is not None else ctx
    fallbacks = int(solver.last_fallbacks().size) if learned is not None else 0
    fp64_iterations = solver.last_fp64_iterations()
    torch.cuda.synchronize()
    result = out.copy()                         # the last timed solve's states, iterations and statuses
    dev = float(np.mean(dev_ms))
    e2e = float(np.mean(wall_ms))
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([dev, e2e], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev, e2e = float(t[0]), float(t[1])

    def histogram(r):
        it = r[:, p.n].astype(int)
        return {str(int(k)): int(v) for k, v in zip(*np.unique(it, return_counts=True))}

    def comparison(prec, refine, pol=native.MIXED_REFINE, start=None):
        """The engine from the base start (or ``start`` [n], e.g. the flat start) on the same batch at a given
        precision and policy: device time per step, iteration histogram, and each scenario's difference from the
        measured configuration's result (scenarios both converged)."""
        xs = x0 if start is None else start
        if cb is not None:
            from olfgpu.security_analysis import ConcurrentBatch
            c = ConcurrentBatch(s, ns, args.parts, prec, refine, pol, part_schedule)
        else:
            c = native.BatchContext(s, ns)
            c.set_linear_solver_settings(prec, refine)
            c.set_mixed_precision_policy(pol)
            c.set_device_loop(args.device_loop)
            if args.schedule == "auto":
                c.set_schedule(native.AUTOTUNE)
            else:
                c.set_schedule(*ctx.schedule()[0])
        for _ in range(args.warmup):
            solve_once(c, c if cb is not None else None, xs)
        pm = []
        for _ in range(args.steps):
            pm.append(solve_once(c, c if cb is not None else None, xs)[0])
        f64 = c.last_fp64_iterations()
        c.close()
        both = (result[:, p.n + 2] == 0) & (out[:, p.n + 2] == 0)
        d = np.abs(result[both, :p.n] - out[both, :p.n])
        return {"solves_per_s": round(ns / (float(np.mean(pm)) * 1e-3), 1), "ms_per_step": round(float(np.mean(pm)), 4),
                "iterations_per_solve": round(float(out[:, p.n].mean()), 3), "iteration_histogram": histogram(out),
                "converged_fraction": round(float((out[:, p.n + 2] == 0).mean()), 4),
                "fp64_iterations": int(f64) if prec == native.MIXED else None,
                "vs_measured": {
                    "max_abs_dVa_rad": float(d[:, 0::2].max()) if both.any() else None,
                    "max_abs_dVm_pu": float(d[:, 1::2].max()) if both.any() else None,
                    "same_status": int((result[:, p.n + 2] == out[:, p.n + 2]).sum()),
                    "extra_iterations_per_solve": round(float(result[:, p.n].mean() - out[:, p.n].mean()), 4)}}

    # the plain FP64 engine from the base start on the same batch (the comparison the metric names) and, with the
    # learned start, the mixed-precision engine from the base start (what the start alone changes)
    plain = mixed_base = flat = refine_policy = None
    if not args.no_plain:
        plain = comparison(native.FP64, 0)
        if learned is not None and precision == native.MIXED:
            mixed_base = comparison(native.MIXED, refinement, policy)
        # the flat start (V = 1 or the set point, angles 0) at the measured precision and policy
        flat = comparison(precision, refinement, policy, start=np.ascontiguousarray(p.x_flat))
        if precision == native.MIXED and policy != native.MIXED_REFINE:
            refine_policy = comparison(native.MIXED, max(refinement, 3), native.MIXED_REFINE)
    # roofline of the Newton iterations (HBM-bound): algorithmic bytes over the device time
    peak, peak_kind = _peaks()
    # FP32 factors only in the iterations that ran in FP32 (the FP64-near policy runs the near ones in FP64)
    all_fp64 = precision != native.MIXED or (args.mixed_policy == "fp64near" and fp64_iterations > 0 and
                                             fp64_iterations >= int(np.max(result[:, p.n])))
    pbytes = 8 if all_fp64 else 4
    refine_bytes = refinement if args.mixed_policy == "refine" else 0
    total_bytes, b_it = algorithmic_bytes(s, p, tot_iters // args.steps, pbytes, refine_bytes)
    achieved = total_bytes / (dev * 1e-3) / 1e9
    # the dominant kernel family, the block-LU factorization (factorLevelKernel + factorRangeKernel launches of one
    # Newton iteration): one more solve of the same batch, after the timed region, with each phase bracketed by CUDA
    # events on the context's stream; algorithmic bytes of one lane's factorization = read J once (8 nnzJ) + write and
    # read the LU once (2 w nnzLU)
    ctx.set_phase_timing(True)
    if learned is not None:
        learned.predict_device(p, x0, outs, out=x0_dev)
    ctx.solve(x0, tgt, mode, dis, max_iter=15, tol=TOL, out=out)
    ph = ctx.last_phase_times()
    ctx.set_phase_timing(False)
    ph_fp64 = ctx.last_fp64_iterations()
    fact_w = 8 if (precision != native.MIXED or (args.mixed_policy == "fp64near" and ph_fp64 >= ph["iterations"])) \
        else 4
    fact_bytes_lane = 8 * s.nnz + 2 * fact_w * s.n_lu_blocks * 4
    fact_launch_ms = ph["factor"] / max(ph["iterations"], 1)
    fact_bytes_launch = fact_bytes_lane * ph["factorized_lanes"] / max(ph["iterations"], 1)
    fact_achieved = fact_bytes_launch / (fact_launch_ms * 1e-3) / 1e9 if fact_launch_ms > 0 else 0.0
    traffic = TRAFFIC.get((args.plan, "fp64" if fact_w == 8 else "mixed"))
    if traffic is not None:
        traffic = int(traffic * ph["factorized_lanes"] / max(ph["iterations"], 1))
    sched = ctx.schedule()[0]
    fact_kernel = "block-LU factorization of one Newton iteration (factorLevelKernel levels"
    if sched[0] in (native.LEVELS_SHARED, native.LEVELS_SHARED_ALL):
        fact_kernel += " + regionPrefixKernel / regionFactorKernel narrow levels in shared memory"
    elif sched[0] == native.LEVELS and sched[1] > 0:
        fact_kernel += " + factorRangeKernel narrow levels"
    elif sched[0] == native.COOPERATIVE:
        fact_kernel = "block-LU factorization of one Newton iteration (factorCoopKernel"
    fact_kernel += (" + denseFrontKernel)" if dense_front(args.plan) else ")")
    if ph["iterations"] == 0:
        # the autotuner picked the persistent schedule: one launch runs the whole Newton loop of the batch
        fact_kernel = "newtonPersistentKernel (the whole Newton loop of the batch in one launch)"
        fact_achieved, fact_launch_ms, fact_bytes_launch, traffic = achieved, dev, total_bytes, None
    words = (ns + 31) // 32
    h2d = p.n * 8 * 2 + p.n * 4 + p.n_elements * words * 4
    if learned is not None:   # outage indices and the compact rows (bus, scenario) of the outages' reach; the node
        # features, flows and outage-free pass depend only on the base state and stay on the device between steps
        h2d += ns * 4 + 2 * 4 * learned.reach(outs)[0].shape[0]
    d2h = ns * (p.n + 3) * 8
    conv = float((statuses == 0).mean())
    line = {
        "metric": METRIC,
        "value": round(world * ns / (dev * 1e-3), 1),
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(dev, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if all_fp64 else "fp32-lu+fp64",
        "data": "synthetic (seeded 9,241-bus grid, random non-bridge branch outages)",
        "config": {"workload": f"{GRID}: 9,241 buses, {p.n_cb} branches, {ns} outages per GPU, "
                               + ("learned warm start (GNN prediction on the device inside the step; per-lane "
                                  "choice against the base start by initial mismatch; fallback to the base start)"
                                  if learned is not None else
                                  "warm start from the base case")
                               + f", tol {TOL} pu, "
                               + (f"FP32 LU + {refinement} FP64 refinement step(s)" if precision == native.MIXED
                                  else "FP64 LU"),
                   "precision": args.precision, "l2": "working set > 1 GB per step, larger than the 126 MB L2",
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
        "e2e": {"value": round(world * ns / (e2e * 1e-3), 1), "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "achieved": round(fact_achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(fact_achieved / peak, 4), "traffic": traffic,
                     "kernel": fact_kernel,
                     "algorithmic_bytes_per_launch": int(fact_bytes_launch), "launch_ms": round(fact_launch_ms, 4),
                     "unit_bytes": "8 nnzJ + 2 w nnzLU per factorized lane",
                     "peak_source": f"{peak_kind} copy bandwidth (hbm_gbs)"},
        "roofline_iteration": {"achieved": round(achieved, 1), "frac": round(achieved / peak, 4),
                               "scope": "whole Newton iterations: (8 nnzJ + 2 w nnzLU + 48 n) bytes per "
                                        "scenario-iteration over the step's device time"},
        "phase_ms": {k: round(v, 3) for k, v in ph.items() if isinstance(v, float)},
        "gpu_launches": None,
        "start": args.start,
        "lu_plan": args.plan,
        "schedule": dict(zip(["schedule", "lanes_per_tile", "threads"], ctx.schedule()[0])),
        "autotune_ms": [[int(a), int(b_), int(c_), round(float(ms), 3)] for a, b_, c_, ms in ctx.schedule()[1]],
        "plain_fp64_base_start": plain,
        "mixed_base_start": mixed_base,
        "starts": None if plain is None else {
            "referee": "the engine's own Newton loop at 1e-8 pu decides every start's convergence",
            "learned" if learned is not None else "base (measured)": {
                "ms_per_step": round(dev, 4), "iterations_per_solve": round(float(result[:, p.n].mean()), 3),
                "iteration_histogram": histogram(result), "converged_fraction": round(conv, 4),
                "scenarios_on_base_start": fallbacks if learned is not None else None},
            "base": mixed_base if mixed_base is not None else plain,
            "flat": flat},
        "mixed_precision": None if precision != native.MIXED else {
            "policy": args.mixed_policy, "refine_below": 1e-2,
            "fp64_iterations_last_step": int(fp64_iterations),
            "refine_policy_base_start": refine_policy,
            "note": "fp64near: an iteration in which some scenario's max |F| is below 1e-2 factorizes and solves in "
                    "FP64 (all its scenarios), the others in FP32 without refinement; refine: FP32 LU every "
                    "iteration, FP64 refinement of the scenarios below 1e-2 to a 1e-11 correction"},
        "device_loop": bool(args.device_loop),
        "concurrent_parts": None if cb is None else {
            "parts": len(cb.ranges), "lanes": [b - a for a, b in cb.ranges], "part_schedule": list(part_schedule),
            "part_autotune_ms": [[list(c), round(ms, 3)] for c, ms in part_tuning],
            "note": "the batch split into lane ranges, each its own context on the shared structure, solved as "
                    "concurrent device-resident Newton loops in one graph launch (results identical to one batch)"},
        "learned_start": None if learned is None else {
            "checkpoint": os.path.relpath(args.checkpoint, ROOT), "prediction_ms_per_step": round(pred_total / args.steps, 4),
            "scenarios_on_base_start": fallbacks},
        "iterations_per_solve": round(tot_iters / args.steps / ns, 3),
        "converged_fraction": round(conv, 4),
        "step_ms": {"device": [round(v, 3) for v in dev_ms], "wall": [round(v, 3) for v in wall_ms]},
        "structure": {"n": s.n, "nnzJ": s.nnz, "nnzLU": s.n_lu_blocks * 4, "factor_levels": s.factor_levels,
                      "solve_levels": s.forward_levels + s.backward_levels, "block_ops": s.block_ops},
        "clocks": sampler.summary(),
    }
    rounds = max(ph["iterations"], 1)
    per_solve = launches_per_solve(s, sched, rounds, dense_front(args.plan), args.plan == "deferred",
                                   precision == native.MIXED and fp64_iterations < rounds,
                                   (rounds - 1) if refinement > 0 and args.mixed_policy == "refine" else 0)
    if args.device_loop:
        per_solve += 2 + rounds * (2 if precision == native.MIXED else 1)   # loop reset, cap; a condition per round
    if learned is not None:
        per_solve += GNN_LAUNCHES + 6          # the prediction, the two-start selection (2 fills and 4 small kernels)
    line["gpu_launches"] = int(per_solve * args.steps)
    line["gpu_launches_basis"] = (f"{per_solve} per step: the level structure under the schedule in force over "
                                  f"{rounds} factorizing Newton rounds (the same count as the ncu launch lists)")
    if not args.no_uneven:
        line["uneven_batch"] = uneven_summary(args)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(p, outs, args.cpu_sample)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def uneven_summary(args):
    """The uneven-batching workload (four grids, reactive limits on), measured inside the default line: one graph
    whose branches are the grids' device-resident Newton loops (the --plan's dense-front plans, shared-memory level
    schedule), the same grids solved back to back one batch each, and the single persistent launch (tiles of 2
    lanes, which run the scaled plan)."""
    from olfgpu import native, packing, synthetic
    from olfgpu.security_analysis import MultiGridAnalysis
    grids = [synthetic.build(nm) for nm, _ in UNEVEN]
    packs = [packing.pack(g) for g in grids]
    counts = [c for _, c in UNEVEN]
    outs = [synthetic.draw_outages(g, c, seed=7000 + i, replace=True) for i, (g, c) in enumerate(zip(grids, counts))]
    total = sum(counts)
    steps = max(3, min(args.steps, 5))

    def timed(fn):
        for _ in range(2):
            fn()
        return float(np.median([fn() for _ in range(steps)]))

    res = {}
    front = plan_flags(args.plan) if dense_front(args.plan) else native.PLAN_DENSE_FRONT
    ma = MultiGridAnalysis(packs, counts, schedule=(0, 0, 0), ordering=front,
                           member_schedule=(native.LEVELS_SHARED_ALL, 0, 256))
    res["one_graph_device_loops"] = timed(lambda: ma.solve(outs)[1])
    loop_res, _ = ma.solve(outs)
    ma.close()
    seq = []
    for p, o in zip(packs, outs):
        st = native.Structure(p, front)
        c = native.BatchContext(st, o.shape[0], native.BATCHED_LU, p.rl)
        c.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
        c.set_device_loop(True)
        seq.append((st, c, p, p.outage_masks(o)))

    def seq_step():
        ms = 0.0
        for st, c, p, dis in seq:
            c.solve(p.x_base, p.target, p.base_row_mode, dis, max_iter=15, tol=TOL)
            ms += c.last_stats()[0]
        return ms
    res["per_grid_batches_back_to_back"] = timed(seq_step)
    same = True
    for (st, c, p, dis), r in zip(seq, loop_res):
        solo = c.solve(p.x_base, p.target, p.base_row_mode, dis, max_iter=15, tol=TOL)
        same = same and np.array_equal(solo[:, :p.n], r.x) and np.array_equal(solo[:, p.n + 2].astype(int), r.status)
        c.close()
        st.close()
    ma = MultiGridAnalysis(packs, counts, schedule=(2, 256, 1))
    res["persistent_tiles"] = timed(lambda: ma.solve(outs)[1])
    ma.close()
    return {"workload": "grid300 x1000 + grid2000q x1000 + grid9241q x500 + grid13659 x250 outages, reactive "
                        "limits on, FP64, tol 1e-8 pu",
            **{k: {"ms": round(v, 3), "solves_per_s": round(total / (v * 1e-3), 1)} for k, v in res.items()},
            "one_graph_equals_solo_solves": bool(same)}


def cpu_baseline(p, outs, sample: int):
    """The oracle (C restatement of the reference Newton-Raphson, sparse LU) on every host core, bounded sample."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    st = O.Structure(p)
    sub = outs[:sample]
    t0 = time.perf_counter()
    r = st.solve_batch(p.x_base, p.outage_masks(sub), max_iter=15, tol=TOL, threads=cores)
    dt = time.perf_counter() - t0
    return {"value": round(sub.shape[0] / dt, 2), "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": f"{sub.shape[0]} of the {outs.shape[0]} outages, {dt:.1f} s on {cores} threads",
            "converged": int((r[:, -1] == 0).sum())}


UNEVEN = [("grid300", 1000), ("grid2000q", 1000), ("grid9241q", 500), ("grid13659", 250)]


def run_uneven(args, rank: int, world: int):
    """Uneven batching: four grids (300 / 2,000 / 9,241 / 13,659 buses; 1,000 / 1,000 / 500 / 250 outages, reactive
    limits on) in ONE graph launch, the schedule picked by the multi-grid autotuner (the grids' device-resident Newton
    loops as the graph's branches, or the persistent tiles), beside a fixed persistent-tile schedule and beside one
    level-schedule batch per grid run back to back."""
    import torch
    from olfgpu import native, packing, synthetic
    from olfgpu.security_analysis import MultiGridAnalysis
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    precision = native.MIXED if args.precision == "mixed" else native.FP64
    grids = [synthetic.build(nm) for nm, _ in UNEVEN]
    packs = [packing.pack(g) for g in grids]
    counts = [c for _, c in UNEVEN]
    outs = [synthetic.draw_outages(g, c, seed=7000 + 17 * rank + i, replace=True)
            for i, (g, c) in enumerate(zip(grids, counts))]
    total = sum(counts)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        dev, wall = [], []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            dev.append(fn())
            wall.append((time.perf_counter() - t0) * 1e3)
        return float(np.mean(dev)), float(np.mean(wall))

    ordering = plan_flags(args.plan)
    member = (native.LEVELS_SHARED_ALL, 0, 256) if dense_front(args.plan) else (native.LEVELS, 2, 256)
    policy = native.MIXED_FP64_NEAR if args.mixed_policy == "fp64near" else native.MIXED_REFINE
    ma = MultiGridAnalysis(packs, counts, precision=precision, refinement_steps=args.refinement, schedule=-1,
                           ordering=ordering, member_schedule=member, mixed_policy=policy)
    ma.solve(outs)                                     # autotunes on the first solve
    pick, tuning = ma.multi.schedule()
    last = {}

    def multi_step():
        res, ms = ma.solve(outs)
        last["res"] = res
        return ms

    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", 0)))
    with sampler:
        dev_auto, wall_auto = timed(multi_step)
    res = last["res"]
    iters = [int(r.total_iterations.sum()) for r in res]
    rounds = [max(int(c.last_stats()[1]) for c, _, _ in mine) for mine in ma.grid_parts]
    ma.close()
    fixed = (2, 256, 0)                                # persistent tiles (the scaled plan: tiles run no dense front)
    mf = MultiGridAnalysis(packs, counts, precision=precision, refinement_steps=args.refinement, schedule=fixed)

    def fixed_step():
        return mf.solve(outs)[1]
    dev_fixed, _ = timed(fixed_step)
    mf.close()
    # one level-schedule batch per grid, back to back (each grid's own launches)
    seq = []
    for p, o in zip(packs, outs):
        st = native.Structure(p, ordering)
        c = native.BatchContext(st, o.shape[0], native.BATCHED_LU, p.rl)
        c.set_linear_solver_settings(precision, args.refinement)
        c.set_mixed_precision_policy(policy)
        c.set_schedule(*member)
        c.set_device_loop(True)
        seq.append((st, c, p, p.outage_masks(o)))

    def seq_step():
        ms = 0.0
        for st, c, p, dis in seq:
            c.solve(p.x_base, p.target, p.base_row_mode, dis, max_iter=15, tol=TOL)
            ms += c.last_stats()[0]
        return ms
    dev_seq, _ = timed(seq_step)
    peak, peak_kind = _peaks()
    pbytes = 4 if precision == native.MIXED else 8
    ref_steps = 1 if precision == native.MIXED else 0
    tot_bytes = 0
    for (st, c, p, dis), it in zip(seq, iters):
        tot_bytes += algorithmic_bytes(st, p, it, pbytes, ref_steps)[0]
    achieved = tot_bytes / (dev_auto * 1e-3) / 1e9
    conv = float(np.mean(np.concatenate([r.status == 0 for r in res])))
    if world > 1:
        t = torch.tensor([dev_auto, wall_auto], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        dev_auto, wall_auto = float(t[0]), float(t[1])
    h2d = sum(p.n * 8 * 2 + p.n * 4 + p.n_elements * ((c + 31) // 32) * 4 for p, c in zip(packs, counts))
    d2h = sum(c * (p.n + 3) * 8 for p, c in zip(packs, counts))
    loops = pick[0] == 0
    if loops:
        launches = 0
        for (st, c, p, dis), r in zip(seq, rounds):
            launches += launches_per_solve(st, member, max(r, 1), dense_front(args.plan), args.plan == "deferred",
                                           precision == native.MIXED, 0) + 2 + max(r, 1)
    else:
        launches = 1 + 4 + 5 * 4
    line = {
        "metric": "N-1 solves/s, uneven batch of four grids in one graph launch (reactive limits on)",
        "value": round(world * total / (dev_auto * 1e-3), 1), "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dev_auto, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32-lu+fp64" if precision == native.MIXED else "f64",
        "data": "synthetic (seeded grids, random non-bridge branch outages drawn with replacement)",
        "config": {"workload": "grid300 x1000 + grid2000q x1000 + grid9241q x500 + grid13659 x250 outages, "
                               "Q limits +-U[0.3,0.6] Pmax, reactive-limit outer loop on, tol 1e-8 pu",
                   "precision": args.precision, "l2": "working set > 1 GB per step, larger than the 126 MB L2",
                   "autotuned_schedule": {"lanes_per_tile": pick[0], "threads": pick[1],
                                          "order": ["as given", "most buses first"][pick[2]],
                                          "ms": round(dev_auto, 3)},
                   "autotuned_kind": ("one graph whose branches are the grids' device-resident Newton loops "
                                      f"(member schedule {member}, plan {args.plan})" if loops else
                                      "one persistent launch of lane tiles"),
                   "fixed_schedule": {"lanes_per_tile": fixed[0], "threads": fixed[1], "order": "as given",
                                      "kind": "persistent tiles, scaled plan",
                                      "ms": round(dev_fixed, 3),
                                      "solves_per_s": round(total / (dev_fixed * 1e-3), 1)},
                   "per_grid_level_batches": {"ms": round(dev_seq, 3),
                                              "solves_per_s": round(total / (dev_seq * 1e-3), 1)},
                   "autotune_candidates": [[int(a), int(b), int(c), round(d, 3)] for a, b, c, d in tuning],
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
        "e2e": {"value": round(world * total / (wall_auto * 1e-3), 1), "unit": "solves/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None,
                     "kernel": ("the four grids' Newton iterations (device-resident loops, one graph)" if loops else
                                "newtonMultiKernel (the whole Newton loop of the four grids in one launch)"),
                     "peak_source": f"{peak_kind} copy bandwidth (hbm_gbs)"},
        "gpu_launches": int(launches * args.steps),
        "iterations_per_solve": round(sum(iters) / total, 3),
        "converged_fraction": round(conv, 4),
        "clocks": sampler.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as O
        cores = os.cpu_count() or 1
        secs = 0.0
        sample = []
        for p, o, c in zip(packs, outs, counts):
            k = max(1, min(c, args.cpu_sample // 4))
            t0 = time.perf_counter()
            O.Structure(p).solve_batch(p.x_base, p.outage_masks(o[:k]), max_iter=15, tol=TOL, reactive_limits=True,
                                       threads=cores)
            dt = time.perf_counter() - t0
            secs += dt / k * c
            sample.append(f"{k}/{c}")
        line["cpu_baseline"] = {"value": round(total / secs, 2), "unit": "solves/s", "cores": cores, "kind": "port",
                                "sample": "oracle with reactive limits on " + ", ".join(sample) +
                                          " outages per grid, scaled to the whole mix"}
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    g, p, outs = workload(0)
    cores = os.cpu_count() or 1
    from oracle import oracle as O
    st = O.Structure(p)
    sub = outs[: args.cpu_sample]
    dis = p.outage_masks(sub)
    for _ in range(args.warmup):
        st.solve_batch(p.x_base, dis[:cores], max_iter=15, tol=TOL, threads=cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        st.solve_batch(p.x_base, dis, max_iter=15, tol=TOL, threads=cores)
        times.append(time.perf_counter() - t0)
    dt = float(np.mean(times))
    v = sub.shape[0] / dt
    line = {"metric": METRIC, "value": round(v, 2), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 2), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded 9,241-bus grid, random branch outages)",
            "impl": "reference",
            "config": {"workload": f"{GRID}: 9,241 buses, {p.n_cb} branches; a step solves {sub.shape[0]} of the "
                                   f"{N_OUTAGES} outages", "precision": "fp64"},
            "cpu_baseline": {"value": round(v, 2), "unit": "solves/s", "cores": cores, "kind": "port",
                             "sample": f"{sub.shape[0]} outages per step on {cores} threads"},
            "e2e": {"value": round(v, 2), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--refinement", type=int, default=3)
    ap.add_argument("--cpu-sample", type=int, default=96)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--start", default=None, choices=["base", "learned"],
                    help="start states: the base case, or the learned warm start (default when its checkpoint exists)")
    ap.add_argument("--checkpoint", default=CHECKPOINT)
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison run")
    ap.add_argument("--plan", default=None, choices=["scaled", "deferred", "dense", "shallow"],
                    help="block-LU plan: L scaled at its task, deferred (half the levels), dense (minimum degree, the "
                         "trailing block factorized in shared memory) or shallow (dense, on minimum degree relaxed "
                         "toward a shallow elimination tree: 121 instead of 201 levels on the 9,241-bus grid; the "
                         "default for the N-1 workload); the uneven workload's persistent launch runs the scaled plan")
    ap.add_argument("--schedule", default="auto", choices=["auto", "levels", "coop", "shared", "shared-all"],
                    help="auto: the engine's autotuner picks the Newton-iteration schedule on the first solve; "
                         "shared: level launches with the narrow factorization levels in shared memory; shared-all: "
                         "the solves' narrow levels too")
    ap.add_argument("--outages", type=int, default=N_OUTAGES,
                    help="outages per GPU (500 is the benchmark; smaller batches are profiling cases)")
    ap.add_argument("--mixed-policy", default="fp64near", choices=["fp64near", "refine"],
                    help="fp64near: iterations with a scenario near convergence run in FP64; refine: FP32 LU with "
                         "FP64 refinement of the scenarios near convergence")
    ap.add_argument("--device-loop", type=int, default=1, choices=[0, 1],
                    help="1: the whole Newton loop as one graph launch (conditional nodes)")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-batching measurement of the default line")
    ap.add_argument("--parts", type=int, default=8,
                    help="split the batch into this many lane ranges solved as concurrent device loops in one graph "
                         "(8 measured fastest on the 500-outage batch: 13.3 vs 15.6 ms per FP64 step)")
    ap.add_argument("--workload", default="n1", choices=["n1", "uneven"],
                    help="n1: the 9,241-bus N-1 batch (default); uneven: four grids in one persistent launch")
    args = ap.parse_args()
    if args.plan is None:
        args.plan = "shallow"
    if args.start is None:
        args.start = "learned" if os.path.exists(args.checkpoint) and args.outages == N_OUTAGES else "base"
    args.warmup = max(args.warmup, 3) if args.impl == "engine" else args.warmup
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.workload == "uneven":
        run_uneven(args, rank, world)
    else:
        run_engine(args, rank, world)


if __name__ == "__main__":
    main()
