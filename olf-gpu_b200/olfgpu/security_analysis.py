"""Batched N-1 AC security analysis on the engine, shaped like the reference's batch entry.

Mirrors ``GpuBatchedSecurityAnalysisSolver.solveBatchN1`` (``ac/solver/gpu/batch/GpuBatchedSecurityAnalysisSolver.java
:107-374``) for single-branch outages: the outages are installed as one disabled element per scenario, solved in
chunks sized by ``recommendBatchSize`` (``GpuBatchChunkSolver.solveQualifiedInChunks``, ``GpuBatchChunkSolver.java
:101,160``), every scenario warm-started from the base-case state, and the results are reassembled in request order.
"""
from __future__ import annotations

import concurrent.futures
import dataclasses
from typing import Optional, Sequence

import numpy as np

from . import native
from .packing import Packed


@dataclasses.dataclass
class BatchResult:
    """Per scenario: outaged closed-branch element, status, Newton iterations of the last solve, ||F||inf, state."""
    outages: np.ndarray
    status: np.ndarray
    iterations: np.ndarray
    norm: np.ndarray
    x: np.ndarray                     # [nS, n] (angles at even rows, magnitudes at odd rows for the packed grids)
    total_iterations: np.ndarray
    device_ms: float

    @property
    def vm(self) -> np.ndarray:
        return self.x[:, 1::2]

    @property
    def va(self) -> np.ndarray:
        return self.x[:, 0::2]


class SecurityAnalysis:
    """Holds the structure and one context per chunk width, reused across calls (GpuBatchContextCache)."""

    def __init__(self, packed: Packed, precision: int = native.FP64, refinement_steps: int = 1,
                 reactive_limits: bool = False, ordering: int = native.PLAN_DEFAULT, max_chunk: int = 4096,
                 schedule: Optional[tuple] = (native.LEVELS_SHARED_ALL, 0, 256)):
        """``schedule``: the arguments of BatchContext.set_schedule for every chunk's context: by default level
        launches with the narrow levels of every phase in shared memory (the fastest measured on the 9,241-bus
        batch; a plan without narrow levels falls back to plain level launches); (native.AUTOTUNE,) times every
        schedule on the first batch of each chunk width; None keeps the engine's own default."""
        self.packed = packed
        self.structure = native.Structure(packed, ordering)
        self.precision = precision
        self.refinement_steps = refinement_steps
        self.reactive_limits = reactive_limits and packed.rl is not None
        self.max_chunk = max_chunk
        self.schedule = schedule
        self._contexts = {}

    def context(self, width: int) -> native.BatchContext:
        ctx = self._contexts.get(width)
        if ctx is None:
            ctx = native.BatchContext(self.structure, width, native.BATCHED_LU,
                                      self.packed.rl if self.reactive_limits else None)
            ctx.set_linear_solver_settings(self.precision, self.refinement_steps)
            if self.schedule is not None:
                ctx.set_schedule(*self.schedule)
            self._contexts[width] = ctx
        return ctx

    def close(self):
        for c in self._contexts.values():
            c.close()
        self._contexts.clear()
        self.structure.close()

    def solve_n1(self, outages: Sequence[int], x0: Optional[np.ndarray] = None,
                 x0_per_scenario: Optional[np.ndarray] = None, max_iter: int = 15, tol: float = 1e-8,
                 reactive_limit_tol: float = 1e-4, max_outer: int = 20, max_pq_pv_switch: int = 3,
                 chunk: Optional[int] = None) -> BatchResult:
        p = self.packed
        outages = np.asarray(outages, dtype=np.int64)
        ns = outages.shape[0]
        if x0 is None:
            x0 = p.x_base if p.x_base is not None else p.x_flat
        width = chunk or self.structure.recommend_batch_size(min(ns, self.max_chunk))
        width = max(1, min(width, ns))
        n = p.n
        out = np.zeros((ns, n + 3))
        tot = np.zeros(ns, np.int32)
        ms = 0.0
        masks = p.outage_masks(outages)
        for a in range(0, ns, width):
            b = min(ns, a + width)
            ctx = self.context(width)
            dis = masks[a:b]
            xf = None if x0_per_scenario is None else x0_per_scenario[a:b]
            if b - a < width:                      # pad the last chunk with copies of its first scenario
                pad = width - (b - a)
                dis = np.concatenate([dis, np.repeat(dis[:1], pad, axis=0)])
                if xf is not None:
                    xf = np.concatenate([xf, np.repeat(xf[:1], pad, axis=0)])
            res = ctx.solve(x0, p.target, p.base_row_mode, dis, x0_full=xf, max_iter=max_iter, tol=tol,
                            reactive_limit_tol=reactive_limit_tol, max_outer=max_outer,
                            max_pq_pv_switch=max_pq_pv_switch)
            out[a:b] = res[: b - a]
            m, _, t = ctx.last_stats()
            tot[a:b] = t[: b - a]
            ms += m
        return BatchResult(outages, out[:, n + 2].astype(int), out[:, n].astype(int), out[:, n + 1], out[:, :n],
                           tot, ms)


class MultiGridAnalysis:
    """N-1 batches of several grids solved by one launch (the engine's multi-grid context).

    Each grid keeps its own structure and a context sized to its batch; ``solve`` stages every grid's outages and runs
    them together, returning one BatchResult per grid.  ``schedule`` is -1 (autotune on the first solve) or a fixed
    (lanes per tile, threads, order): persistent tiles, or lanes per tile 0 for one graph whose branches are the grids'
    device-resident Newton loops under ``member_schedule`` (schedule, lanes, threads of each grid's level schedule)."""

    def __init__(self, packed_grids: Sequence[Packed], counts: Sequence[int], precision: int = native.FP64,
                 refinement_steps: int = 1, reactive_limits: bool = True, schedule=-1, ordering: int = 0,
                 member_schedule=None, mixed_policy: int = native.MIXED_REFINE, parts=1):
        """``parts`` (an int, or one per grid): each grid's batch split into that many lane ranges, each its own member
        context on the grid's structure (for the device loops: more concurrent branches, the same results)."""
        self.packed = list(packed_grids)
        self.counts = [int(c) for c in counts]
        parts = [int(parts)] * len(self.packed) if np.isscalar(parts) else [int(k) for k in parts]
        self.structures = [native.Structure(p, ordering) for p in self.packed]
        self.contexts = []
        self.grid_parts = []           # per grid: [(context, first scenario, end)]
        for p, s, c, k in zip(self.packed, self.structures, self.counts, parts):
            bounds = np.linspace(0, c, max(1, k) + 1).round().astype(int)
            mine = []
            for a, b in zip(bounds[:-1], bounds[1:]):
                if b <= a:
                    continue
                ctx = native.BatchContext(s, int(b - a), native.BATCHED_LU,
                                          p.rl if reactive_limits and p.rl is not None else None)
                ctx.set_linear_solver_settings(precision, refinement_steps)
                ctx.set_mixed_precision_policy(mixed_policy)
                if member_schedule is not None:
                    ctx.set_schedule(*member_schedule)
                self.contexts.append(ctx)
                mine.append((ctx, int(a), int(b)))
            self.grid_parts.append(mine)
        self.multi = native.MultiContext(self.contexts)
        if schedule == -1:
            self.multi.set_schedule(-1)
        else:
            self.multi.set_schedule(*schedule)

    def close(self):
        self.multi.close()
        for c in self.contexts:
            c.close()
        for s in self.structures:
            s.close()

    def solve(self, outages: Sequence[Sequence[int]], max_iter: int = 15, tol: float = 1e-8,
              reactive_limit_tol: float = 1e-4, max_outer: int = 20, max_pq_pv_switch: int = 3):
        """outages[i]: grid i's outaged closed branches (exactly counts[i]); returns ([BatchResult], device ms)."""
        outs_all = []
        for p, mine, c, outs in zip(self.packed, self.grid_parts, self.counts, outages):
            outs = np.asarray(outs, dtype=np.int64)
            if outs.shape[0] != c:
                raise ValueError(f"expected {c} outages, got {outs.shape[0]}")
            x0 = p.x_base if p.x_base is not None else p.x_flat
            masks = p.outage_masks(outs)
            out = np.zeros((c, p.n + 3))
            outs_all.append(out)
            for ctx, a, b in mine:
                ctx.stage(x0, p.target, p.base_row_mode, masks[a:b], max_iter=max_iter, tol=tol,
                          reactive_limit_tol=reactive_limit_tol, max_outer=max_outer,
                          max_pq_pv_switch=max_pq_pv_switch)
        views = [out[a:b] for out, mine in zip(outs_all, self.grid_parts) for _, a, b in mine]
        _, ms = self.multi.solve(views)
        results = []
        for p, mine, outs, out in zip(self.packed, self.grid_parts, outages, outs_all):
            n = p.n
            tot = np.concatenate([ctx.last_stats()[2] for ctx, _, _ in mine])
            results.append(BatchResult(np.asarray(outs), out[:, n + 2].astype(int), out[:, n].astype(int),
                                       out[:, n + 1], out[:, :n], tot, ms))
        return results, ms


class ConcurrentBatch:
    """One batch of scenarios of one network split into ``parts`` lane ranges, each its own context on the shared
    structure, solved by ONE graph launch whose branches are the parts' device-resident Newton loops (the engine's
    multi-grid context with lanesPerTile 0).  The parts' level kernels run concurrently, so one part's dependent-level
    latency overlaps another's work.  Every scenario's result is that of the single batch, bit for bit (lanes never
    interact).  ``solve`` takes the arguments of BatchContext.stage for the whole batch."""

    def __init__(self, structure: native.Structure, n_scenarios: int, parts: int, precision: int = native.FP64,
                 refinement_steps: int = 1, mixed_policy: int = native.MIXED_REFINE,
                 schedule=(native.LEVELS_SHARED_ALL, 0, 256), rl=None):
        self.structure = structure
        self.n = int(n_scenarios)
        bounds = np.linspace(0, self.n, parts + 1).round().astype(int)
        self.ranges = [(int(a), int(b)) for a, b in zip(bounds[:-1], bounds[1:]) if b > a]
        self.contexts = []
        for a, b in self.ranges:
            c = native.BatchContext(structure, b - a, native.BATCHED_LU, rl)
            c.set_linear_solver_settings(precision, refinement_steps)
            c.set_mixed_precision_policy(mixed_policy)
            c.set_schedule(*schedule)
            c.set_device_loop(True)
            self.contexts.append(c)
        self.schedule = tuple(schedule)
        self.multi = native.MultiContext(self.contexts)
        self.multi.set_schedule(0, 0, 0)
        self._pool = None

    def set_schedule(self, schedule):
        """Every part's level schedule, (schedule, lanes per tile, threads) as BatchContext.set_schedule."""
        for c in self.contexts:
            c.set_schedule(*schedule)
        self.schedule = tuple(schedule)

    def autotune(self, x0_base, target, base_row_mode, disabled, candidates, x0_full=None, repeats: int = 2,
                 **kw):
        """Times each candidate schedule on this batch split into its parts (the concurrent parts interleave their
        level kernels, so the fastest schedule of one batch need not be the fastest here): per candidate one solve
        to build its graphs, then the best of ``repeats`` timed solves.  Keeps the fastest and returns
        [(schedule, ms)].  Every candidate's results are those of the single batch, bit for bit."""
        timings = []
        for cand in dict.fromkeys(tuple(c) for c in candidates):
            self.set_schedule(cand)
            self.solve(x0_base, target, base_row_mode, disabled, x0_full, **kw)
            ms = min(self.solve(x0_base, target, base_row_mode, disabled, x0_full, **kw)[1] for _ in range(repeats))
            timings.append((cand, float(ms)))
        best = min(timings, key=lambda t: t[1])[0]
        self.set_schedule(best)
        return timings

    def set_device_start(self, x0_device=None, fallback: bool = True):
        """Per-scenario start states on the device ([nS, n] torch CUDA tensor; each part reads its rows), with the
        base-start selection, fallback and polishing of BatchContext.set_fallback_start."""
        for c, (a, b) in zip(self.contexts, self.ranges):
            c.set_fallback_start(fallback and x0_device is not None)
            c.set_device_start(None if x0_device is None else x0_device[a:b])

    def solve(self, x0_base, target, base_row_mode, disabled, x0_full=None, max_iter: int = 15, tol: float = 1e-8,
              out: Optional[np.ndarray] = None):
        """[nS][n + 3] results in scenario order (written into ``out`` when given); returns (results, device ms)."""
        n = self.structure.n
        if out is None:
            out = np.zeros((self.n, n + 3))

        def stage(k):
            (a, b), c = self.ranges[k], self.contexts[k]
            c.stage(x0_base, target, base_row_mode, disabled[a:b], None if x0_full is None else x0_full[a:b],
                    max_iter=max_iter, tol=tol)
        # the parts' host work (validation, outage bit packing) and uploads run side by side: the library call
        # releases the interpreter lock, and each part has its own buffers and stream
        if self._pool is None:
            self._pool = concurrent.futures.ThreadPoolExecutor(max_workers=len(self.contexts))
        for f in [self._pool.submit(stage, k) for k in range(len(self.contexts))]:
            f.result()
        views = [out[a:b] for a, b in self.ranges]
        _, ms = self.multi.solve(views)
        return out, ms

    def last_fallbacks(self) -> np.ndarray:
        return np.concatenate([c.last_fallbacks() + a for c, (a, _) in zip(self.contexts, self.ranges)])

    def last_fp64_iterations(self) -> int:
        return max(c.last_fp64_iterations() for c in self.contexts)

    def close(self):
        if self._pool is not None:
            self._pool.shutdown()
            self._pool = None
        self.multi.close()
        for c in self.contexts:
            c.close()
