"""Learned warm start for batched N-1: data from the engine's own solves, training on the GPU with the library's
kernels, and prediction of every scenario's start state, with the plain Newton judging every scenario.

* Training data: for load scalings s ~ U[0.8, 1.2] of the grid, the base case is solved on the engine, then a batch of
  random non-bridge branch outages warm-started from it; each converged scenario gives one sample (the base case's
  node features, the outaged branch, the per-bus change (dVm, dVa) of the solution).
* Prediction: x0 = base state + the network's (dVm, dVa); identity rows (slack angle, PV magnitudes) start at their
  targets.  Any scenario the Newton does not converge from the learned start is solved again from the base-case
  start (the fallback), so the result never depends on the network beyond the iteration count.
"""
from __future__ import annotations

import dataclasses
import time
from typing import List, Optional

import numpy as np

from . import native, packing
from .gnn import FEAT_IN, GraphData, WarmStartNet


N_FEAT = 7            # per-bus base-case features; columns 7..9 carry the per-sample outage features


def branch_flows(g, x_base: np.ndarray):
    """Base-case active and reactive flow leaving bus 1 (side 1) of every closed branch (pi model, per unit)."""
    vm, va = x_base[1::2], x_base[0::2]
    y = 1.0 / np.hypot(g.r, g.x)
    ksi = np.arctan2(g.r, g.x)
    v1, v2, r1 = vm[g.f], vm[g.t], g.ratio
    th = ksi - va[g.f] + va[g.t]
    p1 = r1 * v1 * (y * r1 * v1 * np.sin(ksi) - y * v2 * np.sin(th))
    q1 = r1 * v1 * (-g.b / 2 * r1 * v1 + y * r1 * v1 * np.cos(ksi) - y * v2 * np.cos(th))
    return p1, q1


def node_features(p, x_base: np.ndarray) -> np.ndarray:
    """[nb, 7]: base-case Vm, Va, net P, net Q (PQ rows; 0 on voltage-controlled rows), PQ / PV / slack flags."""
    nb = p.n_bus
    vm, va = x_base[1::2], x_base[0::2]
    P = p.target[0::2].copy()
    slack = p.base_row_mode[0::2] == packing.FIXED_VARIABLE
    P[slack] = 0.0
    pv = p.base_row_mode[1::2] == packing.FIXED_VARIABLE
    Q = np.where(pv, 0.0, p.target[1::2])
    return np.stack([vm, va, P, Q, (~pv).astype(float), (pv & ~slack).astype(float), slack.astype(float)], axis=1)


@dataclasses.dataclass
class Dataset:
    x: "object"          # [nScalings, nb, 16] bf16 normalised node features (outage columns zero)
    t: "object"          # [nSamples, nb, 2] fp32 normalised targets
    scaling: "object"    # [nSamples] int64 index into x
    outage: "object"     # [nSamples] int32 closed-branch index
    flows: "object"      # [nScalings, nBranches, 2] fp32 base-case (P, Q) flows, already scaled by flow_std
    feat_mean: np.ndarray
    feat_std: np.ndarray
    tgt_std: np.ndarray
    flow_std: float


class LearnedStart:
    def __init__(self, grid, layers: int = 4, seed: int = 0, net: Optional[WarmStartNet] = None):
        self.grid = grid
        self.graph = GraphData.from_grid(grid)
        self.net = net or WarmStartNet(self.graph, layers, seed)
        self.feat_mean = None
        self.feat_std = None
        self.tgt_std = None
        self.flow_std = 1.0
        self._adj = None
        self._reach_cache = {}
        self._base_cache = {}
        self._branch_ends = None

    # ------------------------------------------------------------------------------------------------------------
    def solve_base(self, g, x_start: np.ndarray) -> np.ndarray:
        p = packing.pack(g, with_reactive_limits=False)
        s = native.Structure(p)
        ctx = native.BatchContext(s, 1)
        r = ctx.solve(x_start, p.target, p.base_row_mode, np.zeros((1, p.n_elements), np.uint8))
        if int(r[0, -1]) != native.CONVERGED:
            raise RuntimeError("base case does not converge")
        return r[0, :p.n].copy()

    def generate(self, n_scalings: int, outages_per_scaling: int, seed: int, lo: float = 0.8, hi: float = 1.2,
                 precision: int = native.FP64) -> Dataset:
        """Samples from the engine's own N-1 solves at n_scalings random load scalings."""
        import torch
        from . import synthetic
        rng = np.random.default_rng(seed)
        base_grid = self.grid
        p0 = packing.pack(base_grid, with_reactive_limits=False)
        x_ref = p0.x_base if p0.x_base is not None else p0.x_flat
        cand = synthetic.outage_candidates(base_grid)
        feats, targets, scal, outs, flows = [], [], [], [], []
        s0 = native.Structure(p0)
        ctx = native.BatchContext(s0, outages_per_scaling)
        ctx.set_linear_solver_settings(precision, 1)
        for k in range(n_scalings):
            sc = float(rng.uniform(lo, hi))
            g = base_grid.scaled(sc)
            p = packing.pack(g, with_reactive_limits=False)
            try:
                xb = self.solve_base(g, x_ref)
            except RuntimeError:
                continue                                    # no base case at this loading: no sample
            o = np.sort(rng.choice(cand, size=outages_per_scaling, replace=False))
            r = ctx.solve(xb, p.target, p.base_row_mode, p.outage_masks(o))
            ok = r[:, -1] == native.CONVERGED
            idx = len(feats)
            feats.append(node_features(p, xb))
            flows.append(np.stack(branch_flows(g, xb), axis=1))
            d = np.stack([r[ok, 1:p.n:2] - xb[1::2], r[ok, 0:p.n:2] - xb[0::2]], axis=2)   # [k, nb, 2]
            targets.append(d.astype(np.float32))
            scal.append(np.full(int(ok.sum()), idx, np.int64))
            outs.append(o[ok].astype(np.int32))
        if not feats:
            raise RuntimeError("no load scaling had a solvable base case")
        f = np.stack(feats)                                         # [nS, nb, 7]
        mean = f.reshape(-1, N_FEAT).mean(0)
        std = np.maximum(f.reshape(-1, N_FEAT).std(0), 1e-6)
        mean[4:] = 0.0
        std[4:] = 1.0
        fx = np.zeros((f.shape[0], f.shape[1], FEAT_IN), np.float32)
        fx[..., :N_FEAT] = (f - mean) / std
        fl = np.stack(flows).astype(np.float32)
        flow_std = float(max(fl.std(), 1e-6))
        t = np.concatenate(targets)
        tstd = np.maximum(t.reshape(-1, 2).std(0), 1e-9).astype(np.float32)
        dev = torch.device("cuda")
        self.feat_mean, self.feat_std, self.tgt_std, self.flow_std = mean, std, tstd, flow_std
        return Dataset(torch.from_numpy(fx).to(dev).to(torch.bfloat16), torch.from_numpy(t / tstd).to(dev),
                       torch.from_numpy(np.concatenate(scal)).to(dev), torch.from_numpy(np.concatenate(outs)).to(dev),
                       torch.from_numpy(fl / flow_std).to(dev), mean, std, tstd, flow_std)

    def _batch_inputs(self, xs, flows, outages):
        """Node inputs [B * nb, 16] bf16: the scaling's features plus the per-sample outage columns (7..9)."""
        import torch
        g = self.grid
        B = outages.shape[0]
        nb = self.graph.nb
        x = xs.clone() if xs.dim() == 3 else xs.unsqueeze(0).expand(B, nb, FEAT_IN).clone()
        fidx = torch.from_numpy(g.f.astype(np.int64)).to(x.device)[outages.long()]
        tidx = torch.from_numpy(g.t.astype(np.int64)).to(x.device)[outages.long()]
        rows = torch.arange(B, device=x.device)
        fl = flows[rows, outages.long()] if flows.dim() == 3 else flows[outages.long()]
        one = torch.ones(B, device=x.device, dtype=x.dtype)
        x[rows, fidx, N_FEAT] = one
        x[rows, tidx, N_FEAT] = one
        x[rows, fidx, N_FEAT + 1] = fl[:, 0].to(x.dtype)
        x[rows, tidx, N_FEAT + 1] = (-fl[:, 0]).to(x.dtype)
        x[rows, fidx, N_FEAT + 2] = fl[:, 1].to(x.dtype)
        x[rows, tidx, N_FEAT + 2] = (-fl[:, 1]).to(x.dtype)
        return x.reshape(B * nb, FEAT_IN).contiguous()

    def split(self, data: Dataset, held_out_scalings: int):
        """(training, held-out) sample indices: the last ``held_out_scalings`` load scalings are held out."""
        import torch
        cut = int(data.x.shape[0]) - held_out_scalings
        mask = data.scaling >= cut
        return torch.nonzero(~mask).flatten(), torch.nonzero(mask).flatten()

    def evaluate(self, data: Dataset, samples=None, chunk: int = 32):
        """(mean normalised squared error of the network, of the base start) over the samples: the base start predicts
        no change, so its error is the mean squared normalised target."""
        import torch
        nb = self.graph.nb
        idx_all = torch.arange(data.t.shape[0], device="cuda") if samples is None else samples
        err = base = 0.0
        cnt = 0
        for a in range(0, idx_all.shape[0], chunk):
            idx = idx_all[a:a + chunk]
            out = data.outage[idx].contiguous()
            x0 = self._batch_inputs(data.x[data.scaling[idx]], data.flows[data.scaling[idx]], out)
            pred = self.net.forward(x0, out)[:, :2]
            tg = data.t[idx].reshape(idx.shape[0] * nb, 2)
            err += float(((pred - tg) ** 2).sum())
            base += float((tg ** 2).sum())
            cnt += tg.numel()
        return err / max(cnt, 1), base / max(cnt, 1)

    def train(self, data: Dataset, epochs: int = 3, batch: int = 32, lr: float = 2e-3, seed: int = 0,
              log: Optional[list] = None, max_seconds: Optional[float] = None, samples=None) -> List[float]:
        """Adam on minibatches (of ``samples``, default all); the learning rate decays linearly to 10 % over the run.
        Returns per-epoch losses."""
        import torch
        self._base_cache.clear()                   # the outage-free pass depends on the weights and normalisation
        self.feat_mean, self.feat_std, self.tgt_std = data.feat_mean, data.feat_std, data.tgt_std
        self.flow_std = data.flow_std
        pool = torch.arange(data.t.shape[0], device="cuda") if samples is None else samples
        n = int(pool.shape[0])
        nb = self.graph.nb
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed)
        steps_total = epochs * max(1, n // batch)
        step = 0
        losses = []
        t0 = time.time()
        for ep in range(epochs):
            perm = pool[torch.randperm(n, device="cuda", generator=gen)]
            acc, cnt = 0.0, 0
            for a in range(0, n - batch + 1, batch):
                idx = perm[a:a + batch]
                out = data.outage[idx].contiguous()
                sc = data.scaling[idx]
                x0 = self._batch_inputs(data.x[sc], data.flows[sc], out)
                tg = data.t[idx].reshape(batch * nb, 2).contiguous()
                rate = lr * (1.0 - 0.9 * step / max(1, steps_total))
                loss = self.net.loss_and_grad(x0, out, tg)
                self.net.adam(rate)
                acc += loss
                cnt += 1
                step += 1
                if log is not None and step % 100 == 0:
                    log.append((step, loss))
                if max_seconds is not None and time.time() - t0 > max_seconds:
                    break
            losses.append(acc / max(cnt, 1))
            if max_seconds is not None and time.time() - t0 > max_seconds:
                break
        torch.cuda.synchronize()
        self.last_train_seconds, self.last_train_steps = time.time() - t0, step
        return losses

    # ------------------------------------------------------------------------------------------------------------
    def reach(self, outages: np.ndarray):
        """The buses each outage can influence through the network: those within `layers` hops of the outaged
        branch's ends (a layer moves information one hop).  Returns int32 arrays (row_node, row_sample) ordered by
        sample then bus, and row_of [B * nb] (-1 outside).  Depends only on the topology and the outages (memoised)."""
        import scipy.sparse as sp
        key = np.asarray(outages, np.int64).tobytes()
        hit = self._reach_cache.get(key)
        if hit is not None:
            return hit
        g = self.grid
        nb = self.graph.nb
        if self._adj is None:
            a = sp.coo_matrix((np.ones(2 * g.f.shape[0], np.float32), (np.concatenate([g.f, g.t]),
                                                                        np.concatenate([g.t, g.f]))), shape=(nb, nb))
            self._adj = (a.tocsr() + sp.identity(nb, dtype=np.float32, format="csr")).astype(bool).astype(np.float32)
        outs = np.asarray(outages, np.int64)
        B = outs.shape[0]
        cols = np.concatenate([np.arange(B), np.arange(B)])
        rws = np.concatenate([g.f[outs], g.t[outs]])
        r = sp.csr_matrix((np.ones(2 * B, np.float32), (rws, cols)), shape=(nb, B))
        for _ in range(self.net.layers):
            r = (self._adj @ r)
            r.data[:] = 1.0
        rc = r.tocsc()
        rc.sort_indices()
        row_sample = np.repeat(np.arange(B, dtype=np.int32), np.diff(rc.indptr)).astype(np.int32)
        row_node = rc.indices.astype(np.int32)
        row_of = np.full(B * nb, -1, np.int32)
        row_of[row_sample.astype(np.int64) * nb + row_node] = np.arange(row_node.shape[0], dtype=np.int32)
        hit = (row_node, row_sample, row_of)
        if len(self._reach_cache) > 8:
            self._reach_cache.clear()
        self._reach_cache[key] = hit
        return hit

    def predict_device(self, p, x_base: np.ndarray, outages: np.ndarray, chunk: int = 128, out=None,
                       compact: bool = True):
        """Start states [nS, n] (float64, a CUDA tensor) for the outages, from the base case state: the network's
        forward passes and the composition of the states (olfgpu_gnn_compose_start) all run on the device.  With
        `compact`, one outage-free forward pass serves every bus an outage cannot reach and only the buses within
        reach of each outage are evaluated per scenario (the same values, bit for bit, at a fraction of the work)."""
        import torch
        from .gnn import _call, _ptr, _stream
        nb = p.n_bus
        # everything that depends only on the base state (features, flows, the outage-free forward pass) is kept for
        # the next call with the same base state and targets
        key = (hash(np.ascontiguousarray(x_base, np.float64).tobytes()), hash(p.target.tobytes()),
               hash(p.base_row_mode.tobytes()), bool(compact))
        base = self._base_cache.get(key)
        if base is None:
            f = node_features(p, x_base)
            fx = np.zeros((nb, FEAT_IN), np.float32)
            fx[:, :N_FEAT] = (f - self.feat_mean) / self.feat_std
            xf = torch.from_numpy(fx).cuda().to(torch.bfloat16)
            # branch impedances do not depend on the loading: the flows come from this grid's branches and x_base
            fl = torch.from_numpy(np.stack(branch_flows(self.grid, x_base), axis=1).astype(np.float32) /
                                  self.flow_std).cuda()
            xb = torch.from_numpy(np.ascontiguousarray(x_base, np.float64)).cuda()
            ident = torch.from_numpy((p.base_row_mode == packing.FIXED_VARIABLE).astype(np.uint8)).cuda()
            tgt = torch.from_numpy(np.ascontiguousarray(p.target, np.float64)).cuda()
            base_out = base_pq = None
            if compact:
                none = torch.full((1,), -1, dtype=torch.int32, device="cuda")
                base_out, base_pq = self.net.forward_rows(xf.contiguous(), none, keep_pq=True)
            base = (xf, fl, xb, ident, tgt, base_out, base_pq)
            self._base_cache.clear()
            self._base_cache[key] = base
        xf, fl, xb, ident, tgt, base_out, base_pq = base
        outs = torch.from_numpy(np.asarray(outages, np.int32)).cuda()
        ns = outs.shape[0]
        x0 = torch.empty((ns, p.n), dtype=torch.float64, device="cuda") if out is None else out
        std0, std1 = float(self.tgt_std[0]), float(self.tgt_std[1])
        if compact:
            rn_h, rs_h, _ = self.reach(outages)
            R = int(rn_h.shape[0])
            # one host-to-device copy for the row lists; the (sample, bus) -> row map is written on the device
            packed = torch.from_numpy(np.concatenate([rn_h, rs_h])).cuda()
            rn, rs = packed[:R], packed[R:]
            ro = torch.full((ns * nb,), -1, dtype=torch.int32, device="cuda")
            if self._branch_ends is None:
                self._branch_ends = (torch.from_numpy(self.grid.f.astype(np.int32)).cuda(),
                                     torch.from_numpy(self.grid.t.astype(np.int32)).cuda())
            xc = torch.empty((R, FEAT_IN), dtype=xf.dtype, device="cuda")
            _call("olfgpu_gnn_compact_inputs", R, nb, N_FEAT, _ptr(rn), _ptr(rs), _ptr(outs),
                  _ptr(self._branch_ends[0]), _ptr(self._branch_ends[1]), _ptr(xf), _ptr(fl), _ptr(xc), _ptr(ro),
                  _stream())
            rows_out = self.net.forward_rows(xc, outs, rows=(rn, rs, ro), base_pq=base_pq)
            _call("olfgpu_gnn_compose_start_compact", ns, nb, _ptr(base_out), _ptr(rows_out), base_out.shape[1],
                  int(rn.shape[0]), _ptr(rn), _ptr(rs), std0, std1, _ptr(xb), _ptr(ident), _ptr(tgt), _ptr(x0),
                  _stream())
            return x0
        for a in range(0, ns, chunk):
            b = min(ns, a + chunk)
            o = outs[a:b].contiguous()
            pred = self.net.forward(self._batch_inputs(xf, fl, o), o)
            _call("olfgpu_gnn_compose_start", b - a, nb, _ptr(pred), pred.shape[1], std0, std1, _ptr(xb), _ptr(ident),
                  _ptr(tgt), _ptr(x0[a:b]), _stream())
        return x0

    def predict(self, p, x_base: np.ndarray, outages: np.ndarray, chunk: int = 128, compact: bool = True):
        """Start states [nS, n] (float64, on the host) for the outages, from the base case state."""
        return self.predict_device(p, x_base, outages, chunk, compact=compact).cpu().numpy()

    def save(self, path: str):
        self.net.save(path, {"feat_mean": self.feat_mean, "feat_std": self.feat_std, "tgt_std": self.tgt_std,
                             "flow_std": np.array(self.flow_std), "fingerprint": fingerprint(self.grid)})

    @staticmethod
    def load(path: str, grid) -> "LearnedStart":
        graph = GraphData.from_grid(grid)
        net, extra = WarmStartNet.load(path, graph)
        if not np.array_equal(extra["fingerprint"], fingerprint(grid)):
            raise ValueError("checkpoint was trained on another grid")
        ls = LearnedStart(grid, net=net)
        ls.feat_mean, ls.feat_std, ls.tgt_std = extra["feat_mean"], extra["feat_std"], extra["tgt_std"]
        ls.flow_std = float(extra["flow_std"])
        return ls


def fingerprint(grid) -> np.ndarray:
    """A few numbers that identify the grid's topology and parameters."""
    return np.array([grid.n_bus, grid.f.shape[0], float(np.sum(grid.f * 7 + grid.t * 13)), float(np.sum(grid.r)),
                     float(np.sum(grid.x)), float(grid.scale)])


def solve_with_fallback(ctx, p, x0_learned, x_base: np.ndarray, disabled: np.ndarray, **kw):
    """Solve from the learned starts (a host array [nS, n] or a CUDA tensor from predict_device).  Each scenario
    keeps whichever of its learned start and the base start has the smaller initial mismatch, and a scenario that
    diverges, reaches the iteration cap or fails its linear solve restarts once from the base start, inside the same
    batch (the engine's fallback start).  Returns (results, total Newton iterations per scenario, indices of the
    scenarios that used the base start)."""
    on_device = hasattr(x0_learned, "data_ptr")
    ctx.set_fallback_start(True)
    try:
        if on_device:
            import torch
            torch.cuda.current_stream().synchronize()      # the prediction ran on torch's stream
            ctx.set_device_start(x0_learned)
            r = ctx.solve(x_base, p.target, p.base_row_mode, disabled, **kw).copy()
        else:
            r = ctx.solve(x_base, p.target, p.base_row_mode, disabled, x0_full=x0_learned, **kw).copy()
    finally:
        ctx.set_fallback_start(False)
        if on_device:
            ctx.set_device_start(None)
    _, _, tot = ctx.last_stats()
    return r, tot.copy(), ctx.last_fallbacks()


# ----------------------------------------------------------------------------------------------------------------
# Command line: train a checkpoint on the engine's own N-1 solutions, and evaluate learned / base / flat starts.
# ----------------------------------------------------------------------------------------------------------------
def _start_error(x0: np.ndarray, sol: np.ndarray, ok: np.ndarray):
    """max |dVm|, max |dVa| and the RMS over buses between the starts and the converged states (converged rows)."""
    if not ok.any():
        return None
    d = x0[ok] - sol[ok]
    return {"max_abs_dVm_pu": float(np.abs(d[:, 1::2]).max()), "max_abs_dVa_rad": float(np.abs(d[:, 0::2]).max()),
            "rms_dVm_pu": float(np.sqrt(np.mean(d[:, 1::2] ** 2))), "rms_dVa_rad": float(np.sqrt(np.mean(d[:, 0::2] ** 2)))}


def _histogram(it: np.ndarray, ok: np.ndarray) -> dict:
    vals, counts = np.unique(it[ok].astype(int), return_counts=True)
    return {str(int(v)): int(c) for v, c in zip(vals, counts)}


def evaluate_starts(ls: "LearnedStart", scaling: float, n_outages: int, seed: int, max_iter: int = 15,
                    tol: float = 1e-8) -> dict:
    """Learned vs base vs flat start on ``n_outages`` outages at the load ``scaling`` (FP64 Newton referees each start
    alone; the learned start is also run the way the product runs it: per scenario the better start by initial
    mismatch, and a failed scenario restarts from the base start).  Iterations, converged fraction, the iteration
    histogram and the start error against the converged states."""
    from . import synthetic
    g = ls.grid.scaled(scaling)
    p = packing.pack(g, with_reactive_limits=False)
    p0 = packing.pack(ls.grid, with_reactive_limits=False)
    xb = ls.solve_base(g, p0.x_base if p0.x_base is not None else p0.x_flat)
    rng = np.random.default_rng(seed)
    outs = np.sort(rng.choice(synthetic.outage_candidates(ls.grid), size=n_outages, replace=False)).astype(np.int32)
    dis = p.outage_masks(outs)
    s = native.Structure(p, native.PLAN_DEFAULT)
    ctx = native.BatchContext(s, n_outages)
    ctx.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
    # the referee: FP64 Newton from the base start (the converged states the starts are measured against)
    ref = ctx.solve(xb, p.target, p.base_row_mode, dis, max_iter=max_iter, tol=tol).copy()
    ok_ref = ref[:, -1] == native.CONVERGED
    learned = ls.predict(p, xb, outs)
    starts = {"learned": learned, "base": np.tile(xb, (n_outages, 1)), "flat": np.tile(p.x_flat, (n_outages, 1))}
    report = {"grid": ls.grid.spec.name, "scaling": scaling, "outages": n_outages, "seed": seed, "tol": tol,
              "referee_converged_fraction": float(ok_ref.mean())}
    for name, x0 in starts.items():
        r = ctx.solve(None, p.target, p.base_row_mode, dis, x0_full=x0, max_iter=max_iter, tol=tol)
        ok = r[:, -1] == native.CONVERGED
        same = ok & ok_ref
        d = np.abs(r[same, :p.n] - ref[same, :p.n]) if same.any() else np.zeros((1, 1))
        report[name] = {"converged_fraction": float(ok.mean()),
                        "iterations_per_solve": float(r[ok, p.n].mean()) if ok.any() else None,
                        "iteration_histogram": _histogram(r[:, p.n], ok),
                        "one_iteration_fraction": float(((r[:, p.n] == 1) & ok).mean()),
                        "start_error": _start_error(x0, ref[:, :p.n], ok_ref),
                        "max_state_difference_vs_referee": float(d.max())}
    r, tot, fell = solve_with_fallback(ctx, p, learned, xb, dis, max_iter=max_iter, tol=tol)
    ok = r[:, -1] == native.CONVERGED
    report["learned_with_fallback"] = {"converged_fraction": float(ok.mean()),
                                       "iterations_per_solve": float(tot[ok].mean()) if ok.any() else None,
                                       "iteration_histogram": _histogram(r[:, p.n], ok),
                                       "scenarios_on_base_start": int(fell.size),
                                       "same_status_as_referee": int((r[:, -1] == ref[:, -1]).sum())}
    return report


def main(argv=None) -> int:
    import argparse
    import json
    import os
    from . import synthetic
    ap = argparse.ArgumentParser(prog="python -m olfgpu.learned_start",
                                 description="Train or evaluate the learned warm start (needs a CUDA GPU).")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train", help="generate N-1 solutions with the engine and train a checkpoint on them")
    t.add_argument("--grid", default="grid9241")
    t.add_argument("--scalings", type=int, default=100, help="load scalings U[lo, hi] (one base case each)")
    t.add_argument("--per-scaling", type=int, default=500, help="random non-bridge outages solved per scaling")
    t.add_argument("--held-out", type=int, default=2, help="the last scalings are held out of training")
    t.add_argument("--lo", type=float, default=0.8)
    t.add_argument("--hi", type=float, default=1.2)
    t.add_argument("--epochs", type=int, default=6)
    t.add_argument("--batch", type=int, default=32)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--seed", type=int, default=9241)
    t.add_argument("--max-seconds", type=float, default=None)
    t.add_argument("--out", required=True, help="checkpoint path (.npz)")
    t.add_argument("--report", default=None, help="JSON report path (default: next to the checkpoint)")
    e = sub.add_parser("eval", help="learned vs base vs flat start on held-out outages at a fresh load scaling")
    e.add_argument("--grid", default="grid9241")
    e.add_argument("--checkpoint", required=True)
    e.add_argument("--scaling", type=float, default=1.07, help="the fresh load scaling (not a training draw)")
    e.add_argument("--outages", type=int, default=500)
    e.add_argument("--seed", type=int, default=424242)
    e.add_argument("--report", default=None)
    a = ap.parse_args(argv)
    g = synthetic.build(a.grid)
    if a.cmd == "train":
        t0 = time.time()
        ls = LearnedStart(g, seed=a.seed)
        data = ls.generate(a.scalings, a.per_scaling, seed=a.seed, lo=a.lo, hi=a.hi)
        gen_s = time.time() - t0
        train_idx, held = ls.split(data, a.held_out)
        before = ls.evaluate(data, held)
        losses = ls.train(data, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed, samples=train_idx,
                          max_seconds=a.max_seconds)
        after = ls.evaluate(data, held)
        ls.save(a.out)
        rep = {"grid": a.grid, "samples": int(data.t.shape[0]), "training_samples": int(train_idx.shape[0]),
               "held_out_samples": int(held.shape[0]), "scalings": a.scalings, "per_scaling": a.per_scaling,
               "load_scaling_range": [a.lo, a.hi], "epochs": a.epochs, "batch": a.batch, "lr": a.lr, "seed": a.seed,
               "adam_steps": int(ls.net.step), "epoch_losses": [float(v) for v in losses],
               "held_out_normalised_mse": {"network": after[0], "untrained": before[0], "base_start": after[1]},
               "generate_seconds": round(gen_s, 1), "train_seconds": round(ls.last_train_seconds, 2),
               "ms_per_adam_step": round(1e3 * ls.last_train_seconds / max(1, ls.last_train_steps), 3),
               "total_seconds": round(time.time() - t0, 1)}
        path = a.report or os.path.splitext(a.out)[0] + ".train.json"
    else:
        ls = LearnedStart.load(a.checkpoint, g)
        rep = evaluate_starts(ls, a.scaling, a.outages, a.seed)
        rep["checkpoint"] = os.path.basename(a.checkpoint)
        path = a.report or os.path.splitext(a.checkpoint)[0] + ".eval.json"
    with open(path, "w") as f:
        json.dump(rep, f, indent=1)
    print(json.dumps(rep, indent=1))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
