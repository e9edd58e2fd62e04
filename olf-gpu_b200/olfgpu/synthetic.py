"""Seeded synthetic transmission grids standing in for the case files the reference benchmarks on.

The reference measures N-1 throughput on pegase9241 / rte6515 case files (``GpuBatchedN1FixedIterTest.java:71``,
``codegen/bench/gen_contingencies.py:4-7``). Those files are not available, so grids of the same shapes are generated
here from a seed:

* topology: a random spanning tree over the buses plus extra random edges (parallel edges allowed, no self loops).
  Buses get random positions in the unit square; the tree joins each bus to a near, earlier-placed bus and the extra
  edges join a bus to one of its nearest neighbours.  Transmission grids are nearly planar with local connections;
  uniformly random extra edges would make an expander graph whose sparse LU fills in densely, which no real grid
  does (pegase9241 factors with 2.0x fill, ``docs/archive/gpu_benchmark.md:45-47``).
* lines: r ~ U[0.005, 0.05] pu, x = r * U[3, 10], total charging b ~ U[0, 0.05] pu split evenly on both sides.
* transformers (a share of the branches): ratio ~ U[0.95, 1.05] on side 1, no phase shift, no charging.
* PV generators with Vset ~ U[0.98, 1.05]; one slack (the largest generator); PQ loads with
  P ~ lognormal(ln 0.3, 0.6) pu and power factor ~ U[0.90, 0.98].
* generation shares the total load: each load is served by its nearest generator (times a random weight U[0.8, 1.2]);
  the slack absorbs the losses.
* a loading scale calibrated by Newton-Raphson on the base case (see ``calibrate_scale``).

Everything is per unit on a 100 MVA base.  The calibration Newton below is input preparation only; the engine that
is measured and shipped is the CUDA library.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


@dataclasses.dataclass
class GridSpec:
    """Shape of one synthetic grid (sizes, shares and the loading rule)."""
    name: str
    n_bus: int
    n_branch: int
    n_gen: int
    n_load: int
    transformer_share: float
    seed: int
    loading: str = "converge6"          # "converge6" (flat start converges in <= 6 iterations) or "collapse80"
    q_limits: bool = False              # generator reactive limits +-U[0.3, 0.6] * Pmax
    shunt_share: float = 0.03           # fixed shunts on PQ buses (exercise the shunt family)
    open_branches: int = 0              # branches open at one end (exercise the open-branch family)


# The five benchmark workloads (sizes from the benchmark definition; seeds fixed here and recorded).
SPECS = {
    "grid118": GridSpec("grid118", 118, 186, 54, 99, 0.10, seed=118, loading="converge6", open_branches=2),
    "grid300": GridSpec("grid300", 300, 480, 60, 195, 0.10, seed=300, loading="converge6", q_limits=True),
    "grid2000": GridSpec("grid2000", 2000, 3200, 400, 1300, 0.10, seed=2000, loading="converge6"),
    "grid2000q": GridSpec("grid2000q", 2000, 3200, 400, 1300, 0.10, seed=2001, loading="converge6", q_limits=True),
    "grid9241": GridSpec("grid9241", 9241, 16000, 1450, 6000, 0.25, seed=9241, loading="collapse80"),
    "grid9241q": GridSpec("grid9241q", 9241, 14786, 1450, 6000, 0.25, seed=9242, loading="collapse80", q_limits=True),
    "grid13659": GridSpec("grid13659", 13659, 21854, 2150, 8900, 0.25, seed=13659, loading="collapse80", q_limits=True),
}


@dataclasses.dataclass
class Grid:
    """A generated grid in plain arrays (per unit).  Branch k joins f[k] -> t[k]; side 1 is f."""
    spec: GridSpec
    n_bus: int
    f: np.ndarray
    t: np.ndarray
    r: np.ndarray
    x: np.ndarray
    b: np.ndarray            # total line charging (split b/2 on each side)
    ratio: np.ndarray        # side-1 ratio rho (1 for lines)
    is_transformer: np.ndarray
    gen_bus: np.ndarray
    gen_p: np.ndarray
    gen_vset: np.ndarray
    gen_pmax: np.ndarray
    gen_minq: np.ndarray
    gen_maxq: np.ndarray
    load_bus: np.ndarray
    load_p: np.ndarray
    load_q: np.ndarray
    shunt_bus: np.ndarray
    shunt_g: np.ndarray
    shunt_b: np.ndarray
    open_bus: np.ndarray     # bus the open branch hangs from
    open_side: np.ndarray    # 1: side 1 connected (side 2 open); 2: side 2 connected (side 1 open)
    open_r: np.ndarray
    open_x: np.ndarray
    open_b: np.ndarray
    slack: int
    scale: float = 1.0       # loading scale applied to loads and generation
    base_vm: Optional[np.ndarray] = None   # base-case solution found by the calibration (the N-1 warm start)
    base_va: Optional[np.ndarray] = None

    @property
    def n_branch(self) -> int:
        return int(self.f.shape[0])

    def scaled(self, s: float) -> "Grid":
        """The same grid with loads and generator set points multiplied by ``s`` (relative to this one)."""
        g = dataclasses.replace(self)
        g.load_p = self.load_p * s
        g.load_q = self.load_q * s
        g.gen_p = self.gen_p * s
        g.scale = self.scale * s
        g.base_vm = g.base_va = None
        return g


def _nearest(pos: np.ndarray, k: int) -> np.ndarray:
    """The k nearest neighbours of every point (excluding itself)."""
    from scipy.spatial import cKDTree
    _, idx = cKDTree(pos).query(pos, k=k + 1)
    return idx[:, 1:].astype(np.int64)


def _find(parent: np.ndarray, i: int) -> int:
    while parent[i] != i:
        parent[i] = parent[parent[i]]
        i = parent[i]
    return i


def _local_spanning_tree(pos: np.ndarray, rng: np.random.Generator):
    """A random spanning tree over local edges: randomized Kruskal on the 8-nearest-neighbour graph, with any
    leftover components joined to their nearest bus outside them."""
    nb = pos.shape[0]
    nn = _nearest(pos, min(8, nb - 1))
    cand = np.stack([np.repeat(np.arange(nb), nn.shape[1]), nn.ravel()], axis=1)
    cand = cand[rng.permutation(cand.shape[0])]
    parent = np.arange(nb)
    edges = []
    for u, v in cand:
        ru, rv = _find(parent, int(u)), _find(parent, int(v))
        if ru != rv:
            parent[ru] = rv
            edges.append((int(u), int(v)))
    while len(edges) < nb - 1:
        roots = np.array([_find(parent, i) for i in range(nb)])
        comp = roots == roots[0]
        ins, outs = np.flatnonzero(comp), np.flatnonzero(~comp)
        from scipy.spatial import cKDTree
        d, j = cKDTree(pos[outs]).query(pos[ins], k=1)
        a = int(np.argmin(d))
        u, v = int(ins[a]), int(outs[int(j[a])])
        parent[_find(parent, u)] = _find(parent, v)
        edges.append((u, v))
    return edges


def generate(spec: GridSpec) -> Grid:
    """Draw the grid of ``spec`` (unscaled loading: ``scale`` = 1)."""
    rng = np.random.default_rng(spec.seed)
    nb = spec.n_bus
    pos = rng.random((nb, 2))
    # spanning tree over local edges
    tree = _local_spanning_tree(pos, rng)
    f_list = [u for u, _ in tree]
    t_list = [v for _, v in tree]
    # extra edges among near neighbours
    nn = _nearest(pos, 6)
    extra = spec.n_branch - (nb - 1)
    while extra > 0:
        u = int(rng.integers(0, nb))
        v = int(nn[u, int(rng.integers(0, 6))])
        if u == v:
            continue
        f_list.append(u)
        t_list.append(v)
        extra -= 1
    f = np.array(f_list, dtype=np.int64)
    t = np.array(t_list, dtype=np.int64)
    nbr = f.shape[0]
    # shuffle branch order so element numbering is not tree-first
    perm = rng.permutation(nbr)
    f, t = f[perm], t[perm]
    flip = rng.random(nbr) < 0.5
    f, t = np.where(flip, t, f), np.where(flip, f, t)
    r = rng.uniform(0.005, 0.05, nbr)
    x = r * rng.uniform(3.0, 10.0, nbr)
    b = rng.uniform(0.0, 0.05, nbr)
    is_tr = rng.random(nbr) < spec.transformer_share
    ratio = np.where(is_tr, rng.uniform(0.95, 1.05, nbr), 1.0)
    b = np.where(is_tr, 0.0, b)

    gen_bus = np.sort(rng.choice(nb, size=spec.n_gen, replace=False))
    load_bus = np.sort(rng.choice(nb, size=spec.n_load, replace=False))
    load_p = rng.lognormal(math.log(0.3), 0.6, spec.n_load)
    pf = rng.uniform(0.90, 0.98, spec.n_load)
    load_q = load_p * np.tan(np.arccos(pf))
    # dispatch: each load is served by its nearest generator (times a random weight), normalised to the total load,
    # so that the remaining imbalance is regional, as in a planned transmission grid
    from scipy.spatial import cKDTree
    _, near_gen = cKDTree(pos[gen_bus]).query(pos[load_bus], k=1)
    served = np.bincount(near_gen, weights=load_p, minlength=spec.n_gen)
    w = rng.uniform(0.8, 1.2, spec.n_gen)
    gen_p = np.maximum(served * w, 0.02)
    gen_p *= load_p.sum() / gen_p.sum()
    gen_vset = rng.uniform(0.98, 1.05, spec.n_gen)
    gen_pmax = gen_p / 0.8
    if spec.q_limits:
        u = rng.uniform(0.3, 0.6, spec.n_gen)
        gen_minq, gen_maxq = -u * gen_pmax, u * gen_pmax
    else:
        gen_minq = np.full(spec.n_gen, -np.inf)
        gen_maxq = np.full(spec.n_gen, np.inf)
    slack = int(gen_bus[int(np.argmax(gen_p))])

    is_gen = np.zeros(nb, dtype=bool)
    is_gen[gen_bus] = True
    pq_buses = np.flatnonzero(~is_gen)
    n_sh = int(round(spec.shunt_share * nb))
    shunt_bus = np.sort(rng.choice(pq_buses, size=min(n_sh, pq_buses.shape[0]), replace=False))
    shunt_g = rng.uniform(0.0, 0.002, shunt_bus.shape[0])
    shunt_b = rng.uniform(-0.05, 0.2, shunt_bus.shape[0])
    n_open = spec.open_branches
    open_bus = np.sort(rng.choice(pq_buses, size=n_open, replace=False)) if n_open else np.zeros(0, dtype=np.int64)
    open_side = rng.integers(1, 3, n_open)
    open_r = rng.uniform(0.005, 0.05, n_open)
    open_x = open_r * rng.uniform(3.0, 10.0, n_open)
    open_b = rng.uniform(0.0, 0.05, n_open)
    return Grid(spec, nb, f, t, r, x, b, ratio, is_tr, gen_bus, gen_p, gen_vset, gen_pmax, gen_minq, gen_maxq,
                load_bus, load_p, load_q, shunt_bus, shunt_g, shunt_b, open_bus, open_side, open_r, open_x, open_b,
                slack)


# ----------------------------------------------------------------------------------------------------------------
# Loading calibration: a compact polar Newton-Raphson on the base case (input preparation only).
# ----------------------------------------------------------------------------------------------------------------

def _branch_terms(vm1, va1, vm2, va2, y, ksi, g1, b1, g2, b2, r1):
    """p1 q1 p2 q2 and their derivatives wrt (ph1, v1, ph2, v2) for arrays of closed branches (A2 = 0, R2 = 1)."""
    th1 = ksi - va1 + va2
    th2 = ksi + va1 - va2
    sk, ck = np.sin(ksi), np.cos(ksi)
    s1, c1, s2, c2 = np.sin(th1), np.cos(th1), np.sin(th2), np.cos(th2)
    p1 = r1 * vm1 * (g1 * r1 * vm1 + y * r1 * vm1 * sk - y * vm2 * s1)
    q1 = r1 * vm1 * (-b1 * r1 * vm1 + y * r1 * vm1 * ck - y * vm2 * c1)
    p2 = vm2 * (g2 * vm2 - y * r1 * vm1 * s2 + y * vm2 * sk)
    q2 = vm2 * (-b2 * vm2 - y * r1 * vm1 * c2 + y * vm2 * ck)
    a = y * r1 * vm1 * vm2
    d = {
        "p1": (a * c1, r1 * (2 * g1 * r1 * vm1 + 2 * y * r1 * vm1 * sk - y * vm2 * s1), -a * c1, -y * r1 * vm1 * s1),
        "q1": (-a * s1, r1 * (-2 * b1 * r1 * vm1 + 2 * y * r1 * vm1 * ck - y * vm2 * c1), a * s1, -y * r1 * vm1 * c1),
        "p2": (-a * c2, -y * r1 * vm2 * s2, a * c2, 2 * g2 * vm2 - y * r1 * vm1 * s2 + 2 * y * vm2 * sk),
        "q2": (a * s2, -y * r1 * vm2 * c2, -a * s2, -2 * b2 * vm2 - y * r1 * vm1 * c2 + 2 * y * vm2 * ck),
    }
    return p1, q1, p2, q2, d


def _open_equivalent(g: Grid):
    """Shunt admittance an open-ended branch adds at its connected bus (series admittance into the far charging)."""
    ysk = 1.0 / (g.open_r + 1j * g.open_x)
    yo = 1j * g.open_b / 2
    return yo + ysk * yo / (ysk + yo)


def newton_polar(g: Grid, v0: Optional[np.ndarray] = None, th0: Optional[np.ndarray] = None,
                 max_iter: int = 30, tol: float = 1e-8, distributed: bool = False,
                 pq_gen: Optional[np.ndarray] = None, q_fixed: Optional[np.ndarray] = None):
    """Plain NR in the stable-row form (row 2b: P balance / slack angle, row 2b+1: Q balance / PV voltage).

    Returns (converged, iterations, vm, va), plus the generation factor lambda when ``distributed``: then every
    generator produces gen_p * (1 + lambda) and the slack bus's P balance is one more equation.  ``pq_gen`` marks
    generators that hold their reactive output at ``q_fixed`` instead of their voltage set point.  Used to calibrate
    the loading and the dispatch of the synthetic grids.
    """
    nb = g.n_bus
    n = 2 * nb
    y = 1.0 / np.hypot(g.r, g.x)
    ksi = np.arctan2(g.r, g.x)
    bh = g.b / 2
    f, t = g.f, g.t
    tgt = np.zeros(n)
    np.add.at(tgt, 2 * g.gen_bus, g.gen_p)
    np.add.at(tgt, 2 * g.load_bus, -g.load_p)
    np.add.at(tgt, 2 * g.load_bus + 1, -g.load_q)
    ident = np.zeros(n, dtype=bool)
    ident[2 * g.slack] = True
    pv = np.ones(g.gen_bus.shape[0], dtype=bool) if pq_gen is None else ~pq_gen
    ident[2 * g.gen_bus[pv] + 1] = True
    tgt[2 * g.slack] = 0.0
    tgt[2 * g.gen_bus[pv] + 1] = g.gen_vset[pv]
    if pq_gen is not None:
        np.add.at(tgt, 2 * g.gen_bus[pq_gen] + 1, q_fixed[pq_gen])
    ysh = np.zeros(nb, dtype=complex)
    np.add.at(ysh, g.shunt_bus, g.shunt_g + 1j * g.shunt_b)
    np.add.at(ysh, g.open_bus, _open_equivalent(g))
    gs, bs = ysh.real, ysh.imag
    x = np.zeros(n)
    x[1::2] = 1.0 if v0 is None else v0
    if th0 is not None:
        x[0::2] = th0
    x[ident] = tgt[ident]
    rows_b = np.stack([2 * f, 2 * f + 1, 2 * t, 2 * t + 1])          # p1 q1 p2 q2 rows
    cols_b = np.stack([2 * f, 2 * f + 1, 2 * t, 2 * t + 1])          # ph1 v1 ph2 v2 cols
    rr = np.repeat(rows_b, 4, axis=0).ravel()
    cc = np.tile(cols_b, (4, 1)).ravel()
    keep_b = ~ident[rr]
    idx_ident = np.flatnonzero(ident)
    best = np.inf
    lam = 0.0
    gen_rows = 2 * g.gen_bus
    slack_gen = int(np.flatnonzero(g.gen_bus == g.slack)[0])
    slack_load = float(np.sum(g.load_p[g.load_bus == g.slack]))

    def out(ok, it_):
        vm_, va_ = x[1::2].copy(), x[0::2].copy()
        return (ok, it_, vm_, va_, lam) if distributed else (ok, it_, vm_, va_)

    for it in range(max_iter + 1):
        va, vm = x[0::2], x[1::2]
        p1, q1, p2, q2, d = _branch_terms(vm[f], va[f], vm[t], va[t], y, ksi, 0.0, bh, 0.0, bh, g.ratio)
        fl = np.zeros(n)
        np.add.at(fl, 2 * f, p1)
        np.add.at(fl, 2 * f + 1, q1)
        np.add.at(fl, 2 * t, p2)
        np.add.at(fl, 2 * t + 1, q2)
        fl[0::2] += gs * vm * vm
        fl[1::2] += -bs * vm * vm
        F = fl - tgt
        if distributed:
            np.add.at(F, gen_rows, -lam * g.gen_p)
            f_slack = fl[2 * g.slack] - (g.gen_p[slack_gen] * (1 + lam) - slack_load)
        F[ident] = x[ident] - tgt[ident]
        nrm = np.max(np.abs(F))
        if distributed:
            nrm = max(nrm, abs(f_slack))
        if not np.isfinite(nrm) or nrm > 1e6 * max(best, 1.0):
            return out(False, it)
        best = min(best, nrm)
        if nrm < tol and it > 0:
            return out(True, it)
        if it == max_iter:
            return out(False, it)
        vals = np.concatenate([np.stack(d[k]).ravel() for k in ("p1", "q1", "p2", "q2")])
        jr = np.concatenate([rr[keep_b], 2 * np.arange(nb), 2 * np.arange(nb) + 1, idx_ident])
        jc = np.concatenate([cc[keep_b], 2 * np.arange(nb) + 1, 2 * np.arange(nb) + 1, idx_ident])
        sh_p = np.where(ident[0::2], 0.0, 2 * gs * vm)
        sh_q = np.where(ident[1::2], 0.0, -2 * bs * vm)
        jv = np.concatenate([vals[keep_b], sh_p, sh_q, np.ones(idx_ident.shape[0])])
        if distributed:
            # bordered system: extra column d F / d lambda (-gen_p on generator P rows), extra row = slack P balance
            keep_g = ~ident[gen_rows]
            srow = 2 * g.slack
            sl_r = np.flatnonzero(rr == srow)
            xr = np.concatenate([jr, gen_rows[keep_g], np.full(sl_r.shape[0], n), [n, n]])
            xc = np.concatenate([jc, np.full(int(keep_g.sum()), n), cc[sl_r], [2 * g.slack + 1, n]])
            xv = np.concatenate([jv, -g.gen_p[keep_g], vals[sl_r], [2 * gs[g.slack] * vm[g.slack],
                                                                  -g.gen_p[slack_gen]]])
            jac = sp.csc_matrix((xv, (xr, xc)), shape=(n + 1, n + 1))
            rhs = -np.concatenate([F, [f_slack]])
        else:
            jac = sp.csc_matrix((jv, (jr, jc)), shape=(n, n))
            rhs = -F
        try:
            dx = spla.splu(jac).solve(rhs)
        except RuntimeError:
            return out(False, it)
        if not np.all(np.isfinite(dx)):
            return out(False, it)
        x += dx[:n]
        if distributed:
            lam += dx[n]
    return out(False, max_iter)


def balanced(g: Grid, s: float, vm=None, va=None, max_iter: int = 20):
    """The grid at loading ``s`` with generator set points rescaled so that the slack only carries its share of the
    losses (a distributed-slack solve); None when that solve does not converge.  Returns (grid, vm, va)."""
    gs = g.scaled(s)
    res = newton_polar(gs, vm, va, max_iter=max_iter, distributed=True)
    ok, it, vm2, va2, lam = res
    if not ok:
        return None
    gb = dataclasses.replace(gs)
    gb.gen_p = gs.gen_p * (1 + lam)
    gb.base_vm, gb.base_va = vm2, va2
    return gb, vm2, va2


def solve_with_q_limits(g: Grid, max_outer: int = 12):
    """Base case with the generators' reactive limits: a generator whose reactive output leaves its limits holds it
    at the limit (PV -> PQ, no switching back).  Returns True when that converges.  Calibration helper only."""
    if g.base_vm is None:
        return False
    pq = np.zeros(g.gen_bus.shape[0], dtype=bool)
    qf = np.zeros(g.gen_bus.shape[0])
    vm, va = g.base_vm, g.base_va
    y = 1.0 / np.hypot(g.r, g.x)
    ksi = np.arctan2(g.r, g.x)
    bh = g.b / 2
    load_q_bus = np.zeros(g.n_bus)
    np.add.at(load_q_bus, g.load_bus, g.load_q)
    ysh = np.zeros(g.n_bus, dtype=complex)
    np.add.at(ysh, g.shunt_bus, g.shunt_g + 1j * g.shunt_b)
    np.add.at(ysh, g.open_bus, _open_equivalent(g))
    for _ in range(max_outer):
        ok, _, vm, va = newton_polar(g, vm, va, max_iter=30, pq_gen=pq, q_fixed=qf)
        if not ok:
            return False
        _, q1, _, q2, _ = _branch_terms(vm[g.f], va[g.f], vm[g.t], va[g.t], y, ksi, 0.0, bh, 0.0, bh, g.ratio)
        qinj = np.zeros(g.n_bus)
        np.add.at(qinj, g.f, q1)
        np.add.at(qinj, g.t, q2)
        qinj += -ysh.imag * vm * vm
        qgen = qinj[g.gen_bus] + load_q_bus[g.gen_bus]
        slack_gen = g.gen_bus == g.slack
        hi = ~pq & ~slack_gen & (qgen > g.gen_maxq)
        lo = ~pq & ~slack_gen & (qgen < g.gen_minq)
        if not (hi.any() or lo.any()):
            return True
        qf[hi], qf[lo] = g.gen_maxq[hi], g.gen_minq[lo]
        pq |= hi | lo
    return False


def calibrate(g: Grid) -> Grid:
    """The grid at the loading its spec asks for, loss-balanced.

    ``converge6``: the largest scale s <= 1 (bisection, 12 steps) at which the balanced base case converges from a
    flat start in at most 6 iterations.  ``collapse80``: 0.8 x the voltage-collapse scale, the largest scale at which
    a warm-started continuation of balanced solves still converges (growth by 25 % then bisection, 10 steps).
    """
    spec = g.spec
    if spec.loading == "converge6":
        def good(s):
            r = balanced(g, s)
            if r is None:
                return None
            ok, it, _, _ = newton_polar(r[0], max_iter=6)
            return r[0] if ok else None
        top = good(1.0)
        if top is not None:
            return top
        lo, lo_grid, hi = 0.0, None, 1.0
        for _ in range(12):
            mid = 0.5 * (lo + hi)
            r = good(mid)
            if r is not None:
                lo, lo_grid = mid, r
            else:
                hi = mid
        if lo_grid is None:
            raise RuntimeError(f"{spec.name}: no loading converges")
        return lo_grid
    lo, vm, va = 0.0, None, None
    s, hi = 0.05, None
    solved = []                                        # (scale, vm, va) of every converged balanced solve
    while hi is None:
        r = balanced(g, s, vm, va)
        if r is not None:
            lo, vm, va = s, r[1], r[2]
            solved.append((s, vm, va))
            s *= 1.25
            if s > 64:
                hi = s
        else:
            hi = s
    if not solved:
        raise RuntimeError(f"{spec.name}: no loading converges")
    for _ in range(10):
        mid = 0.5 * (lo + hi)
        r = balanced(g, mid, vm, va)
        if r is not None:
            lo, vm, va = mid, r[1], r[2]
            solved.append((mid, vm, va))
        else:
            hi = mid
    target = 0.8 * lo
    below = [e for e in solved if e[0] <= target]
    start = max(below, key=lambda e: e[0]) if below else (None, None, None)
    r = balanced(g, target, start[1], start[2])
    if r is None:
        r = balanced(g, target)
    if r is None:
        raise RuntimeError(f"{spec.name}: the calibrated loading does not converge")
    return r[0]


def _within_q_limits(g: Grid) -> Grid:
    """A grid with reactive limits backs its loading off by 5 % steps until its base case converges with the limits
    (the reactive-limit outer loop needs a feasible base case)."""
    cur = g
    for _ in range(30):
        if solve_with_q_limits(cur):
            return cur
        r = balanced(g, cur.scale / g.scale * 0.95, cur.base_vm, cur.base_va)
        if r is None:
            break
        cur = r[0]
    raise RuntimeError(f"{g.spec.name}: no loading converges within the reactive limits")


_CACHE = {}


def build(name: str, calibrate: bool = True) -> Grid:
    """Generate (and calibrate) the named grid; memoised per process."""
    key = (name, calibrate)
    if key not in _CACHE:
        g = generate(SPECS[name])
        if calibrate:
            g = globals()["calibrate"](g)
            if g.spec.q_limits:
                g = _within_q_limits(g)
        _CACHE[key] = g
    return _CACHE[key]


# ----------------------------------------------------------------------------------------------------------------
# Outage selection: single-branch, non-bridge, non-parallel (gen_contingencies.py:46-62 keeps unique-pair,
# non-islanding branches).
# ----------------------------------------------------------------------------------------------------------------

def bridges(nb: int, f: np.ndarray, t: np.ndarray) -> np.ndarray:
    """Boolean per branch: removing it disconnects the graph (iterative Tarjan on the multigraph)."""
    m = f.shape[0]
    adj_ptr = np.zeros(nb + 1, dtype=np.int64)
    np.add.at(adj_ptr, f + 1, 1)
    np.add.at(adj_ptr, t + 1, 1)
    adj_ptr = np.cumsum(adj_ptr)
    adj_to = np.empty(2 * m, dtype=np.int64)
    adj_e = np.empty(2 * m, dtype=np.int64)
    fill = adj_ptr[:-1].copy()
    for e in range(m):
        a, b = int(f[e]), int(t[e])
        adj_to[fill[a]] = b
        adj_e[fill[a]] = e
        fill[a] += 1
        adj_to[fill[b]] = a
        adj_e[fill[b]] = e
        fill[b] += 1
    disc = np.full(nb, -1, dtype=np.int64)
    low = np.zeros(nb, dtype=np.int64)
    is_bridge = np.zeros(m, dtype=bool)
    timer = 0
    for root in range(nb):
        if disc[root] >= 0:
            continue
        stack = [(root, -1, int(adj_ptr[root]))]
        disc[root] = low[root] = timer
        timer += 1
        while stack:
            u, pe, ptr = stack[-1]
            if ptr < adj_ptr[u + 1]:
                stack[-1] = (u, pe, ptr + 1)
                v, e = int(adj_to[ptr]), int(adj_e[ptr])
                if e == pe:
                    continue
                if disc[v] < 0:
                    disc[v] = low[v] = timer
                    timer += 1
                    stack.append((v, e, int(adj_ptr[v])))
                else:
                    low[u] = min(low[u], disc[v])
            else:
                stack.pop()
                if stack:
                    p = stack[-1][0]
                    low[p] = min(low[p], low[u])
                    if low[u] > disc[p]:
                        is_bridge[pe] = True
    return is_bridge


def outage_candidates(g: Grid) -> np.ndarray:
    """Branch indices whose single outage keeps the grid connected and that have no parallel twin."""
    br = bridges(g.n_bus, g.f, g.t)
    lo = np.minimum(g.f, g.t)
    hi = np.maximum(g.f, g.t)
    key = lo * g.n_bus + hi
    uniq, counts = np.unique(key, return_counts=True)
    par = np.isin(key, uniq[counts > 1])
    return np.flatnonzero(~br & ~par)


def draw_outages(g: Grid, count: Optional[int], seed: int, replace: bool = False) -> np.ndarray:
    """``count`` random candidates (all of them, in branch order, when ``count`` is None).  With ``replace`` the draw
    is with replacement, so a grid with fewer candidates than ``count`` still yields exactly ``count`` outages."""
    cand = outage_candidates(g)
    rng = np.random.default_rng(seed)
    if replace and count is not None:
        return np.sort(rng.choice(cand, size=count, replace=True))
    if count is None or count >= cand.shape[0]:
        return cand
    return np.sort(rng.choice(cand, size=count, replace=False))
