"""Device violation screening after an N-1 solve (sa/olf_gpu_violations.cu:160-361) against the oracle's restatement
on the same states (needs a B200).  Thresholds are drawn away from the values (a margin far above the last-bit
differences of device and host arithmetic), so both screens must return the same candidate sets."""
import numpy as np
import pytest

from conftest import grid

pytestmark = pytest.mark.gpu


def _tables(p, rng, n_elem):
    """Limited elements (closed branches, and the open-ended ones when the grid has some), two groups each (side 1
    current with three thresholds, side 2 apparent power with two; an open-ended branch only its connected side)."""
    elems = list(rng.choice(p.n_cb, size=n_elem, replace=False)) + [p.n_cb + e for e in range(p.n_ob)]
    gptr, side, qty, lptr = [0], [], [], [0]
    for e in elems:
        sides = [1, 2]
        if e >= p.n_cb:
            sides = [1] if p.ob_idx[e - p.n_cb][4] >= 0 else [2]
        for sd in sides:
            side.append(sd)
            qty.append(0 if sd == 1 else 2)
            lptr.append(lptr[-1] + (3 if sd == 1 else 2))
        gptr.append(len(side))
    return np.array(elems), np.array(gptr), np.array(side), np.array(qty), np.array(lptr)


def test_screen_matches_oracle(engine_lib, oracle_mod):
    from olfgpu import native, synthetic
    g, p = grid("grid118")
    outs = synthetic.outage_candidates(g)[:40]
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    ctx = native.BatchContext(s, outs.shape[0])
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    x = r[:, :p.n]
    rng = np.random.default_rng(7)
    elems, gptr, side, qty, lptr = _tables(p, rng, 60)
    # thresholds from the base-case values: descending within a group, some below the contingency values
    vals = []
    oracle_mod.screen_violations(p, x, dis, elems, gptr, side, qty, lptr, np.full(lptr[-1], np.inf), [], [], [],
                                 values=vals)
    base = np.zeros(lptr[-1])
    for s_, l, v, t in vals:
        base[l] = max(base[l], v)
    thr = base * rng.uniform(0.85, 1.1, base.shape)
    bus_vrow = np.arange(1, p.n, 2, dtype=np.int32)
    high = np.full(p.n_bus, 1.05)
    low = np.full(p.n_bus, 0.97)
    low[::7] = np.nan
    # keep every comparison value clear of its threshold (relative 1e-6, far above device / host rounding)
    vals = []
    oracle_mod.screen_violations(p, x, dis, elems, gptr, side, qty, lptr, thr, [], [], [], values=vals)
    for s_, l, v, t in vals:
        if abs(v - t) <= 1e-6 * abs(t):
            thr[l] *= 1.001
    got, cnt = ctx.screen_violations(elems, gptr, side, qty, lptr, thr, bus_vrow, high, low, realistic=True,
                                     min_v=0.95, max_v=1.06, capacity=256)
    ref = oracle_mod.screen_violations(p, x, dis, elems, gptr, side, qty, lptr, thr, bus_vrow, high, low,
                                       realistic=True, min_v=0.95, max_v=1.06)
    assert [list(map(int, a)) for a in got] == ref
    assert sum(len(a) for a in ref) > 0                # the limits bind somewhere
    # an outaged branch yields nothing in its scenario
    k = int(np.flatnonzero(np.isin(elems, outs))[0]) if np.isin(elems, outs).any() else None
    if k is not None:
        e = elems[k]
        sc = int(np.flatnonzero(outs == e)[0])
        assert not any(lptr[gptr[k]] <= rid < lptr[gptr[k + 1]] for rid in got[sc])
    # a small capacity truncates and reports the full count
    got2, cnt2 = ctx.screen_violations(elems, gptr, side, qty, lptr, thr, bus_vrow, high, low, capacity=1)
    assert np.array_equal(cnt2, [len(a) for a in oracle_mod.screen_violations(
        p, x, dis, elems, gptr, side, qty, lptr, thr, bus_vrow, high, low)])
