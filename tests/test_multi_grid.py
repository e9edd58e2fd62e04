"""Uneven batching: outages of several grids through one persistent launch, against the oracle (needs a B200)."""
import numpy as np
import pytest

from conftest import grid

pytestmark = pytest.mark.gpu

STATE_TOL = 1e-8


def _compare(r, ref, n):
    st = ref[:, n + 2].astype(int)
    assert np.array_equal(r.status, st), f"status mismatch at {np.flatnonzero(r.status != st)[:10]}"
    conv = st == 0
    if conv.any():
        d = np.max(np.abs(r.x[conv] - ref[conv, :n]))
        assert d <= STATE_TOL, d


@pytest.mark.parametrize("precision", [0, 1])
def test_multi_grid_matches_oracle(engine_lib, oracle_mod, precision):
    """Three grids of different sizes (two with reactive limits) in one launch give each grid's oracle result."""
    from olfgpu import synthetic
    from olfgpu.security_analysis import MultiGridAnalysis
    names, counts = ["grid300", "grid2000q", "grid118"], [70, 45, 20]
    packs = [grid(nm)[1] for nm in names]
    outs = [synthetic.draw_outages(grid(nm)[0], c, seed=40 + i) for i, (nm, c) in enumerate(zip(names, counts))]
    ma = MultiGridAnalysis(packs, counts, precision=precision, schedule=(2, 256, 0))
    res, ms = ma.solve(outs)
    assert ms > 0
    for p, o, r in zip(packs, outs, res):
        ref = oracle_mod.Structure(p).solve_batch(p.x_base, p.outage_masks(o), reactive_limits=p.rl is not None)
        _compare(r, ref, p.n)
    # a second solve on the same contexts (graph replay) gives the same answers
    res2, _ = ma.solve(outs)
    for a, b in zip(res, res2):
        assert np.array_equal(a.status, b.status) and np.array_equal(a.x, b.x)
    ma.close()


def test_multi_grid_autotuner_and_orders(engine_lib, oracle_mod):
    """The autotuner times the members' device-resident loops and 16 tile schedules (lanes 1-8 x 256/512 threads x two
    member orders) and keeps the fastest; every fixed schedule gives the oracle's statuses and states within
    tolerance."""
    from olfgpu import synthetic
    from olfgpu.security_analysis import MultiGridAnalysis
    names, counts = ["grid2000q", "grid300"], [40, 33]
    packs = [grid(nm)[1] for nm in names]
    outs = [synthetic.draw_outages(grid(nm)[0], c, seed=60 + i) for i, (nm, c) in enumerate(zip(names, counts))]
    ma = MultiGridAnalysis(packs, counts, schedule=-1)
    tuned, _ = ma.solve(outs)
    pick, timings = ma.multi.schedule()
    assert len(timings) == 17 and timings[0][0] == 0
    best = min(timings, key=lambda t: t[3])
    assert pick == (int(best[0]), int(best[1]), int(best[2]))
    refs = [oracle_mod.Structure(p).solve_batch(p.x_base, p.outage_masks(o), reactive_limits=True)
            for p, o in zip(packs, outs)]
    for sched in [(0, 0, 0), (1, 512, 1), (4, 256, 0), (8, 512, 1)]:
        ma.multi.set_schedule(*sched)
        res, _ = ma.solve(outs)
        for p, r, ref in zip(packs, res, refs):
            _compare(r, ref, p.n)
    for p, r, ref in zip(packs, tuned, refs):
        _compare(r, ref, p.n)
    ma.close()


def test_multi_grid_rejects_bad_members(engine_lib):
    from olfgpu import native
    p1, p2 = grid("grid118")[1], grid("grid300")[1]
    s1, s2 = native.Structure(p1), native.Structure(p2)
    c1, c2 = native.BatchContext(s1, 4), native.BatchContext(s2, 4)
    c2.set_linear_solver_settings(native.MIXED, 1)
    m = native.MultiContext([c1, c2])
    with pytest.raises(native.NativeError, match="staged"):
        m.solve()
    c1.stage(p1.x_base, p1.target, p1.base_row_mode, np.zeros((4, p1.n_elements), np.uint8))
    c2.stage(p2.x_base, p2.target, p2.base_row_mode, np.zeros((4, p2.n_elements), np.uint8))
    with pytest.raises(native.NativeError, match="precision"):
        m.solve()
    with pytest.raises(native.NativeError, match="twice"):
        native.MultiContext([c1, c1])


def test_uneven_batch_four_grids_full_size(engine_lib, oracle_mod):
    """300 / 2,000 / 9,241 / 13,659 buses with 1,000 / 1,000 / 500 / 250 outages and reactive limits in one launch;
    a sample of every grid's scenarios checked against the oracle."""
    from olfgpu import synthetic
    from olfgpu.security_analysis import MultiGridAnalysis
    names, counts = ["grid300", "grid2000q", "grid9241q", "grid13659"], [1000, 1000, 500, 250]
    gs = [grid(nm) for nm in names]
    packs = [gp[1] for gp in gs]
    outs = [synthetic.draw_outages(gp[0], c, seed=3000 + i, replace=True) for i, (gp, c) in enumerate(zip(gs, counts))]
    ma = MultiGridAnalysis(packs, counts, schedule=(2, 256, 1))
    res, ms = ma.solve(outs)
    for p, o, r in zip(packs, outs, res):
        pick = np.arange(0, o.shape[0], max(1, o.shape[0] // 12))
        ref = oracle_mod.Structure(p).solve_batch(p.x_base, p.outage_masks(o[pick]), reactive_limits=True)
        st = ref[:, p.n + 2].astype(int)
        assert np.array_equal(r.status[pick], st)
        conv = st == 0
        assert np.max(np.abs(r.x[pick][conv] - ref[conv, :p.n])) <= STATE_TOL
    ma.close()


@pytest.mark.parametrize("precision,policy", [(0, 0), (1, 0), (1, 1)])
def test_multi_grid_device_loops_match_solo_solves(engine_lib, oracle_mod, precision, policy):
    """lanesPerTile 0: one graph whose branches are the grids' own device-resident Newton loops (dense-front plans,
    shared-memory level schedule, reactive limits) gives every grid exactly its solo solve, and the oracle's result."""
    from olfgpu import native, synthetic
    from olfgpu.security_analysis import MultiGridAnalysis
    names, counts = ["grid300", "grid2000q", "grid9241"], [90, 60, 40]
    packs = [grid(nm)[1] for nm in names]
    outs = [synthetic.draw_outages(grid(nm)[0], c, seed=80 + i) for i, (nm, c) in enumerate(zip(names, counts))]
    ma = MultiGridAnalysis(packs, counts, precision=precision, refinement_steps=3, schedule=(0, 0, 0),
                           ordering=native.PLAN_DENSE_FRONT, member_schedule=(4, 0, 256), mixed_policy=policy)
    res, ms = ma.solve(outs)
    assert ms > 0
    for p, o, r in zip(packs, outs, res):
        s = native.Structure(p, native.PLAN_DENSE_FRONT)
        c = native.BatchContext(s, o.shape[0], native.BATCHED_LU, p.rl)
        c.set_linear_solver_settings(precision, 3)
        c.set_mixed_precision_policy(policy)
        c.set_schedule(4, 0, 256)
        solo = c.solve(p.x_base, p.target, p.base_row_mode, p.outage_masks(o))
        assert np.array_equal(r.x, solo[:, :p.n]) and np.array_equal(r.status, solo[:, p.n + 2].astype(int))
        assert np.array_equal(r.iterations, solo[:, p.n].astype(int))
        ref = oracle_mod.Structure(p).solve_batch(p.x_base, p.outage_masks(o), reactive_limits=p.rl is not None)
        _compare(r, ref, p.n)
    ma.close()
