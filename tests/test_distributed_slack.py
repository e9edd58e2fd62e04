"""Distributed-slack outer loop (bus level, static factors): after a scenario converges, the slack bus's closed-branch
P minus its target is water-filled over the participating buses' P targets in proportion to their factors, within
their bounds, and the scenario re-solves until the mismatch is within slackBusPMaxMismatch
(outerloop/distributed_slack.cu:211-616).  The engine's results match the oracle's restatement; GPU tests need a
B200."""
import dataclasses

import numpy as np
import pytest

from conftest import grid

STATE_TOL = 1e-8


def _compare(r, ref, n, tol=STATE_TOL):
    st_e, st_o = r[:, n + 2].astype(int), ref[:, n + 2].astype(int)
    assert np.array_equal(st_e, st_o), f"status mismatch at {np.flatnonzero(st_e != st_o)[:10]}"
    conv = st_o == 0
    if conv.any():
        assert np.max(np.abs(r[conv, :n] - ref[conv, :n])) <= tol
        assert np.array_equal(r[conv, n].astype(int), ref[conv, n].astype(int))


def _tight(ds, room):
    """The same participants with every bound cut to ``room`` pu of movement."""
    return dataclasses.replace(ds, max_delta=np.minimum(ds.max_delta, room), min_delta=np.maximum(ds.min_delta, -room))


def test_oracle_distribution_moves_states_and_rejects_when_bounded(oracle_mod):
    from olfgpu import packing, synthetic
    g, p = grid("grid118")
    ds = packing.distributed_slack(g, p)
    assert ds.row.size > 0 and np.all(ds.max_delta >= 0) and np.all(ds.min_delta <= 0)
    st = oracle_mod.Structure(p)
    outs = synthetic.outage_candidates(g)[:12]
    dis = p.outage_masks(outs)
    plain = st.solve_batch(p.x_base, dis)
    r = st.solve_batch(p.x_base, dis, distributed_slack=ds)
    n = p.n
    assert np.all(r[:, n + 2] == 0)
    assert np.max(np.abs(r[:, :n] - plain[:, :n])) > 1e-3     # the slack's share moved to the participants
    # bounds far below the mismatch: the distribution cannot place it; with the reject switch the scenario ends REJECTED
    tight = _tight(ds, 1e-5)
    kept = st.solve_batch(p.x_base, dis, distributed_slack=tight)
    rej = st.solve_batch(p.x_base, dis, distributed_slack=tight, reject_slack_distribution_failure=True)
    assert np.all(kept[:, n + 2] == 0)
    assert np.all(np.isin(rej[:, n + 2], (0, -2))) and np.count_nonzero(rej[:, n + 2] == -2) >= 6
    ok = rej[:, n + 2] == 0          # a scenario whose mismatch fit into the bounds is not rejected
    np.testing.assert_array_equal(rej[ok], kept[ok])


@pytest.mark.gpu
@pytest.mark.parametrize("name,count", [("grid118", 60), ("grid2000", 120)])
@pytest.mark.parametrize("precision,schedule", [(0, 0), (0, 4), (1, 4)])
def test_distributed_slack_matches_oracle(engine_lib, oracle_mod, name, count, precision, schedule):
    from olfgpu import native, packing, synthetic
    g, p = grid(name)
    ds = packing.distributed_slack(g, p)
    outs = synthetic.draw_outages(g, count, seed=77)
    dis = p.outage_masks(outs)
    s = native.Structure(p, native.PLAN_DENSE_FRONT if schedule == 4 else native.MIN_DEGREE)
    ctx = native.BatchContext(s, outs.shape[0], ds=ds)
    ctx.set_linear_solver_settings(precision, 3)
    ctx.set_schedule(schedule, 0, 256)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    ref = oracle_mod.Structure(p).solve_batch(p.x_base, dis, distributed_slack=ds)
    _compare(r, ref, p.n)
    assert not ctx.last_slack_distribution_failures().any()
    # the outer loop can be switched off for a solve (DriverNative.setBatchOuterLoops)
    ctx.set_outer_loops(distributed_slack=False, reactive_limits=True)
    r0 = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    _compare(r0, oracle_mod.Structure(p).solve_batch(p.x_base, dis), p.n)


@pytest.mark.gpu
def test_distributed_slack_with_reactive_limits_matches_oracle(engine_lib, oracle_mod):
    """Both outer loops: the distribution first, then the PV->PQ check, as the reference's outer-loop order."""
    from olfgpu import native, packing, synthetic
    g, p = grid("grid300")
    assert p.rl is not None
    ds = packing.distributed_slack(g, p)
    outs = synthetic.draw_outages(g, 100, seed=301)
    dis = p.outage_masks(outs)
    ctx = native.BatchContext(native.Structure(p), outs.shape[0], rl=p.rl, ds=ds)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    ref = oracle_mod.Structure(p).solve_batch(p.x_base, dis, reactive_limits=True, distributed_slack=ds)
    _compare(r, ref, p.n)


@pytest.mark.gpu
def test_distribution_failure_flags_and_reject(engine_lib, oracle_mod):
    from olfgpu import native, packing, synthetic
    g, p = grid("grid2000")
    ds = _tight(packing.distributed_slack(g, p), 1e-6)
    outs = synthetic.draw_outages(g, 64, seed=78)
    dis = p.outage_masks(outs)
    ctx = native.BatchContext(native.Structure(p), outs.shape[0], ds=ds)
    st = oracle_mod.Structure(p)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    _compare(r, st.solve_batch(p.x_base, dis, distributed_slack=ds), p.n)
    assert ctx.last_slack_distribution_failures().any()
    rej = ctx.solve(p.x_base, p.target, p.base_row_mode, dis, reject_slack_distribution_failure=True)
    ref = st.solve_batch(p.x_base, dis, distributed_slack=ds, reject_slack_distribution_failure=True)
    _compare(rej, ref, p.n)
    assert np.any(rej[:, p.n + 2] == -2)


@pytest.mark.gpu
def test_distributed_slack_needs_a_level_schedule(engine_lib):
    """The persistent-tile schedule has no distributed-slack loop: the solve is refused, not run without it."""
    from olfgpu import native, packing, synthetic
    g, p = grid("grid118")
    outs = synthetic.draw_outages(g, 8, seed=1)
    ctx = native.BatchContext(native.Structure(p), outs.shape[0], ds=packing.distributed_slack(g, p))
    ctx.set_schedule(native.PERSISTENT, 2, 256)
    with pytest.raises(RuntimeError):
        ctx.solve(p.x_base, p.target, p.base_row_mode, p.outage_masks(outs))
