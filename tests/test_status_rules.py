"""Status rules of the Newton loop, engine against oracle on the same host inputs (needs a B200).

The rules follow the reference's batched Newton (newton_iteration.cu:276-397 with the linear-solve guard of :615-647,
state_vector_scaling.cu:53-97, realistic_voltage_check.cu:23-44); the oracle restates them in C.  Every failure here is
made on the host (an islanded bus, a tiny iteration budget, a voltage band): nothing faults the GPU.
"""
import numpy as np
import pytest

from conftest import grid
from test_gpu_engine import MIXED_STATE_TOL, STATE_TOL, _compare

pytestmark = pytest.mark.gpu


def _islanding_mask(p, g, bus):
    """Element flags that disable every closed branch at `bus` (the bus keeps its equations and loses its terms)."""
    m = np.zeros(p.n_elements, np.uint8)
    at = np.flatnonzero((g.f == bus) | (g.t == bus))
    m[at] = 1
    return m, at


def _pq_bus(p, g):
    # a PQ bus (both rows equations) with at least two branches
    for b in range(g.n_bus):
        deg = int(((g.f == b) | (g.t == b)).sum())
        if deg >= 2 and p.base_row_mode[2 * b] == 1 and p.base_row_mode[2 * b + 1] == 1:
            return b
    raise AssertionError("no PQ bus")


@pytest.mark.parametrize("schedule,lanes,threads", [(0, 2, 256), (4, 0, 256), (1, 2, 256)])
@pytest.mark.parametrize("precision", [0, 1])
def test_singular_lane_fails_alone(engine_lib, oracle_mod, schedule, lanes, threads, precision):
    """One scenario whose Jacobian is exactly singular (an islanded PQ bus: its angle column is zero) ends
    LINEAR_SOLVE_FAILED at the iteration that met the singular pivot, as the oracle's pivoting LU does; every other
    scenario is bit-identical to the same batch without it."""
    from olfgpu import native, synthetic
    g, p = grid("grid118")
    outs = synthetic.outage_candidates(g)[:12]
    dis = p.outage_masks(outs)
    bus = _pq_bus(p, g)
    bad, _ = _islanding_mask(p, g, bus)
    dis_bad = dis.copy()
    dis_bad[5] = bad
    s = native.Structure(p)
    ctx = native.BatchContext(s, dis.shape[0])
    ctx.set_linear_solver_settings(precision, 3)
    ctx.set_schedule(schedule, lanes, threads)
    clean = ctx.solve(p.x_base, p.target, p.base_row_mode, dis).copy()
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis_bad).copy()
    assert r[5, p.n + 2] == native.LINEAR_SOLVE_FAILED
    assert r[5, p.n] == 0                       # failed at the first factorization: no step taken
    keep = [k for k in range(dis.shape[0]) if k != 5]
    assert np.array_equal(r[keep], clean[keep])
    ref = oracle_mod.Structure(p).solve_batch(p.x_base, dis_bad)
    _compare(r, ref, p.n, MIXED_STATE_TOL if precision else STATE_TOL)
    assert r[5, p.n] == ref[5, p.n]
    assert np.all(np.isfinite(r[5, :p.n]))      # the failed lane's state stays finite (no garbage step)


@pytest.mark.parametrize("max_iter", [1, 2, 3])
@pytest.mark.parametrize("precision", [0, 1])
def test_iteration_budget_scoring_matches_oracle(engine_lib, oracle_mod, max_iter, precision):
    """Tiny budgets: the solve before the budget is scored (a sound one leaves MAX_ITERATION_REACHED), the second
    iteration of the first solve passes the linear-solve guard; statuses and iteration counts equal the oracle's."""
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 48, seed=501)
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    ctx = native.BatchContext(s, outs.shape[0])
    ctx.set_linear_solver_settings(precision, 3)
    r = ctx.solve(p.x_flat, p.target, p.base_row_mode, dis, max_iter=max_iter)
    ref = oracle_mod.Structure(p).solve_batch(p.x_flat, dis, max_iter=max_iter)
    assert np.array_equal(r[:, p.n + 2], ref[:, p.n + 2])
    assert np.array_equal(r[:, p.n], ref[:, p.n])
    assert np.all(r[:, p.n + 2] != native.REJECTED)


@pytest.mark.parametrize("eps", [1e-4, 1e-7])
@pytest.mark.parametrize("schedule,lanes", [(0, 2), (4, 0), (2, 0)])
def test_norm2_stopping_criterion_matches_oracle(engine_lib, oracle_mod, eps, schedule, lanes):
    """convEpsPerEq > 0: OLF's ||F||2 < sqrt(eps^2 n) decides convergence (newton_iteration.cu:105,241-250)."""
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 64, seed=502)
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    ctx = native.BatchContext(s, outs.shape[0])
    ctx.set_schedule(schedule, lanes, 512 if schedule == 2 else 256)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis, conv_eps_per_eq=eps)
    ref = oracle_mod.Structure(p).solve_batch(p.x_base, dis, conv_eps_per_eq=eps)
    _compare(r, ref, p.n)
    assert np.array_equal(r[:, p.n], ref[:, p.n])
    if eps == 1e-4:
        # the looser criterion stops earlier than the 1e-8 infinity-norm test on some scenario
        inf = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
        assert r[:, p.n].sum() < inf[:, p.n].sum()


def test_norm2_and_clamp_rejected_by_persistent_tiles(engine_lib):
    from olfgpu import native
    p = grid("grid118")[1]
    s = native.Structure(p)
    ctx = native.BatchContext(s, 2)
    ctx.set_schedule(native.PERSISTENT, 2, 256)
    dis = np.zeros((2, p.n_elements), np.uint8)
    with pytest.raises(native.NativeError, match="persistent"):
        ctx.solve(p.x_base, p.target, p.base_row_mode, dis, conv_eps_per_eq=1e-4)


@pytest.mark.parametrize("precision", [0, 1])
def test_max_voltage_change_matches_oracle(engine_lib, oracle_mod, precision):
    """MAX_VOLTAGE_CHANGE: each step scaled so max |dV| <= maxDv and max |dphi| <= maxDphi (the clamp binds from the
    flat start); statuses, iterations and states equal the oracle's."""
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 64, seed=503)
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    ctx = native.BatchContext(s, outs.shape[0])
    ctx.set_linear_solver_settings(precision, 3)
    kw = dict(svs_mode=native.SVS_MAX_VOLTAGE_CHANGE, max_dv=0.02, max_dphi=0.05, var_type=p.var_type)
    r = ctx.solve(p.x_flat, p.target, p.base_row_mode, dis, max_iter=30, **kw)
    ref = oracle_mod.Structure(p).solve_batch(p.x_flat, dis, max_iter=30, svs_mode=2, max_dv=0.02, max_dphi=0.05,
                                             var_type=p.var_type)
    _compare(r, ref, p.n, MIXED_STATE_TOL if precision else STATE_TOL)
    assert np.array_equal(r[:, p.n], ref[:, p.n])
    plain = ctx.solve(p.x_flat, p.target, p.base_row_mode, dis, max_iter=30)
    assert r[:, p.n].sum() > plain[:, p.n].sum()     # the clamp binds: more iterations than the plain step
    with pytest.raises(native.NativeError, match="varType"):
        ctx.solve(p.x_flat, p.target, p.base_row_mode, dis, svs_mode=native.SVS_MAX_VOLTAGE_CHANGE)
    with pytest.raises(native.NativeError, match="not supported"):
        ctx.solve(p.x_flat, p.target, p.base_row_mode, dis, svs_mode=native.SVS_LINE_SEARCH)


def test_realistic_voltage_band_matches_oracle(engine_lib, oracle_mod):
    """A converged state with a checked voltage outside the band is UNREALISTIC_STATE (status 2), its state kept."""
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 64, seed=504)
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    ctx = native.BatchContext(s, outs.shape[0])
    free = ctx.solve(p.x_base, p.target, p.base_row_mode, dis).copy()
    v = free[:, 1:p.n:2]
    # a band that the lowest voltages of some converged scenarios leave
    lo = float(np.quantile(v.min(axis=1), 0.5))
    rows = np.zeros(p.n, np.uint8)
    rows[1::2] = 1
    ctx.set_realistic_check(rows, lo, 2.0)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    ref = oracle_mod.Structure(p).solve_batch(p.x_base, dis, v_check=rows, min_v=lo, max_v=2.0)
    _compare(r, ref, p.n)
    assert 0 < int((r[:, p.n + 2] == native.UNREALISTIC_STATE).sum()) < outs.shape[0]
    unreal = r[:, p.n + 2] == native.UNREALISTIC_STATE
    assert np.array_equal(r[unreal, :p.n], free[unreal, :p.n])
    ctx.set_realistic_check(enabled=False)
    again = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    assert np.array_equal(again, free)


def test_unsupported_arguments_are_rejected_by_name(engine_lib):
    """The reference's solveBatchContext arguments this engine does not model fail loudly, naming the argument."""
    from olfgpu import native
    p = grid("grid118")[1]
    s = native.Structure(p)
    ctx = native.BatchContext(s, 2)
    dis = np.zeros((2, p.n_elements), np.uint8)
    for name in native.UNSUPPORTED_SOLVE_ARRAYS:
        with pytest.raises(native.NativeError, match=name):
            ctx.solve(p.x_base, p.target, p.base_row_mode, dis, unsupported={name: np.ones(3)})
    with pytest.raises(native.NativeError, match="pauseAtEnded"):
        ctx.solve(p.x_base, p.target, p.base_row_mode, dis, pause_at_ended=1)
    ok = ctx.solve(p.x_base, p.target, p.base_row_mode, dis, unsupported={n: np.zeros(0) for n in
                                                                          native.UNSUPPORTED_SOLVE_ARRAYS})
    assert np.all(ok[:, -1] == 0)


def test_skip_reactive_limits_phase(engine_lib, oracle_mod):
    """skipReactiveLimitsPhase: the context's reactive-limit entries stay installed but this solve runs without them."""
    from olfgpu import native, synthetic
    g, p = grid("grid300")
    outs = synthetic.draw_outages(g, 32, seed=505)
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    ctx = native.BatchContext(s, outs.shape[0], rl=p.rl)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis, skip_reactive_limits=True)
    _compare(r, oracle_mod.Structure(p).solve_batch(p.x_base, dis), p.n)
    r2 = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    _compare(r2, oracle_mod.Structure(p).solve_batch(p.x_base, dis, reactive_limits=True), p.n)
