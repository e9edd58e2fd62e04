"""Parity of the CUDA engine with the oracle, through the C ABI (needs a B200)."""
import numpy as np
import pytest

from conftest import grid, oracle_rows

pytestmark = pytest.mark.gpu

# converged states must agree within 1e-8 pu / rad, statuses exactly
STATE_TOL = 1e-8
# mixed precision against the FP64 oracle: the same bar.  A scenario near convergence refines its FP32 solve until the
# correction is below 1e-11, so its last Newton step is FP64-accurate; a scenario whose mixed-precision solve fails
# restarts in FP64 and fails as the FP64 engine does
MIXED_STATE_TOL = 1e-8
# mixed precision with refinement switched off (refineBelow below any mismatch): the last step keeps its FP32 error
UNREFINED_STATE_TOL = 1e-6


def _tol(precision):
    return MIXED_STATE_TOL if precision == 1 else STATE_TOL


def _perturbed_states(p, ns, seed, scale=0.05):
    rng = np.random.default_rng(seed)
    x0 = p.x_base if p.x_base is not None else p.x_flat
    x = np.tile(x0, (ns, 1))
    x[:, 0::2] += rng.uniform(-scale, scale, (ns, p.n_bus))
    x[:, 1::2] += rng.uniform(-scale, scale, (ns, p.n_bus))
    return x


@pytest.mark.parametrize("name", ["grid118", "grid2000"])
def test_fill_matches_oracle(engine_lib, oracle_mod, name):
    from olfgpu import native, synthetic
    g, p = grid(name)
    ns = 40
    s = native.Structure(p)
    ctx = native.BatchContext(s, ns)
    x = _perturbed_states(p, ns, 1)
    outs = synthetic.draw_outages(g, ns, seed=7)
    dis = p.outage_masks(outs)
    J, F = ctx.debug_fill(x, p.target, p.base_row_mode, dis)
    st = oracle_mod.Structure(p)
    for k in range(ns):
        Jo, Fo = st.fill(x[k], p.target, p.base_row_mode, dis[k])
        scale = np.maximum(np.abs(Jo), 1.0)
        assert np.max(np.abs(J[k] - Jo) / scale) < 1e-12
        assert np.max(np.abs(F[k] - Fo)) < 1e-10


@pytest.mark.parametrize("precision,tol", [(0, 1e-9), (1, 2e-3)])
def test_linear_solve_matches_oracle(engine_lib, oracle_mod, precision, tol):
    from olfgpu import native
    g, p = grid("grid2000")
    ns = 36
    s = native.Structure(p)
    ctx = native.BatchContext(s, ns)
    x = _perturbed_states(p, ns, 2, 0.02)
    st = oracle_mod.Structure(p)
    zero = np.zeros(p.n_elements, np.uint8)
    J = np.stack([st.fill(x[k], p.target, p.base_row_mode, zero)[0] for k in range(ns)])
    rng = np.random.default_rng(3)
    rhs = rng.standard_normal((ns, p.n))
    z = ctx.debug_linear_solve(J, rhs, precision)
    for k in range(ns):
        zo = st.linear_solve(J[k], rhs[k])
        assert np.max(np.abs(z[k] - zo)) / np.max(np.abs(zo)) < tol


def _compare(res, ref, n, tol=STATE_TOL):
    st_e = res[:, n + 2].astype(int)
    st_o = ref[:, n + 2].astype(int)
    assert np.array_equal(st_e, st_o), f"status mismatch at {np.flatnonzero(st_e != st_o)[:10]}"
    conv = st_o == 0
    if conv.any():
        d = np.max(np.abs(res[conv, :n] - ref[conv, :n]))
        assert d <= tol, d
    return st_o


@pytest.mark.parametrize("name,count", [("grid118", None), ("grid2000", 600)])
def test_n1_fp64_matches_oracle(engine_lib, oracle_mod, name, count):
    from olfgpu import native, synthetic
    from olfgpu.security_analysis import SecurityAnalysis
    g, p = grid(name)
    outs = synthetic.draw_outages(g, count, seed=11)
    sa = SecurityAnalysis(p, precision=native.FP64)
    r = sa.solve_n1(outs)
    st = oracle_mod.Structure(p)
    ref = st.solve_batch(p.x_base, p.outage_masks(outs))
    out = np.concatenate([r.x, r.iterations[:, None], r.norm[:, None], r.status[:, None]], axis=1)
    status = _compare(out, ref, p.n)
    assert (status == 0).mean() > 0.9
    assert np.array_equal(r.iterations[status == 0], ref[status == 0, p.n].astype(int))


@pytest.mark.parametrize("name", ["grid118", "grid300"])
def test_engine_matches_reference_component_newton(engine_lib, name):
    """The engine against the committed Newton solves made only of the reference's own code (tests/golden/
    newton_<grid>.npz: its generated formulas, its scatter map, its host LU), with no oracle in between: the base case
    from a flat start as a batch of one, and 24 N-1 outages from the base-case start as one batch."""
    import os
    from olfgpu import native
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", f"newton_{name}.npz"))
    g, p = grid(name)
    for k in ("cb_params", "cb_idx", "ob_params", "ob_idx", "sh_params", "sh_idx", "target", "base_row_mode"):
        assert np.array_equal(getattr(p, k), d[k]), f"the synthetic grid no longer matches the fixture ({k})"
    s = native.Structure(p)
    ref = d["ref_rows"]
    dis = d["disabled"]
    base = native.BatchContext(s, 1)
    base.set_linear_solver_settings(native.FP64, 1)
    out0 = base.solve(d["x0"][0], p.target, p.base_row_mode, dis[:1])
    n1 = native.BatchContext(s, dis.shape[0] - 1)
    n1.set_linear_solver_settings(native.FP64, 1)
    out1 = n1.solve(p.x_base, p.target, p.base_row_mode, dis[1:])
    out = np.concatenate([out0, out1])
    _compare(out, ref, p.n)
    assert np.array_equal(out[:, p.n], ref[:, p.n]), "iteration counts differ"


def test_n1_9241_subset_matches_oracle(engine_lib, oracle_mod):
    from olfgpu import native, synthetic
    from olfgpu.security_analysis import SecurityAnalysis
    g, p = grid("grid9241")
    outs = synthetic.draw_outages(g, 500, seed=9241)[:48]
    sa = SecurityAnalysis(p, precision=native.FP64)
    r = sa.solve_n1(outs)
    ref = oracle_mod.Structure(p).solve_batch(p.x_base, p.outage_masks(outs))
    out = np.concatenate([r.x, r.iterations[:, None], r.norm[:, None], r.status[:, None]], axis=1)
    _compare(out, ref, p.n)


@pytest.mark.parametrize("steps", [1, 2])
def test_n1_mixed_precision_matches_fp64_oracle(engine_lib, oracle_mod, steps):
    from olfgpu import native, synthetic
    from olfgpu.security_analysis import SecurityAnalysis
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 300, seed=12)
    sa = SecurityAnalysis(p, precision=native.MIXED, refinement_steps=steps)
    r = sa.solve_n1(outs)
    ref = oracle_mod.Structure(p).solve_batch(p.x_base, p.outage_masks(outs))
    out = np.concatenate([r.x, r.iterations[:, None], r.norm[:, None], r.status[:, None]], axis=1)
    _compare(out, ref, p.n, MIXED_STATE_TOL)


def test_replicated_scenarios_equal_single_solve(engine_lib):
    """GpuBatchedN1Test.java:80-131: K identical scenarios match the single solve to 1e-12."""
    from olfgpu import native
    g, p = grid("grid118")
    s = native.Structure(p)
    one = native.BatchContext(s, 1).solve(p.x_flat, p.target, p.base_row_mode, np.zeros((1, p.n_elements), np.uint8))
    many = native.BatchContext(s, 8).solve(p.x_flat, p.target, p.base_row_mode, np.zeros((8, p.n_elements), np.uint8))
    assert one[0, -1] == 0
    assert np.max(np.abs(many - one[0])) <= 1e-12


def test_disabled_mask_changes_result(engine_lib):
    """GpuBatchedN1Test.java:134-183: a scenario with a disabled branch differs from the base."""
    from olfgpu import native, synthetic
    g, p = grid("grid118")
    s = native.Structure(p)
    outs = synthetic.outage_candidates(g)[:2]
    dis = np.zeros((3, p.n_elements), np.uint8)
    dis[1, outs[0]] = 1
    dis[2, outs[1]] = 1
    r = native.BatchContext(s, 3).solve(p.x_base, p.target, p.base_row_mode, dis)
    assert np.all(r[:, -1] == 0)
    assert np.max(np.abs(r[1, :p.n] - r[0, :p.n])) > 1e-6
    assert np.max(np.abs(r[2, :p.n] - r[0, :p.n])) > 1e-6


def test_nan_lane_diverges_alone(engine_lib):
    """A non-finite mismatch retires only its lane (newton_iteration.cu:344-351); the others are bit-identical."""
    from olfgpu import native, synthetic
    g, p = grid("grid118")
    s = native.Structure(p)
    outs = synthetic.outage_candidates(g)[:5]
    dis = p.outage_masks(outs)
    ctx = native.BatchContext(s, 5)
    clean = ctx.solve(p.x_base, p.target, p.base_row_mode, dis).copy()
    row = int(np.flatnonzero(p.base_row_mode == 1)[0])
    bad = ctx.solve(p.x_base, p.target, p.base_row_mode, dis, target_override_index=np.array([2 * p.n + row]),
                    target_override_value=np.array([np.nan]))
    assert bad[2, -1] == native.DIVERGED
    keep = [0, 1, 3, 4]
    assert np.array_equal(bad[keep], clean[keep])


def test_iteration_budget_statuses(engine_lib, oracle_mod):
    from olfgpu import native
    g, p = grid("grid118")
    s = native.Structure(p)
    dis = np.zeros((1, p.n_elements), np.uint8)
    ctx = native.BatchContext(s, 1)
    full = ctx.solve(p.x_flat, p.target, p.base_row_mode, dis)
    it = int(full[0, -3])
    for budget in (1, it - 1, it, it + 1):
        e = ctx.solve(p.x_flat, p.target, p.base_row_mode, dis, max_iter=budget)
        o = oracle_mod.Structure(p).solve_batch(p.x_flat, dis, max_iter=budget)
        assert e[0, -1] == o[0, -1], budget
        assert e[0, -3] == o[0, -3], budget


# the state after k fixed Newton steps: the engine's block LU and the oracle's sparse LU round differently (measured
# ~1e-14 between the oracle's LU and the reference's own host LU on these grids); the mismatch norm at its rounding floor
# near convergence is compared with an absolute floor
TRAJECTORY_TOL = 1e-9


@pytest.mark.parametrize("name,start,count,steps", [("grid118", "flat", 16, 5), ("grid2000", "base", 48, 3),
                                                    ("grid9241", "base", 16, 3)])
def test_fixed_iteration_trajectories_match_oracle(engine_lib, oracle_mod, name, start, count, steps):
    """The design of the reference's GPU-vs-CPU fixed-iteration test: from the same start, a budget of k Newton
    iterations stops every lane still iterating with MAX_ITERATION_REACHED at its k-th state, which must equal the
    oracle's after k steps, with the same mismatch norm, for k = 1 .. steps (converged lanes as usual)."""
    from olfgpu import native, synthetic
    g, p = grid(name)
    x0 = p.x_flat if start == "flat" else p.x_base
    outs = synthetic.draw_outages(g, count, seed=41)
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    st = oracle_mod.Structure(p)
    n = p.n
    for k in range(1, steps + 1):
        e = native.BatchContext(s, count).solve(x0, p.target, p.base_row_mode, dis, max_iter=k)
        o = st.solve_batch(x0, dis, max_iter=k)
        assert np.array_equal(e[:, n + 2], o[:, n + 2]), k
        assert np.array_equal(e[:, n], o[:, n]), k
        assert np.max(np.abs(e[:, :n] - o[:, :n])) <= TRAJECTORY_TOL, k
        assert np.all(np.abs(e[:, n + 1] - o[:, n + 1]) <= 1e-10 + 1e-6 * np.abs(o[:, n + 1])), k


def test_per_scenario_start_and_ragged_batch(engine_lib, oracle_mod):
    from olfgpu import native, synthetic
    g, p = grid("grid118")
    s = native.Structure(p)
    ns = 37
    outs = synthetic.outage_candidates(g)[:ns]
    dis = p.outage_masks(outs)
    x0 = _perturbed_states(p, ns, 5, 0.01)
    r = native.BatchContext(s, ns).solve(None, p.target, p.base_row_mode, dis, x0_full=x0)
    ref = oracle_mod.Structure(p).solve_batch(x0, dis)
    _compare(r, ref, p.n)


def test_row_mode_entries_switch_a_pv_bus(engine_lib, oracle_mod):
    from olfgpu import native
    g, p = grid("grid118")
    s = native.Structure(p)
    pv_rows = np.flatnonzero((p.base_row_mode == 0) & (np.arange(p.n) % 2 == 1))
    row = int(pv_rows[1])
    ns = 2
    dis = np.zeros((ns, p.n_elements), np.uint8)
    r = native.BatchContext(s, ns).solve(p.x_base, p.target, p.base_row_mode, dis,
                                          row_mode_entries=np.array([[1, row, 1]]),
                                          target_override_index=np.array([1 * p.n + row]),
                                          target_override_value=np.array([0.05]))
    mode = p.base_row_mode.copy()
    mode[row] = 1
    t = p.target.copy()
    t[row] = 0.05
    ref = oracle_mod.Structure(p).solve_batch(p.x_base, dis[1:], target=t, mode=mode)
    _compare(r[1:], ref, p.n)


def test_reactive_limits_match_oracle(engine_lib, oracle_mod):
    from olfgpu import native, synthetic
    from olfgpu.security_analysis import SecurityAnalysis
    g, p = grid("grid300")
    outs = synthetic.draw_outages(g, 120, seed=300)
    sa = SecurityAnalysis(p, precision=native.FP64, reactive_limits=True)
    r = sa.solve_n1(outs)
    ref = oracle_mod.Structure(p).solve_batch(p.x_base, p.outage_masks(outs), reactive_limits=True)
    out = np.concatenate([r.x, r.iterations[:, None], r.norm[:, None], r.status[:, None]], axis=1)
    _compare(out, ref, p.n)
    # the limits actually bind somewhere
    plain = oracle_mod.Structure(p).solve_batch(p.x_base, p.outage_masks(outs))
    assert np.max(np.abs(plain[:, :p.n] - ref[:, :p.n])) > 1e-4


def test_final_targets_and_row_modes_match_oracle(engine_lib, oracle_mod):
    """BatchReadbackNative.readBatchTargets / readBatchRowModes: after a solve with the reactive-limit outer loop, the
    targets and row modes each converged scenario ended with equal the oracle's (its PV rows switched to PQ at a Q
    limit), every changed row is a reactive-limit voltage row, and a chosen slot list comes back in its order."""
    from olfgpu import native, synthetic
    g, p = grid("grid300")
    outs = synthetic.draw_outages(g, 40, seed=303)
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    ctx = native.BatchContext(s, outs.shape[0], rl=p.rl)
    res = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    ref, tg, md = oracle_mod.Structure(p).solve_batch(p.x_base, dis, reactive_limits=True, final_equations=True)
    _compare(res, ref, p.n)
    targets, modes = ctx.read_targets(), ctx.read_row_modes()
    conv = ref[:, p.n + 2] == 0
    assert np.array_equal(modes[conv], md[conv])
    assert np.max(np.abs(targets[conv] - tg[conv])) <= 1e-12
    changed = (modes != p.base_row_mode) | (targets != p.target)
    assert changed.any(), "the limits bind"
    assert set(np.flatnonzero(changed.any(axis=0)).tolist()) <= set(p.rl.voltage_row.tolist())
    slots = np.array([5, 0, 17], np.int32)
    assert np.array_equal(ctx.read_row_modes(slots), modes[slots])
    assert np.array_equal(ctx.read_targets(slots), targets[slots])
    # without the outer loop the installed equations come back unchanged
    ctx.set_outer_loops(reactive_limits=False)
    ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    assert np.array_equal(ctx.read_row_modes(), np.tile(p.base_row_mode, (outs.shape[0], 1)))
    assert np.array_equal(ctx.read_targets(), np.tile(p.target, (outs.shape[0], 1)))


@pytest.mark.parametrize("schedule,lanes,threads", [(0, 0, 256), (0, 1, 256), (0, 2, 256), (0, 4, 256), (1, 1, 256),
                                                    (1, 2, 512), (1, 4, 512), (1, 8, 256), (2, 0, 512),
                                                    (3, 0, 512), (3, 2, 512), (4, 0, 256), (5, 0, 256)])
@pytest.mark.parametrize("precision", [0, 1])
def test_schedules_match_oracle(engine_lib, oracle_mod, schedule, lanes, threads, precision):
    """Every schedule (level launches, persistent tiles of 1-8 lanes) gives the oracle's states and statuses."""
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 150, seed=21)
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    ctx = native.BatchContext(s, outs.shape[0])
    ctx.set_linear_solver_settings(precision, 1)
    ctx.set_schedule(schedule, lanes, threads)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    ref = oracle_rows(oracle_mod, "grid2000", p.x_base, dis)
    _compare(r, ref, p.n, _tol(precision))


def test_autotuner_picks_a_schedule_and_keeps_results(engine_lib, oracle_mod):
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 64, seed=22)
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    ctx = native.BatchContext(s, outs.shape[0])
    ctx.set_schedule(native.AUTOTUNE)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    (sc, lanes, threads), tuning = ctx.schedule()
    assert len(tuning) == 13      # 4 level, 3 shared-memory level, 1 subtree-bin, 1 cooperative, 4 persistent
    best = min(tuning, key=lambda t: t[3])
    assert (sc, lanes, threads) == (int(best[0]), int(best[1]), int(best[2]))
    ref = oracle_mod.Structure(p).solve_batch(p.x_base, dis)
    _compare(r, ref, p.n)


def test_persistent_reactive_limits_match_oracle(engine_lib, oracle_mod):
    from olfgpu import native, synthetic
    g, p = grid("grid300")
    outs = synthetic.draw_outages(g, 64, seed=301)
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    for sched in (0, 1, 2, 3, 4):
        ctx = native.BatchContext(s, outs.shape[0], rl=p.rl)
        ctx.set_schedule(sched, 2, 256)
        r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
        ref = oracle_mod.Structure(p).solve_batch(p.x_base, dis, reactive_limits=True)
        _compare(r, ref, p.n)


@pytest.mark.parametrize("schedule,lanes,threads", [(0, 2, 256), (1, 2, 256)])
def test_fallback_start_restarts_failed_lanes(engine_lib, oracle_mod, schedule, lanes, threads):
    """Lanes whose start state fails (NaN: DIVERGED at once) restart from the base start inside the same solve and
    end with the oracle's base-start result; the other lanes keep their own start and are not restarted."""
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 70, seed=77)
    dis = p.outage_masks(outs)
    x0 = np.tile(p.x_base, (outs.shape[0], 1))
    bad = np.array([0, 5, 33, 69])
    x0[bad] = np.nan
    s = native.Structure(p)
    ctx = native.BatchContext(s, outs.shape[0])
    ctx.set_schedule(schedule, lanes, threads)
    ctx.set_fallback_start(True)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis, x0_full=x0)
    assert np.array_equal(ctx.last_fallbacks(), bad)
    ref = oracle_mod.Structure(p).solve_batch(p.x_base, dis)
    _compare(r, ref, p.n)
    # without the fallback the NaN lanes diverge
    ctx.set_fallback_start(False)
    r2 = ctx.solve(p.x_base, p.target, p.base_row_mode, dis, x0_full=x0)
    assert np.all(r2[bad, p.n + 2] == -1)
    assert ctx.last_fallbacks().size == 0


def test_phase_timing_reports_every_phase(engine_lib):
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 64, seed=78)
    s = native.Structure(p)
    ctx = native.BatchContext(s, outs.shape[0])
    ref = ctx.solve(p.x_base, p.target, p.base_row_mode, p.outage_masks(outs)).copy()
    ctx.set_phase_timing(True)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, p.outage_masks(outs))
    ph = ctx.last_phase_times()
    assert np.array_equal(r, ref)        # same kernels, same order: the same bits
    assert ph["iterations"] >= 2 and ph["factor"] > 0 and ph["solve"] > 0 and ph["fill"] > 0
    assert ph["factorized_lanes"] >= outs.shape[0]


@pytest.mark.parametrize("schedule", [0, 3, 4])
def test_pivot_growth_refactors_in_fp64(engine_lib, oracle_mod, schedule):
    """Mixed precision: with the growth limit at its minimum every lane's FP32 factorization is flagged and redone in
    FP64 in the same iteration, which reproduces the FP64 engine bit for bit; with the default limit at most a few lanes
    of this well-conditioned batch are flagged (which depends on the FP32 rounding along each lane's iterations) and
    the result matches the oracle."""
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 96, seed=91)
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    c64 = native.BatchContext(s, outs.shape[0])
    c64.set_schedule(schedule, 2, 256)
    r64 = c64.solve(p.x_base, p.target, p.base_row_mode, dis)
    cm = native.BatchContext(s, outs.shape[0])
    cm.set_schedule(schedule, 2, 256)
    cm.set_linear_solver_settings(native.MIXED, 1)
    cm.set_mixed_precision_controls(1e-2, 1.0)
    rm = cm.solve(p.x_base, p.target, p.base_row_mode, dis)
    assert cm.last_fp64_refactors().size == outs.shape[0]
    assert np.array_equal(rm, r64)
    cm.set_mixed_precision_controls(1e-2, 1e4)
    rm = cm.solve(p.x_base, p.target, p.base_row_mode, dis)
    assert cm.last_fp64_refactors().size <= outs.shape[0] // 20
    _compare(rm, oracle_rows(oracle_mod, "grid2000", p.x_base, dis), p.n, MIXED_STATE_TOL)


@pytest.mark.parametrize("refine_below", [float("inf"), 1e-2, 1e-12])
def test_adaptive_refinement_matches_oracle(engine_lib, oracle_mod, refine_below):
    """Refinement in every iteration, near convergence only, or never: the same statuses; the states at 1e-8 when the
    last step is refined (without refinement the last step keeps its FP32 error)."""
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 96, seed=92)
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    ctx = native.BatchContext(s, outs.shape[0])
    ctx.set_linear_solver_settings(native.MIXED, 3)
    ctx.set_mixed_precision_controls(refine_below, 1e4)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    tol = UNREFINED_STATE_TOL if refine_below < 1e-9 else MIXED_STATE_TOL
    _compare(r, oracle_rows(oracle_mod, "grid2000", p.x_base, dis), p.n, tol)


@pytest.mark.parametrize("schedule,lanes,threads", [(0, 2, 256), (0, 0, 256), (1, 2, 256), (2, 0, 512),
                                                    (3, 2, 512)])
@pytest.mark.parametrize("precision", [0, 1])
def test_deferred_l_plan_matches_oracle(engine_lib, oracle_mod, schedule, lanes, threads, precision):
    """The deferred-L block-LU plan (half the factorization levels) gives the oracle's states and statuses."""
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 120, seed=93)
    dis = p.outage_masks(outs)
    s = native.Structure(p, ordering=native.PLAN_DEFERRED_L)
    base = native.Structure(p)
    assert s.factor_levels < base.factor_levels
    ctx = native.BatchContext(s, outs.shape[0])
    ctx.set_linear_solver_settings(precision, 1)
    ctx.set_schedule(schedule, lanes, threads)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    _compare(r, oracle_rows(oracle_mod, "grid2000", p.x_base, dis), p.n, _tol(precision))


@pytest.mark.parametrize("precision", [0, 1])
def test_cooperative_sweeps_match_level_launches(engine_lib, precision):
    """The cooperative schedule runs the same arithmetic in the same order as the level launches: identical results."""
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 80, seed=94)
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    res = []
    for sched in (0, 2):
        ctx = native.BatchContext(s, outs.shape[0])
        ctx.set_linear_solver_settings(precision, 1)
        ctx.set_schedule(sched, 0, 512 if sched == 2 else 256)
        res.append(ctx.solve(p.x_base, p.target, p.base_row_mode, dis).copy())
    assert np.array_equal(res[0], res[1])


@pytest.mark.parametrize("schedule,lanes,threads", [(0, 2, 256), (0, 0, 256), (2, 0, 512), (3, 0, 512),
                                                    (3, 2, 512), (4, 0, 256), (5, 0, 256)])
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", ["grid2000", "grid9241"])
@pytest.mark.parametrize("plan", [16, 19])
def test_dense_front_plan_matches_oracle(engine_lib, oracle_mod, schedule, lanes, threads, precision, name, plan):
    """The dense-front plans (the trailing dense block factorized in shared memory; on plain minimum degree, 16, and
    on minimum degree toward a shallow elimination tree, 19) give the oracle's statuses and states, with fewer
    dependency levels."""
    from olfgpu import native, synthetic
    g, p = grid(name)
    outs = synthetic.draw_outages(g, 64, seed=96)
    dis = p.outage_masks(outs)
    s = native.Structure(p, ordering=plan)
    assert s.factor_levels < native.Structure(p).factor_levels
    ctx = native.BatchContext(s, outs.shape[0])
    ctx.set_linear_solver_settings(precision, 1)
    ctx.set_schedule(schedule, lanes, threads)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    _compare(r, oracle_rows(oracle_mod, name, p.x_base, dis), p.n, _tol(precision))


def test_dense_front_plan_rejected_by_tiles(engine_lib):
    from olfgpu import native
    p = grid("grid2000")[1]
    s = native.Structure(p, ordering=native.PLAN_DENSE_FRONT)
    ctx = native.BatchContext(s, 4)
    ctx.set_schedule(native.PERSISTENT, 2, 256)
    with pytest.raises(native.NativeError, match="dense-front"):
        ctx.solve(p.x_base, p.target, p.base_row_mode, np.zeros((4, p.n_elements), np.uint8))
    # a multi-grid launch takes the member, but its persistent tiles refuse the plan (its device loops run it)
    ctx.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
    ctx.stage(p.x_base, p.target, p.base_row_mode, np.zeros((4, p.n_elements), np.uint8))
    m = native.MultiContext([ctx])
    m.set_schedule(2, 256, 0)
    with pytest.raises(native.NativeError, match="dense-front"):
        m.solve()
    m.set_schedule(0, 0, 0)
    outs, _ = m.solve()
    assert np.all(outs[0][:, p.n + 2] == 0)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", ["grid2000", "grid13659"])
def test_subtree_bins_match_oracle(engine_lib, oracle_mod, precision, name):
    """Schedule 5 (the wide levels' subtrees as bins, one launch per phase) on the plain and dense-front plans: the
    oracle's statuses and states; the FP64 result stays within rounding of schedule 4's (the same arithmetic in
    another split)."""
    from olfgpu import native, synthetic
    g, p = grid(name)
    outs = synthetic.draw_outages(g, 96, seed=97)
    dis = p.outage_masks(outs)
    ref = oracle_rows(oracle_mod, name, p.x_base, dis)
    for plan in (0, native.PLAN_DENSE_FRONT, native.PLAN_DEFAULT):
        s = native.Structure(p, ordering=plan)
        assert s.subtrees()["bins"] > 0
        r = {}
        for sched in (4, 5):
            ctx = native.BatchContext(s, outs.shape[0])
            ctx.set_linear_solver_settings(precision, 3)
            ctx.set_schedule(sched, 0, 256)
            r[sched] = ctx.solve(p.x_base, p.target, p.base_row_mode, dis).copy()
        _compare(r[5], ref, p.n, _tol(precision))
        if precision == 0:
            assert np.array_equal(r[5][:, -1], r[4][:, -1])
            assert np.max(np.abs(r[5][:, :p.n] - r[4][:, :p.n])) < 1e-11


@pytest.mark.parametrize("precision,tol", [(0, 1e-9), (1, 2e-3)])
@pytest.mark.parametrize("name,plan", [("grid2000", 0), ("grid2000", 16), ("grid9241", 16), ("grid9241", 19)])
def test_transposed_solve_matches_oracle(engine_lib, oracle_mod, precision, tol, name, plan):
    """J^T y = c on the factors of J (the adjoint solve, lu/transposed_solve.cuh): against the oracle's LU of the
    explicit transpose; the plain solve of the same call against the oracle's LU of J."""
    from olfgpu import native
    g, p = grid(name)
    ns = 24
    s = native.Structure(p, ordering=plan)
    ctx = native.BatchContext(s, ns)
    x = _perturbed_states(p, ns, 4, 0.02)
    st = oracle_mod.Structure(p)
    zero = np.zeros(p.n_elements, np.uint8)
    J = np.stack([st.fill(x[k], p.target, p.base_row_mode, zero)[0] for k in range(ns)])
    rng = np.random.default_rng(5)
    rhs, rhs_t = rng.standard_normal((ns, p.n)), rng.standard_normal((ns, p.n))
    xs, ys = ctx.linear_solve_transposed(J, rhs, rhs_t, precision)
    for k in range(0, ns, 5):
        zo = st.linear_solve(J[k], rhs[k])
        yo = st.linear_solve_transposed(J[k], rhs_t[k])
        assert np.max(np.abs(xs[k] - zo)) / np.max(np.abs(zo)) < tol
        assert np.max(np.abs(ys[k] - yo)) / np.max(np.abs(yo)) < tol
    # adjoint identity: <y, J x> = <J^T y, x> = <c, x> for the solved pairs
    _, y_only = ctx.linear_solve_transposed(J, None, rhs_t, precision)
    assert np.array_equal(y_only, ys)


def test_config1_every_non_bridge_outage_of_the_2000_bus_grid(engine_lib, oracle_mod):
    """The batched N-1 configuration at full size: every non-bridge (non-parallel) single-branch outage of the
    2,000-bus grid in ONE uniform FP64 batch sharing one structure, warm-started from the base case, tol 1e-8 pu,
    through the device-resident loop; every scenario's status and converged state match the oracle."""
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.outage_candidates(g)
    assert outs.shape[0] > 2000
    dis = p.outage_masks(outs)
    s = native.Structure(p, native.PLAN_DEFAULT)
    ctx = native.BatchContext(s, outs.shape[0])
    ctx.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
    ctx.set_device_loop(True)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
    ref = oracle_mod.Structure(p).solve_batch(p.x_base, dis)
    _compare(r, ref, p.n)
    assert np.array_equal(r[:, p.n].astype(int), ref[:, p.n].astype(int))
