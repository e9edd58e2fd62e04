"""Parity on the benchmark's own configuration (needs a B200): the 9,241-bus grid's 500 drawn outages, the learned
warm start with the base-start fallback, FP32 LU with FP64 refinement and the dense-front plans (on plain minimum
degree, and on the shallow-tree minimum degree the benchmark runs) under the shared-memory level schedule: every scenario's status equals the FP64 oracle's and every converged state is within 1e-8 pu / rad of
it; the plain FP64 engine on the same batch agrees too."""
import os

import numpy as np
import pytest

from conftest import ROOT, grid

pytestmark = pytest.mark.gpu

CHECKPOINT = os.path.join(ROOT, "olf-gpu_b200", "checkpoints", "warmstart_grid9241.npz")
STATE_TOL = 1e-8


@pytest.fixture(scope="module")
def headline(oracle_mod):
    from olfgpu import synthetic
    g, p = grid("grid9241")
    outs = synthetic.draw_outages(g, 500, seed=9241)
    ref = oracle_mod.Structure(p).solve_batch(p.x_base, p.outage_masks(outs))
    return g, p, outs, ref


def _check(r, ref, n):
    st_e, st_o = r[:, n + 2].astype(int), ref[:, n + 2].astype(int)
    assert np.array_equal(st_e, st_o), f"status mismatch at {np.flatnonzero(st_e != st_o)[:10]}"
    conv = st_o == 0
    assert conv.any()
    d = np.abs(r[conv, :n] - ref[conv, :n])
    assert d[:, 1::2].max() <= STATE_TOL, ("Vm", float(d[:, 1::2].max()))
    assert d[:, 0::2].max() <= STATE_TOL, ("Va", float(d[:, 0::2].max()))


PLANS = {"dense": 16, "shallow": 19}     # native.PLAN_DENSE_FRONT, native.PLAN_DEFAULT


@pytest.mark.parametrize("plan", sorted(PLANS))
@pytest.mark.parametrize("policy", [0, 1])
def test_learned_mixed_matches_oracle_on_the_benchmark_batch(engine_lib, headline, policy, plan):
    """Both mixed-precision policies; the scenarios that converge from their learned start take the polishing step
    (on by default), the others run from the base start as the oracle does."""
    import torch
    from olfgpu import native
    from olfgpu.learned_start import LearnedStart
    g, p, outs, ref = headline
    ns = outs.shape[0]
    s = native.Structure(p, PLANS[plan])
    ctx = native.BatchContext(s, ns)
    ctx.set_linear_solver_settings(native.MIXED, 3)
    ctx.set_mixed_precision_policy(policy)
    ctx.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
    learned = LearnedStart.load(CHECKPOINT, g)
    x0_dev = torch.empty((ns, p.n), dtype=torch.float64, device="cuda")
    ctx.set_fallback_start(True)
    ctx.set_device_start(x0_dev)
    learned.predict_device(p, p.x_base, outs, out=x0_dev)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, p.outage_masks(outs))
    _check(r, ref, p.n)
    ctx.set_device_start(None)


def test_polishing_step_brings_learned_lanes_next_to_the_solution(engine_lib, headline):
    """Without the polishing step a scenario that converged from its learned start may stop anywhere in the tolerance
    ball; with it, every converged state lies within 1e-9 of the FP64 engine's polished base-start state."""
    import torch
    from olfgpu import native
    from olfgpu.learned_start import LearnedStart
    g, p, outs, ref = headline
    ns = outs.shape[0]
    dis = p.outage_masks(outs)
    s = native.Structure(p, native.PLAN_DENSE_FRONT)
    learned = LearnedStart.load(CHECKPOINT, g)
    x0_dev = torch.empty((ns, p.n), dtype=torch.float64, device="cuda")
    learned.predict_device(p, p.x_base, outs, out=x0_dev)
    out, kept = {}, {}
    for ratio in (0.0, 1e-2):
        ctx = native.BatchContext(s, ns)
        ctx.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
        ctx.set_fallback_start(True)
        ctx.set_start_polish(ratio)
        ctx.set_device_start(x0_dev)
        out[ratio] = ctx.solve(p.x_base, p.target, p.base_row_mode, dis)
        kept[ratio] = np.ones(ns, bool)                    # the scenarios that stayed on their learned start
        kept[ratio][ctx.last_fallbacks()] = False
        ctx.set_device_start(None)
    # the solution itself: the base-start states taken one step further (max |F| far below the tolerance)
    base = native.BatchContext(s, ns)
    base.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
    x_star = base.solve(p.x_base, p.target, p.base_row_mode, dis, x0_full=np.ascontiguousarray(ref[:, :p.n]),
                        tol=1e-11, max_iter=3)
    n = p.n
    conv = (out[1e-2][:, n + 2] == 0) & (x_star[:, n + 2] == 0)
    assert conv.sum() > 0.9 * ns
    learned_lanes = conv & kept[1e-2] & kept[0.0]
    assert learned_lanes.sum() >= 5
    polished = np.abs(out[1e-2][learned_lanes, :n] - x_star[learned_lanes, :n]).max()
    plain = np.abs(out[0.0][learned_lanes, :n] - x_star[learned_lanes, :n]).max()
    assert polished <= 1e-9 and polished <= plain, (polished, plain)
    # the scenarios on the base start follow the oracle's own trajectory
    base_lanes = conv & ~kept[1e-2]
    assert np.abs(out[1e-2][base_lanes, :n] - ref[base_lanes, :n]).max() <= 1e-11


@pytest.mark.parametrize("plan", sorted(PLANS))
@pytest.mark.parametrize("precision", [0, 1])
def test_base_start_matches_oracle_on_the_benchmark_batch(engine_lib, headline, precision, plan):
    from olfgpu import native
    g, p, outs, ref = headline
    s = native.Structure(p, PLANS[plan])
    ctx = native.BatchContext(s, outs.shape[0])
    ctx.set_linear_solver_settings(precision, 3)
    ctx.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
    r = ctx.solve(p.x_base, p.target, p.base_row_mode, p.outage_masks(outs))
    _check(r, ref, p.n)
