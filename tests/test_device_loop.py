"""The device-resident Newton loop (one graph launch with conditional nodes) gives exactly the host-driven loop's
results under every level schedule, precision policy and outer loop (needs a B200)."""
import numpy as np
import pytest

from conftest import grid

pytestmark = pytest.mark.gpu


def _both(make, solve):
    """Results of the host-driven and the device-resident loop on fresh contexts, and their batched iterations."""
    out = []
    for loop in (False, True):
        ctx = make()
        ctx.set_device_loop(loop)
        r = solve(ctx)
        r2 = solve(ctx)                       # a second solve replays the cached graph
        assert np.array_equal(r, r2, equal_nan=True)
        out.append((r, ctx.last_stats()[1], ctx.last_fp64_iterations()))
        ctx.close()
    return out


def _same(a, b):
    assert np.array_equal(a[0], b[0], equal_nan=True)
    assert a[1] == b[1] and a[2] == b[2]


@pytest.mark.parametrize("schedule,plan", [((0, 0, 256), 0), ((0, 2, 256), 0), ((3, 0, 512), 0), ((4, 0, 256), 16),
                                           ((5, 0, 256), 16)])
@pytest.mark.parametrize("precision,policy", [(0, 0), (1, 0), (1, 1)])
def test_device_loop_equals_host_loop(engine_lib, schedule, plan, precision, policy):
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 120, seed=31)
    dis = p.outage_masks(outs)
    s = native.Structure(p, plan)

    def make():
        c = native.BatchContext(s, outs.shape[0])
        c.set_linear_solver_settings(precision, 3)
        c.set_mixed_precision_policy(policy)
        c.set_schedule(*schedule)
        return c

    host, dev = _both(make, lambda c: c.solve(p.x_base, p.target, p.base_row_mode, dis))
    _same(host, dev)


def test_device_loop_with_outer_loops_and_rules(engine_lib):
    """Reactive limits, distributed slack, the 2-norm test and the MAX_VOLTAGE_CHANGE clamp inside the device loop."""
    from olfgpu import native, packing, synthetic
    g, p = grid("grid300")
    outs = synthetic.draw_outages(g, 80, seed=32)
    dis = p.outage_masks(outs)
    s = native.Structure(p)
    ds = packing.distributed_slack(g, p)
    for kwargs, solve_kw in [(dict(rl=p.rl), {}), (dict(ds=ds), {}), (dict(rl=p.rl, ds=ds), {}),
                             ({}, dict(conv_eps_per_eq=1e-9)),
                             ({}, dict(svs_mode=native.SVS_MAX_VOLTAGE_CHANGE, var_type=p.var_type, max_dv=0.02,
                                       max_dphi=0.05))]:
        host, dev = _both(lambda: native.BatchContext(s, outs.shape[0], **kwargs),
                          lambda c: c.solve(p.x_base, p.target, p.base_row_mode, dis, **solve_kw))
        _same(host, dev)


def test_device_loop_with_fallback_start(engine_lib):
    """Own starts with the base-start fallback and the polishing step: start selection before the loop, restarts and
    the extra step inside it."""
    from olfgpu import native, synthetic
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 96, seed=33)
    dis = p.outage_masks(outs)
    rng = np.random.default_rng(5)
    x0 = np.tile(p.x_base, (outs.shape[0], 1))
    x0[:, 0::2] += rng.normal(0, 0.02, (outs.shape[0], p.n_bus)) * (rng.random((outs.shape[0], 1)) < 0.5)
    x0[:12, 0::2] += 3.0                          # starts that fail and fall back
    s = native.Structure(p)

    def make():
        c = native.BatchContext(s, outs.shape[0])
        c.set_fallback_start(True)
        return c

    host, dev = _both(make, lambda c: c.solve(p.x_base, p.target, p.base_row_mode, dis, x0_full=x0))
    _same(host, dev)


@pytest.mark.parametrize("parts", [2, 4])
def test_concurrent_parts_equal_the_single_batch(engine_lib, parts):
    """A batch split into lane ranges solved as concurrent device loops in one graph launch (ConcurrentBatch) gives
    every scenario the single batch's result bit for bit, with device-resident starts, selection and fallback."""
    import torch
    from olfgpu import native, synthetic
    from olfgpu.security_analysis import ConcurrentBatch
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 150, seed=34)
    dis = p.outage_masks(outs)
    rng = np.random.default_rng(9)
    x0 = np.tile(p.x_base, (outs.shape[0], 1))
    x0[:, 0::2] += rng.normal(0, 0.01, (outs.shape[0], p.n_bus))
    x0[:9, 0::2] += 3.0
    x0_dev = torch.from_numpy(x0).cuda()
    s = native.Structure(p, native.PLAN_DENSE_FRONT)
    single = native.BatchContext(s, outs.shape[0])
    single.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
    single.set_device_loop(True)
    single.set_fallback_start(True)
    single.set_device_start(x0_dev)
    ref = single.solve(p.x_base, p.target, p.base_row_mode, dis)
    cb = ConcurrentBatch(s, outs.shape[0], parts)
    cb.set_device_start(x0_dev)
    r, ms = cb.solve(p.x_base, p.target, p.base_row_mode, dis)
    assert ms > 0
    assert np.array_equal(r, ref)
    assert np.array_equal(np.sort(cb.last_fallbacks()), np.sort(single.last_fallbacks()))
    cb.close()
