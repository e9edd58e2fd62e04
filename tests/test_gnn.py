"""Learned warm start: the library's BF16 graph-network kernels against float64 references (needs a B200)."""
import numpy as np
import pytest

from conftest import grid

pytestmark = pytest.mark.gpu

# BF16 activations and weights with FP32 accumulation: ~3 significant digits
REL_FWD = 3e-2
REL_GRAD = 6e-2


def _bf16_round(a):
    import torch
    return torch.from_numpy(np.asarray(a, np.float32)).to(torch.bfloat16).to(torch.float64).numpy()


@pytest.mark.parametrize("M", [1000, 128 * 700 + 37])
@pytest.mark.parametrize("k1,k2,n", [(16, 0, 64), (64, 0, 128), (64, 64, 64), (64, 0, 16), (128, 0, 64)])
def test_gemm_matches_float64(engine_lib, k1, k2, n, M):
    """The tensor-core GEMM (tcgen05, 128-row tiles; the larger M walks more tiles than CTAs) with bias, ReLU,
    residual, the saved pre-residual z and FP32 output; none of its waits gave up."""
    import torch
    from olfgpu import gnn
    rng = np.random.default_rng(k1 + k2 + n)
    a1 = rng.standard_normal((M, k1)).astype(np.float32)
    a2 = rng.standard_normal((M, k2)).astype(np.float32) if k2 else None
    w = (rng.standard_normal((k1 + k2, n)) / 8).astype(np.float32)
    bias = rng.standard_normal(n).astype(np.float32)
    res = rng.standard_normal((M, n)).astype(np.float32)
    d = lambda x: torch.from_numpy(x).cuda().to(torch.bfloat16).contiguous()  # noqa: E731
    A1, A2, W, R = d(a1), (d(a2) if k2 else None), d(w), d(res)
    B = torch.from_numpy(bias).cuda()
    out = torch.empty((M, n), dtype=torch.float32, device="cuda")
    z = torch.empty((M, n), dtype=torch.bfloat16, device="cuda")
    gnn._call("olfgpu_gnn_gemm", M, k1, k2, n, gnn._ptr(A1), gnn._ptr(A2), gnn._ptr(W), gnn._ptr(B), 1, gnn._ptr(R),
              None, gnn._ptr(out), n, gnn._ptr(z), gnn._stream())
    torch.cuda.synchronize()
    aa = np.concatenate([_bf16_round(a1)] + ([_bf16_round(a2)] if k2 else []), axis=1)
    ref_z = np.maximum(aa @ _bf16_round(w) + bias, 0)
    ref = ref_z + _bf16_round(res)
    assert np.max(np.abs(out.cpu().numpy() - ref)) / np.max(np.abs(ref)) < 1e-5
    assert np.max(np.abs(z.float().cpu().numpy() - ref_z)) / np.max(np.abs(ref_z)) < 1e-2
    # the BF16 output without bias, ReLU or residual
    ob, _ = gnn.gemm(A1, A2, W)
    torch.cuda.synchronize()
    ref_y = aa @ _bf16_round(w)
    assert np.max(np.abs(ob.float().cpu().numpy() - ref_y)) / np.max(np.abs(ref_y)) < 1e-2
    assert gnn.tc_timeouts() == 0


@pytest.mark.parametrize("k1,k2,n", [(16, 0, 64), (64, 0, 128), (64, 64, 64), (64, 0, 16)])
def test_weight_gradient_matches_float64(engine_lib, k1, k2, n):
    import torch
    from olfgpu import gnn
    rng = np.random.default_rng(7 + k1 + n)
    M = 5000
    a1 = rng.standard_normal((M, k1)).astype(np.float32)
    a2 = rng.standard_normal((M, k2)).astype(np.float32) if k2 else None
    dz = rng.standard_normal((M, n)).astype(np.float32)
    d = lambda x: torch.from_numpy(x).cuda().to(torch.bfloat16).contiguous()  # noqa: E731
    dw = torch.empty((k1 + k2, n), dtype=torch.float32, device="cuda")
    db = torch.empty(n, dtype=torch.float32, device="cuda")
    partial = torch.empty(37 * ((k1 + k2) * n + n), dtype=torch.float32, device="cuda")
    A1, A2, DZ = d(a1), (d(a2) if k2 else None), d(dz)      # keep the inputs alive until the kernel has run
    gnn._call("olfgpu_gnn_gemm_dw", M, k1, k2, n, gnn._ptr(A1), gnn._ptr(A2), gnn._ptr(DZ), gnn._ptr(dw),
              gnn._ptr(db), gnn._ptr(partial), 37, gnn._stream())
    torch.cuda.synchronize()
    aa = np.concatenate([_bf16_round(a1)] + ([_bf16_round(a2)] if k2 else []), axis=1)
    ref = aa.T @ _bf16_round(dz)
    assert np.max(np.abs(dw.cpu().numpy() - ref)) / np.max(np.abs(ref)) < 1e-4
    assert np.max(np.abs(db.cpu().numpy() - _bf16_round(dz).sum(0))) < 1e-2


def _small_problem(name="grid118", B=4, seed=0):
    import torch
    from olfgpu import synthetic
    from olfgpu.gnn import FEAT_IN, GraphData, WarmStartNet, init_params
    g, p = grid(name)
    graph = GraphData.from_grid(g)
    rng = np.random.default_rng(seed)
    params = init_params(4, seed)
    # give the biases and the padded output columns non-trivial values so every path is exercised
    for k in params:
        if k.startswith("b_"):
            params[k] = (rng.standard_normal(params[k].shape) * 0.05).astype(np.float32)
    net = WarmStartNet(graph, 4, params=params)
    x0 = np.zeros((B * g.n_bus, FEAT_IN), np.float32)
    x0[:, :7] = rng.standard_normal((B * g.n_bus, 7))
    outs = synthetic.outage_candidates(g)[:B].astype(np.int32)
    target = rng.standard_normal((B * g.n_bus, 2)).astype(np.float32)
    x0b = torch.from_numpy(x0).cuda().to(torch.bfloat16)
    gnp = {k: getattr(graph, k).cpu().numpy() for k in ("src", "dst", "branch", "es")}
    return g, graph, net, params, x0, x0b, outs, target, gnp


def test_forward_and_gradients_match_the_float64_oracle(engine_lib):
    import torch
    from oracle import gnn_oracle
    g, graph, net, params, x0, x0b, outs, target, gnp = _small_problem()
    out = net.forward(x0b, torch.from_numpy(outs).cuda(), keep=False).cpu().numpy()
    loss_ref, out_ref, grads_ref = gnn_oracle.loss_and_grads(params, _bf16_round(x0), outs, target, gnp, g.n_bus, 4)
    assert np.max(np.abs(out[:, :2] - out_ref[:, :2])) / np.max(np.abs(out_ref[:, :2])) < REL_FWD
    loss = net.loss_and_grad(x0b, torch.from_numpy(outs).cuda(), torch.from_numpy(target).cuda())
    assert abs(loss - loss_ref) / loss_ref < REL_FWD
    for k, gr in grads_ref.items():
        mine = net.grad[k].cpu().numpy().reshape(gr.shape)
        if k == "w_out" or k == "b_out":
            mine, gr = mine[..., :2], gr[..., :2]
        rel = np.linalg.norm(mine - gr) / max(np.linalg.norm(gr), 1e-12)
        assert rel < REL_GRAD, (k, rel)


def test_backward_is_deterministic(engine_lib):
    import torch
    g, graph, net, params, x0, x0b, outs, target, gnp = _small_problem(B=6, seed=3)
    o = torch.from_numpy(outs).cuda()
    t = torch.from_numpy(target).cuda()
    net.loss_and_grad(x0b, o, t)
    first = {k: v.clone() for k, v in net.grad.items()}
    net.loss_and_grad(x0b, o, t)
    for k in first:
        assert torch.equal(first[k], net.grad[k]), k


def test_checkpoint_resume_is_exact(engine_lib, tmp_path):
    import torch
    from olfgpu.gnn import WarmStartNet
    g, graph, net, params, x0, x0b, outs, target, gnp = _small_problem(B=3, seed=5)
    o, t = torch.from_numpy(outs).cuda(), torch.from_numpy(target).cuda()
    for _ in range(3):
        net.loss_and_grad(x0b, o, t)
        net.adam(1e-3)
    path = str(tmp_path / "ckpt.npz")
    net.save(path)
    for _ in range(2):
        net.loss_and_grad(x0b, o, t)
        net.adam(1e-3)
    resumed, _ = WarmStartNet.load(path, graph)
    for _ in range(2):
        resumed.loss_and_grad(x0b, o, t)
        resumed.adam(1e-3)
    for k in net.w:
        assert torch.equal(net.w[k], resumed.w[k]), k


def test_learned_start_trains_and_predicts_closer_starts(engine_lib, oracle_mod):
    """On the 2,000-bus grid: training on the engine's own N-1 solutions brings the held-out start error (load
    scalings the network never saw) below both the untrained network's and the base start's; solving from the learned
    starts, with the on-device fallback, reproduces the oracle's statuses and states.  The Newton iterations from both
    starts are reported, not asserted: a start must be within the quadratic region to save a whole iteration."""
    from olfgpu import native, packing, synthetic
    from olfgpu.learned_start import LearnedStart, solve_with_fallback
    g, p = grid("grid2000")
    ls = LearnedStart(g, seed=1)
    data = ls.generate(n_scalings=36, outages_per_scaling=128, seed=2, lo=0.9, hi=1.1)
    train, held = ls.split(data, 4)
    before, base_err = ls.evaluate(data, held)
    ls.train(data, epochs=8, batch=32, lr=1e-3, samples=train)
    after, _ = ls.evaluate(data, held)
    print(f"held-out normalised start error: base start {base_err:.4f}, untrained {before:.4f}, trained {after:.4f}")
    assert after < before and after < base_err
    gs = g.scaled(0.97)
    ps = packing.pack(gs, with_reactive_limits=False)
    xb = ls.solve_base(gs, p.x_base)
    rng = np.random.default_rng(99)
    outs = np.sort(rng.choice(synthetic.outage_candidates(g), size=160, replace=False))
    dis = ps.outage_masks(outs)
    s = native.Structure(ps)
    ctx = native.BatchContext(s, outs.shape[0])
    ctx.solve(xb, ps.target, ps.base_row_mode, dis)
    _, _, it_base = ctx.last_stats()
    it_base = it_base.copy()
    x0 = ls.predict(ps, xb, outs)
    learned, it_learned, bad = solve_with_fallback(ctx, ps, x0, xb, dis)
    print(f"Newton iterations per solve: base start {it_base.mean():.3f}, learned start {it_learned.mean():.3f}, "
          f"{bad.size} fallbacks")
    ref = oracle_mod.Structure(ps).solve_batch(xb, dis)
    assert np.array_equal(learned[:, -1], ref[:, -1])
    conv = ref[:, -1] == 0
    assert np.max(np.abs(learned[conv, :p.n] - ref[conv, :p.n])) <= 1e-8


def test_compact_inference_equals_full_inference(engine_lib):
    """Evaluating only the buses within reach of each outage (plus one outage-free pass) gives the full batched
    forward's start states bit for bit."""
    from olfgpu import synthetic
    from olfgpu.learned_start import LearnedStart
    g, p = grid("grid2000")
    ls = LearnedStart(g, seed=4)
    ls.feat_mean, ls.feat_std = np.zeros(7), np.ones(7)
    ls.tgt_std, ls.flow_std = np.array([0.01, 0.02], np.float32), 1.0
    outs = synthetic.draw_outages(g, 150, seed=95)
    full = ls.predict(p, p.x_base, outs, compact=False)
    compact = ls.predict(p, p.x_base, outs, compact=True)
    rn, rs, _ = ls.reach(outs)
    assert rn.shape[0] < 0.2 * outs.shape[0] * p.n_bus      # far fewer rows than the full batch
    assert np.array_equal(full, compact)
