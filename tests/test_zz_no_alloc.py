"""The allocation-free batched linear solve (olfgpu_linear_solve_noalloc), through the C ABI, on a GPU.

Some callers cannot allocate device memory when they solve (their GPU memory was reserved up front by a JVM or a
service, or they must avoid cudaMalloc/cudaFree because those synchronise the device).  This entry point keeps its
scratch in a fixed array inside the library and works on device buffers the caller owns.  Its results must equal those
of the ordinary entry point (olfgpu_debug_linear_solve) on two calls in a row, and the second call must not change the
device's free memory.  This file is collected last on purpose.
"""
import numpy as np
import pytest

from conftest import grid

pytestmark = pytest.mark.gpu

# the tolerances of the engine's linear-solve parity test: FP64 factors, FP32 factors (relative to the FP64 answer)
TOL = {0: 1e-9, 1: 2e-3}


def _inputs(p, oracle_mod, ns, seed):
    rng = np.random.default_rng(seed)
    x = np.tile(p.x_base, (ns, 1))
    x[:, 0::2] += rng.uniform(-0.02, 0.02, (ns, p.n_bus))
    x[:, 1::2] += rng.uniform(-0.02, 0.02, (ns, p.n_bus))
    st = oracle_mod.Structure(p)
    zero = np.zeros(p.n_elements, np.uint8)
    J = np.stack([st.fill(x[k], p.target, p.base_row_mode, zero)[0] for k in range(ns)])
    rhs = rng.standard_normal((ns, p.n))
    return J, rhs


@pytest.mark.parametrize("name,plan", [("grid118", 0), ("grid2000", 16)])
@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_solve_matches_the_allocating_solve(engine_lib, oracle_mod, name, plan, precision):
    """FP64 and FP32 factors, on the plain plan and on a dense-front plan (whose front runs in the scratch layout)."""
    import torch
    from olfgpu import native
    g, p = grid(name)
    ns = 40 if name == "grid118" else 24
    s = native.Structure(p, ordering=plan)
    ctx = native.BatchContext(s, ns)          # uploads the structure to this device (allocates, before the calls)
    dev = torch.device("cuda:0")
    J1, r1 = _inputs(p, oracle_mod, ns, 1)
    J2, r2 = _inputs(p, oracle_mod, ns, 2)
    # caller-owned device buffers, allocated by the caller before the calls
    bufs = [torch.from_numpy(a).to(dev) for a in (J1, r1, J2, r2)]
    out = torch.zeros((ns, p.n), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    results = []
    for k, (Jd, rd) in enumerate(((bufs[0], bufs[1]), (bufs[2], bufs[3]))):
        free_before = torch.cuda.mem_get_info(0)[0]
        s.linear_solve_noalloc(ns, Jd.data_ptr(), rd.data_ptr(), out.data_ptr(), precision, 0)
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info(0)[0]
        if k == 1:
            assert free_after == free_before, "the second call changed the device's free memory"
        results.append(out.cpu().numpy().copy())
    ref1 = ctx.debug_linear_solve(J1, r1, native.FP64)
    ref2 = ctx.debug_linear_solve(J2, r2, native.FP64)
    for got, ref in ((results[0], ref1), (results[1], ref2)):
        assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < TOL[precision]
    if precision == 1:
        # the same FP32 factors as the allocating entry point's FP32 solve
        for got, (J, r) in ((results[0], (J1, r1)), (results[1], (J2, r2))):
            ref32 = ctx.debug_linear_solve(J, r, native.MIXED)
            assert np.max(np.abs(got - ref32)) / np.max(np.abs(ref32)) < 1e-5
    # the two calls solved different systems: the shared scratch did not leak the first into the second
    assert np.max(np.abs(results[0] - results[1])) > 1e-3


def test_noalloc_rejects_a_batch_beyond_its_scratch(engine_lib):
    import torch
    from olfgpu import native
    g, p = grid("grid2000")
    s = native.Structure(p)
    native.BatchContext(s, 1)
    big = 4096
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    with pytest.raises(native.NativeError, match="scratch"):
        s.linear_solve_noalloc(big, dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), native.FP64, 0)


def test_noalloc_marks_a_singular_system_with_nan(engine_lib, oracle_mod):
    """A scenario whose factorization meets a singular pivot gets NaN throughout; the other scenarios are solved."""
    import torch
    from olfgpu import native
    g, p = grid("grid118")
    ns = 8
    s = native.Structure(p)
    ctx = native.BatchContext(s, ns)
    J, r = _inputs(p, oracle_mod, ns, 3)
    # zero the two rows and columns of one PQ bus in scenario 3: its 2x2 pivot is exactly singular
    ex = s.export()
    bus = int(np.flatnonzero(p.base_row_mode[0::2] == 1)[3])
    rows = (2 * bus, 2 * bus + 1)
    for k in range(ex["row_ptr"][rows[0]], ex["row_ptr"][rows[1] + 1]):
        J[3, k] = 0.0
    cols = np.isin(ex["col_idx"], rows)
    J[3, cols] = 0.0
    dev = torch.device("cuda:0")
    Jd, rd = torch.from_numpy(J).to(dev), torch.from_numpy(r).to(dev)
    out = torch.zeros((ns, p.n), dtype=torch.float64, device=dev)
    s.linear_solve_noalloc(ns, Jd.data_ptr(), rd.data_ptr(), out.data_ptr(), native.FP64, 0)
    got = out.cpu().numpy()
    assert np.all(np.isnan(got[3]))
    keep = [k for k in range(ns) if k != 3]
    ref = ctx.debug_linear_solve(J[keep[:1] * ns], r[keep[:1] * ns], native.FP64)[0]
    assert np.all(np.isfinite(got[keep]))
    assert np.max(np.abs(got[keep[0]] - ref)) / np.max(np.abs(ref)) < TOL[0]
