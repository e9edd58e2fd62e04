"""The oracle (C restatement) against the reference's golden vectors and its own compiled code (CPU)."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")

# codegen/java2cuda/prove.py:59 checks the formula bodies to this tolerance
REL = 1e-12


def _rel(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-12))


def test_formulas_match_golden_manifests(oracle_mod):
    d = np.load(os.path.join(GOLD, "formulas.npz"))
    for i in range(d["cb_in"].shape[0]):
        x = d["cb_in"][i]
        o = oracle_mod.closed_branch(x[:8], x[8], x[9], x[10], x[11], x[12], x[13])
        assert _rel(o, d["cb_gold"][i]) <= REL
        assert np.array_equal(o, d["cb_ref"][i]), "closed branch differs from the reference's generated header"
    for i in range(d["ob_in"].shape[0]):
        x = d["ob_in"][i]
        o = oracle_mod.open_branch(x[:7], x[7], x[8])
        assert _rel(o, d["ob_gold"][i]) <= REL
        assert _rel(o, d["ob_ref"][i]) <= 1e-15
    for i in range(d["sh_in"].shape[0]):
        x = d["sh_in"][i]
        o = oracle_mod.shunt(x[:2], x[2])
        assert _rel(o, d["sh_gold"][i]) <= REL
        assert np.array_equal(o, d["sh_ref"][i])


class _P:
    """Packed arrays loaded from a structure fixture."""

    def __init__(self, d):
        self.n = int(d["n"])
        self.cb_params, self.cb_idx = d["cb_params"], d["cb_idx"]
        self.ob_params, self.ob_idx = d["ob_params"], d["ob_idx"]
        self.sh_params, self.sh_idx = d["sh_params"], d["sh_idx"]
        self.identity_rows = np.zeros(0, np.int32)
        self.n_cb, self.n_ob, self.n_sh = self.cb_idx.shape[0], self.ob_idx.shape[0], self.sh_idx.shape[0]
        self.n_elements = self.n_cb + self.n_ob + self.n_sh


@pytest.mark.parametrize("name", ["grid118", "grid300"])
def test_oracle_structure_matches_reference(oracle_mod, name):
    d = np.load(os.path.join(GOLD, f"structure_{name}.npz"))
    p = _P(d)
    st = oracle_mod.Structure(p)
    a = st.export()
    for k in ("row_map", "row_ptr", "col_idx", "diag_pos", "cb_dest", "ob_dest", "sh_dest"):
        assert np.array_equal(a[k], d["ref_" + k]), k


def test_oracle_newton_flat_start_grid118(oracle_mod):
    from conftest import grid
    g, p = grid("grid118")
    st = oracle_mod.Structure(p)
    r = st.solve_batch(p.x_flat, np.zeros((1, p.n_elements), np.uint8))
    assert r[0, -1] == 0 and r[0, -3] <= 6 and r[0, -2] < 1e-8


def test_oracle_status_rules(oracle_mod):
    """newton_iteration.cu:352-395: a test that passes only at the budget is MAX_ITERATION_REACHED; NaN diverges."""
    from conftest import grid
    g, p = grid("grid118")
    st = oracle_mod.Structure(p)
    flat = np.zeros((1, p.n_elements), np.uint8)
    conv = st.solve_batch(p.x_flat, flat)
    it = int(conv[0, -3])
    at_budget = st.solve_batch(p.x_flat, flat, max_iter=it)
    assert at_budget[0, -1] == 1
    more = st.solve_batch(p.x_flat, flat, max_iter=it + 1)
    assert more[0, -1] == 0
    t = p.target.copy()
    t[2 * int(np.flatnonzero(p.base_row_mode == 1)[0])] = np.nan
    nan = st.solve_batch(p.x_flat, flat, target=t)
    assert nan[0, -1] == -1


class _PN(_P):
    """Packed arrays, targets and row modes loaded from a Newton fixture."""

    def __init__(self, d):
        super().__init__(d)
        self.identity_rows = d["identity_rows"]
        self.target, self.base_row_mode = d["target"], d["base_row_mode"]


# the oracle's solve against Newton solves made of the reference's own formula headers, scatter map and host LU: the
# two factorizations round differently (partial pivoting vs static pivots on another order), nothing else differs
NEWTON_STATE_TOL = 1e-12
LU_REL_TOL = 1e-11


@pytest.mark.parametrize("name", ["grid118", "grid300"])
def test_oracle_newton_matches_reference_components(oracle_mod, name):
    """newton_<grid>.npz (tests/golden/make_golden.py): the base case from a flat start and 24 N-1 outages from the
    base-case start, each solved by a Newton loop whose fill is the reference's generated formulas scattered through
    its own scatter map and whose linear solve is its own host LU (native/host/lu_transposed_check.cpp:74-145 on the
    plan of scalar_lu_plan.cu).  The oracle must take the same iterations to the same status and state."""
    d = np.load(os.path.join(GOLD, f"newton_{name}.npz"))
    p = _PN(d)
    st = oracle_mod.Structure(p)
    a = st.export()
    assert np.array_equal(a["row_ptr"], d["row_ptr"]) and np.array_equal(a["col_idx"], d["col_idx"])
    ref = d["ref_rows"]
    out = st.solve_batch(d["x0"], d["disabled"])
    n = p.n
    assert np.array_equal(out[:, n + 2], ref[:, n + 2]), "statuses differ"
    assert np.array_equal(out[:, n], ref[:, n]), "iteration counts differ"
    conv = ref[:, n + 2] == 0
    assert conv.all()
    assert np.max(np.abs(out[conv, :n] - ref[conv, :n])) <= NEWTON_STATE_TOL


@pytest.mark.parametrize("name", ["grid118", "grid300"])
def test_oracle_linear_solve_matches_reference_host_lu(oracle_mod, name):
    """Jacobians at perturbed states solved by the reference's host LU (newton_<grid>.npz), J x = b and J^T x = b,
    against the oracle's."""
    d = np.load(os.path.join(GOLD, f"newton_{name}.npz"))
    st = oracle_mod.Structure(_PN(d))
    assert not d["lin_trouble"].any(), "the reference's fast engine trusts these systems"
    for vals, b, xr, xt in zip(d["lin_vals"], d["lin_b"], d["lin_x"], d["lin_xt"]):
        x = st.linear_solve(vals, b)
        assert np.max(np.abs(x - xr)) / np.max(np.abs(xr)) <= LU_REL_TOL
        # the transposed solve (lu/transposed_solve.cuh on the same factors) against the oracle's on the transpose
        y = st.linear_solve_transposed(vals, b)
        assert np.max(np.abs(y - xt)) / np.max(np.abs(xt)) <= LU_REL_TOL


def test_reference_components_live_grid2000(oracle_mod):
    """Where the reference sources are present (oracle/_ref built from them): the same pin, live, on the 2,000-bus
    grid (its fill, LU and Newton), beyond the committed fixtures' sizes."""
    if not (oracle_mod.ref_available() and oracle_mod.ref_lu_available()):
        pytest.skip("oracle/_ref not built: no reference tree here")
    from conftest import grid
    from olfgpu import synthetic
    g, p = grid("grid2000")
    st = oracle_mod.Structure(p)
    rs = oracle_mod.ref_structure(p)
    lu = oracle_mod.RefLu(rs["row_ptr"], rs["col_idx"])
    outs = synthetic.draw_outages(g, 4, seed=2000)
    dis = p.outage_masks(outs)
    vo, Fo = st.fill(p.x_base, p.target, p.base_row_mode, dis[0])
    vr, Fr = oracle_mod.ref_component_fill(p, rs, p.x_base, p.target, p.base_row_mode, dis[0])
    assert np.array_equal(vo, vr) and np.array_equal(Fo, Fr)
    b = np.random.default_rng(2000).standard_normal(p.n)
    for solve, mine in ((lu.solve, st.linear_solve), (lu.solve_transposed, st.linear_solve_transposed)):
        xr, trouble = solve(vo, b)
        assert trouble == 0
        assert np.max(np.abs(mine(vo, b) - xr)) / np.max(np.abs(xr)) <= LU_REL_TOL
    out = st.solve_batch(p.x_base, dis)
    for k in range(dis.shape[0]):
        r = oracle_mod.newton_with(
            lambda x: oracle_mod.ref_component_fill(p, rs, x, p.target, p.base_row_mode, dis[k]),
            lambda v, b: lu.solve(v, b)[0], p.x_base)
        assert r[p.n + 2] == out[k, p.n + 2] == 0
        assert r[p.n] == out[k, p.n]
        assert np.max(np.abs(r[:p.n] - out[k, :p.n])) <= NEWTON_STATE_TOL


@pytest.mark.parametrize("name,outage", [("grid118", None), ("grid118", 3), ("grid300", 7)])
def test_jacobian_matches_central_differences(oracle_mod, name, outage):
    """A finite-difference audit of the assembled Jacobian (the reference audits its hand Jacobian the same way,
    codegen/java2cuda/prove.py): every column of J at a perturbed state equals the central difference of the mismatch
    F, through the scatter map and the identity rows, with and without an outaged branch.  The engine's Jacobian equals
    the oracle's to 1e-12 (tests/test_gpu_engine.py), so this audits both."""
    from conftest import grid
    from olfgpu import synthetic
    g, p = grid(name)
    st = oracle_mod.Structure(p)
    a = st.export()
    rp, ci = a["row_ptr"], a["col_idx"]
    dis = np.zeros(p.n_elements, np.uint8)
    if outage is not None:
        dis[synthetic.outage_candidates(g)[outage]] = 1
    rng = np.random.default_rng(17)
    x = p.x_base.copy()
    x[0::2] += rng.uniform(-0.05, 0.05, p.n_bus)
    x[1::2] += rng.uniform(-0.03, 0.03, p.n_bus)
    vals, _ = st.fill(x, p.target, p.base_row_mode, dis)
    J = np.zeros((p.n, p.n))
    for r in range(p.n):
        J[r, ci[rp[r]:rp[r + 1]]] += vals[rp[r]:rp[r + 1]]
    h = 1e-6
    worst = 0.0
    for c in range(p.n):
        xp, xm = x.copy(), x.copy()
        xp[c] += h
        xm[c] -= h
        fd = (st.fill(xp, p.target, p.base_row_mode, dis)[1] - st.fill(xm, p.target, p.base_row_mode, dis)[1]) / (2 * h)
        worst = max(worst, float(np.max(np.abs(fd - J[:, c]) / np.maximum(np.abs(J[:, c]), 1.0))))
    assert worst < 1e-6, worst


def test_oracle_final_equations_after_reactive_limits(oracle_mod):
    """The oracle's per-scenario final equations (what the engine's targets / row-mode read-backs are checked
    against): rows that differ from the installed ones are reactive-limit voltage rows switched to an equation row at
    a Q limit (its target the limit less the load), and every converged state solves the equations it ended with."""
    from conftest import grid
    from olfgpu import synthetic
    g, p = grid("grid300")
    outs = synthetic.draw_outages(g, 40, seed=303)
    dis = p.outage_masks(outs)
    st = oracle_mod.Structure(p)
    rows, tg, md = st.solve_batch(p.x_base, dis, reactive_limits=True, final_equations=True)
    assert np.array_equal(rows, st.solve_batch(p.x_base, dis, reactive_limits=True))
    rl = p.rl
    switched = 0
    for k in range(outs.shape[0]):
        for r in np.flatnonzero((md[k] != p.base_row_mode) | (tg[k] != p.target)):
            i = np.flatnonzero(rl.voltage_row == r)
            assert i.size == 1 and md[k, r] == 1
            i = int(i[0])
            assert tg[k, r] in (rl.min_q[i] - rl.load_q[i], rl.max_q[i] - rl.load_q[i])
            switched += 1
        if rows[k, p.n + 2] == 0:
            _, F = st.fill(rows[k, :p.n], tg[k], md[k], dis[k])
            assert np.max(np.abs(F)) < 1e-8
    assert switched > 0
    plain, tg0, md0 = st.solve_batch(p.x_base, dis, final_equations=True)
    assert np.array_equal(md0, np.tile(p.base_row_mode, (outs.shape[0], 1)))
    assert np.array_equal(tg0, np.tile(p.target, (outs.shape[0], 1)))
