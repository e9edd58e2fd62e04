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
