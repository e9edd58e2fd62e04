"""The engine's host structure (through the C ABI, no GPU needed) against the reference's own structure code."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def test_library_exports_every_declared_symbol(engine_lib):
    header = open(os.path.join(ROOT, "include", "olfgpu_b200.h")).read()
    names = set(re.findall(r"\b(olfgpu_\w+)\s*\(", header))
    assert len(names) >= 13
    for name in names:
        assert hasattr(engine_lib, name), name


@pytest.mark.parametrize("name", ["grid118", "grid300"])
def test_engine_structure_matches_reference(engine_lib, name):
    from olfgpu import native
    from test_oracle import _P
    d = np.load(os.path.join(GOLD, f"structure_{name}.npz"))
    s = native.Structure(_P(d))
    a = s.export()
    for k in ("row_map", "row_ptr", "col_idx", "diag_pos", "cb_dest", "ob_dest", "sh_dest"):
        assert np.array_equal(a[k], d["ref_" + k]), k


@pytest.mark.parametrize("name", ["grid118", "grid2000"])
def test_engine_structure_matches_oracle(engine_lib, oracle_mod, name):
    from conftest import grid
    from olfgpu import native
    _, p = grid(name)
    a = native.Structure(p).export()
    b = oracle_mod.Structure(p).export()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_block_plan_statistics(engine_lib):
    from conftest import grid
    from olfgpu import native
    _, p = grid("grid2000")
    s = native.Structure(p)
    assert s.n_bus == 2000 and s.n == 4000
    # 2x2 blocks: the LU holds every A block plus fill-in, well under 3x the Jacobian for a transmission grid
    assert s.n_a_blocks * 4 >= s.nnz
    assert s.n_lu_blocks >= s.n_a_blocks
    assert s.n_lu_blocks * 4 < 3 * s.nnz
    assert s.factor_levels < 400 and s.forward_levels < 200


def test_bad_inputs_are_errors_not_crashes(engine_lib):
    from conftest import grid
    from olfgpu import native
    _, p = grid("grid118")
    import copy
    q = copy.copy(p)
    q.cb_idx = p.cb_idx.copy()
    q.cb_idx[3, 5] = p.n + 7
    with pytest.raises(native.NativeError, match="bad closedBranchIndices"):
        native.Structure(q)
    q.cb_idx = p.cb_idx.copy()
    q.cb_idx[0, 9] = 3
    with pytest.raises(native.NativeError, match="not supported"):
        native.Structure(q)
    with pytest.raises(native.NativeError, match="invalid structure handle"):
        native._check(native.load().olfgpu_structure_info(0, None, None))
