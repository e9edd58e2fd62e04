"""The engine's host structure (through the C ABI, no GPU needed) against the reference's own structure code."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def test_every_declaration_names_its_reference_interface():
    """Each entry point of include/olfgpu_b200.h is documented with the reference interface it replaces (a file:line
    citation) or says that it has no counterpart in the reference."""
    header = open(os.path.join(ROOT, "include", "olfgpu_b200.h")).read()
    last, missing = "", []
    for m in re.finditer(r"((?:/\*.*?\*/\s*)?)((?:const char\*|int)\s+(olfgpu_\w+)\s*\([^;]*\);)", header, re.S):
        if m.group(1).strip():
            last = m.group(1)
        if not (re.search(r"\w+\.(cu|cuh|java|h|cpp):\d+", last) or "no counterpart" in last.lower()):
            missing.append(m.group(3))
    assert not missing, missing


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
    with pytest.raises(native.NativeError, match="invalid batch solver context"):
        native._check(native.load().olfgpu_read_batch_targets(0, 0, None, None))
    with pytest.raises(native.NativeError, match="invalid batch solver context"):
        native._check(native.load().olfgpu_read_batch_row_modes(0, 0, None, None))
    s = native.Structure(p)
    with pytest.raises(native.NativeError, match="plantedFault"):
        native._check(native.load().olfgpu_structure_check_plan(s.handle, 7, None, None, 0))


@pytest.mark.parametrize("plan", ["scaled", "deferred", "dense", "shallow"])
def test_level_schedules_cover_every_block_once(engine_lib, plan):
    """The factorization levels hold every LU block exactly once with every block update, and the forward and
    backward solve levels every row (a dense-front plan leaves its front rows to the dense front's backward solve)."""
    from conftest import grid
    from olfgpu import native
    _, p = grid("grid2000")
    flag = {"scaled": 0, "deferred": native.PLAN_DEFERRED_L, "dense": native.PLAN_DENSE_FRONT,
            "shallow": native.PLAN_DEFAULT}[plan]
    s = native.Structure(p, flag)
    f, ops, fw, bw = s.levels()
    assert f[0] == 0 and f[-1] == s.n_lu_blocks and np.all(np.diff(f) > 0)
    assert int(ops.sum()) == s.block_ops
    assert fw[0] == 0 and fw[-1] == s.n_bus and np.all(np.diff(fw) > 0)
    assert bw[0] == 0 and np.all(np.diff(bw) > 0)
    front = s.n_bus - int(bw[-1])
    if plan in ("dense", "shallow"):
        assert 4 <= front <= 32
    else:
        assert front == 0


def test_plan_variants_shorten_the_dependency_chain(engine_lib):
    """The deferred-L plan advances about one level per pivot, the dense-front plan removes the root separators'
    levels: both have fewer factorization levels than the scaled plan of the same structure, with the same blocks."""
    from conftest import grid
    from olfgpu import native
    _, p = grid("grid2000")
    scaled = native.Structure(p)
    deferred = native.Structure(p, native.PLAN_DEFERRED_L)
    dense = native.Structure(p, native.PLAN_DENSE_FRONT)
    assert deferred.factor_levels < scaled.factor_levels
    assert dense.factor_levels < scaled.factor_levels
    assert scaled.n_lu_blocks == deferred.n_lu_blocks == dense.n_lu_blocks


@pytest.mark.parametrize("name", ["grid2000", "grid9241", "grid13659"])
def test_shallow_ordering_shortens_the_chain_at_about_the_same_fill(engine_lib, name):
    """Minimum degree relaxed toward a shallow elimination tree: fewer factorization and solve levels than plain
    minimum degree (with and without the dense front), at most 5 % more LU blocks."""
    from conftest import grid
    from olfgpu import native
    _, p = grid(name)
    md, sh = native.Structure(p, native.MIN_DEGREE), native.Structure(p, native.MIN_DEGREE_SHALLOW)
    dense, default = native.Structure(p, native.PLAN_DENSE_FRONT), native.Structure(p, native.PLAN_DEFAULT)
    assert sh.factor_levels < 0.85 * md.factor_levels
    assert default.factor_levels < 0.85 * dense.factor_levels
    assert default.forward_levels < dense.forward_levels and default.backward_levels < dense.backward_levels
    assert sh.n_lu_blocks <= 1.05 * md.n_lu_blocks
    again = native.Structure(p, native.MIN_DEGREE_SHALLOW)       # the order is deterministic
    assert all(np.array_equal(x, y) for x, y in zip(again.levels(), sh.levels()))


@pytest.mark.parametrize("name", ["grid2000", "grid9241", "grid13659"])
@pytest.mark.parametrize("plan", [0, 16])
def test_subtree_bins_keep_every_dependency(engine_lib, name, plan):
    """The subtree bins of the wide levels (schedule 5): every LU block and every position scheduled exactly once
    between the bins and the remaining level launches, and every block or solution entry a bin reads is produced
    before it (same bin on an earlier level, or an earlier phase); the check runs in the library on the host."""
    from olfgpu import native, packing, synthetic
    g = synthetic.build(name)
    s = native.Structure(packing.pack(g), ordering=plan)
    st = s.subtrees()
    assert st["bins"] > 0 and st["phases"] >= 1
    assert st["bin_blocks"] > 0.7 * s.n_lu_blocks          # most of the factorization moves into the bins
    assert st["max_bin_levels"] <= st["wide_levels"]


@pytest.mark.parametrize("name", ["grid118", "grid2000", "grid9241", "grid13659"])
@pytest.mark.parametrize("plan", [0, 3, 8, 11, 16, 19])
def test_block_plan_is_race_free(engine_lib, name, plan):
    """The host check of every block-LU plan variant (plain / shallow-tree minimum degree, scaled / deferred-L, with
    and without the dense front): the symbolic factorization is closed, every update list complete, every level task
    reads only blocks of strictly earlier levels, and both sweeps read only entries of strictly earlier levels, so no
    level launch shares data between its tasks.  A copy with one planted error of each kind fails the check."""
    from conftest import grid
    from olfgpu import native
    _, p = grid(name)
    s = native.Structure(p, ordering=plan)
    assert s.check_plan() == (0, "")
    moved, dropped, swapped = (s.check_plan(k) for k in (1, 2, 3))
    assert moved[0] > 0 and "level" in moved[1]
    assert dropped[0] > 0 and "update list" in dropped[1]
    assert swapped[0] > 0 and "forward" in swapped[1]


def test_tiny_and_empty_networks(engine_lib):
    """Edge inputs of the structure entry point are errors or sound plans, never crashes: an empty system, a network
    with no elements and a bus with only a shunt (a P row with no angle column: no diagonal pairing, the row map's rule)
    are refused with the reason; the smallest meshed case, two buses and one branch, plans under every variant and
    passes the plan check."""
    from olfgpu import native

    class _Net:
        def __init__(self, n, cb=(), sh=()):
            self.n = n
            self.cb_params = np.array([c[0] for c in cb], float).reshape(-1, 8)
            self.cb_idx = np.array([c[1] for c in cb], np.int32).reshape(-1, 12)
            self.ob_params, self.ob_idx = np.zeros((0, 7)), np.zeros((0, 6), np.int32)
            self.sh_params = np.array([s[0] for s in sh], float).reshape(-1, 2)
            self.sh_idx = np.array([s[1] for s in sh], np.int32).reshape(-1, 5)
            self.identity_rows = np.zeros(0, np.int32)
            self.n_cb, self.n_ob, self.n_sh = len(self.cb_idx), 0, len(self.sh_idx)
            self.n_elements = self.n_cb + self.n_sh

    with pytest.raises(native.NativeError, match="empty system"):
        native.Structure(_Net(0))
    with pytest.raises(native.NativeError, match="no diagonal pairing"):
        native.Structure(_Net(2))
    with pytest.raises(native.NativeError, match="no diagonal pairing"):
        native.Structure(_Net(2, sh=[([0.0, 0.1], [0, 1, 1, -1, -1])]))
    branch = ([10.0, 0.0, 0.0, 0.01, 0.01, 1.4, 1.0, 0.0], [0, 1, 2, 3, 0, 1, 2, 3, -1, -1, -1, -1])
    for plan in (0, native.PLAN_DEFERRED_L, native.PLAN_DEFAULT):
        s = native.Structure(_Net(4, cb=[branch]), ordering=plan)
        assert (s.n, s.nnz, s.n_lu_blocks) == (4, 16, 4)
        assert s.check_plan() == (0, "")
