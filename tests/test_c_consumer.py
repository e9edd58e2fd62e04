"""The C ABI from plain C: tests/c/structure_consumer.c, compiled with gcc against include/olfgpu_b200.h alone and
linked with the engine library, drives the host-only entry points (structure creation, sizes, the block-LU plan
check, the pattern export, the error path) as a cgo / JNI / FFI binding would, and agrees with the Python binding.
No GPU is needed."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, grid

SRC = os.path.join(ROOT, "tests", "c", "structure_consumer.c")


def _write_network(path, p):
    with open(path, "wb") as f:
        np.array([p.n, p.n_cb, p.n_ob, p.n_sh, p.identity_rows.shape[0]], np.int32).tofile(f)
        for a, t in ((p.cb_params, np.float64), (p.cb_idx, np.int32), (p.ob_params, np.float64), (p.ob_idx, np.int32),
                     (p.sh_params, np.float64), (p.sh_idx, np.int32), (p.identity_rows, np.int32)):
            np.ascontiguousarray(a, dtype=t).tofile(f)


@pytest.mark.parametrize("name", ["grid118", "grid2000"])
def test_c_program_drives_the_structure_entry_points(engine_lib, tmp_path, name):
    from olfgpu import native
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    lib_dir = os.path.dirname(native.LIB_PATH)
    exe = str(tmp_path / "consumer")
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
                           "-L", lib_dir, "-lolfgpu_b200", "-Wl,-rpath," + lib_dir, "-o", exe])
    _, p = grid(name)
    net = str(tmp_path / "net.bin")
    _write_network(net, p)
    # the CUDA runtime the engine library links, where this process loaded it from
    env = dict(os.environ)
    with open("/proc/self/maps") as maps:
        dirs = {os.path.dirname(line.split()[-1]) for line in maps if "libcudart.so" in line}
    env["LD_LIBRARY_PATH"] = os.pathsep.join(sorted(dirs) + [env.get("LD_LIBRARY_PATH", "")])
    out = subprocess.run([exe, net], capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0, out.stderr
    n, nnz, buses, lu_blocks, levels, violations, checksum = (int(v) for v in out.stdout.split())
    s = native.Structure(p, ordering=native.PLAN_DEFAULT)
    a = s.export()
    expect = int(sum(int(k % 97 + 1) * int(c) for k, c in enumerate(a["col_idx"]))) + int(a["row_ptr"].sum())
    assert (n, nnz, buses, lu_blocks, levels) == (p.n, s.nnz, s.n_bus, s.n_lu_blocks, s.factor_levels)
    assert violations == 0
    assert checksum == expect
