import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "olf-gpu_b200"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built engine library")


@pytest.fixture(scope="session")
def engine_lib():
    """The engine library (built in-tree when missing; loading it needs no GPU)."""
    from olfgpu import native
    if not os.path.exists(native.LIB_PATH):
        import importlib.util
        spec = importlib.util.spec_from_file_location("olfgpu_build", os.path.join(ROOT, "olf-gpu_b200", "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    return native.load()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    if not os.path.exists(O.LIB):
        O.build()
    return O


_GRIDS = {}


def grid(name):
    """A synthetic grid and its packed arrays, generated once per session."""
    if name not in _GRIDS:
        from olfgpu import packing, synthetic
        g = synthetic.build(name)
        _GRIDS[name] = (g, packing.pack(g))
    return _GRIDS[name]


_ORACLE_ROWS = {}


def oracle_rows(oracle_mod, name, x0, disabled):
    """The oracle's batched solve (no outer loops, default settings) of a grid's scenarios, memoised per session:
    the parametrizations of one parity test solve the same scenarios, and the oracle's rows depend only on them."""
    import hashlib
    import numpy as np
    x0 = np.ascontiguousarray(x0, dtype=np.float64)
    disabled = np.ascontiguousarray(disabled, dtype=np.uint8)
    key = (name, hashlib.sha1(x0.tobytes()).hexdigest(), hashlib.sha1(disabled.tobytes()).hexdigest(), disabled.shape)
    if key not in _ORACLE_ROWS:
        _ORACLE_ROWS[key] = oracle_mod.Structure(grid(name)[1]).solve_batch(x0, disabled)
    return _ORACLE_ROWS[key].copy()
