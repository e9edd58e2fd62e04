"""The JNI layer (lib/libolfgpu.so) driven through a hand-built JNIEnv function table.

The table has the JNI specification's slot layout; Java arrays are numpy arrays behind opaque handles.  The tests
call the exported Java_com_powsybl_openloadflow_* symbols with the reference's argument lists (StructureNative.java,
BatchSolveNative.java, NewtonSettingsNative, ReactiveLimitsNative, DriverNative, BatchReadbackNative) and compare with
the engine's C ABI.  Structure creation, settings and error paths need no GPU; the solves do (marked gpu).
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import ROOT, grid

JNI_LIB = os.path.join(ROOT, "olf-gpu_b200", "lib", "libolfgpu.so")
PREFIX = "Java_com_powsybl_openloadflow_"
HOT_SET = [
    "ac_equations_vector_gpu_StructureNative_createStructure",
    "ac_equations_vector_gpu_StructureNative_destroyStructure",
    "ac_equations_vector_gpu_StructureNative_recommendBatchSize",
    "ac_solver_gpu_BatchSolveNative_createBatchContext",
    "ac_solver_gpu_BatchSolveNative_solveBatchContext",
    "ac_solver_gpu_BatchSolveNative_destroyBatchContext",
    "ac_solver_gpu_BatchSolveNative_setBatchStatesToHost",
    "ac_solver_gpu_BatchSolveNative_readBatchHandedBackSlots",
    "ac_solver_gpu_BatchSolveNative_beginBatchInstall",
    "ac_solver_gpu_NewtonSettingsNative_setLinearSolverSettings",
    "ac_solver_gpu_NewtonSettingsNative_readLinearSolverSettings",
    "ac_outerloop_gpu_ReactiveLimitsNative_setBatchReactiveLimitStrongestPvKeys",
    "ac_outerloop_gpu_ReactiveLimitsNative_setBatchRealisticCheck",
    "ac_solver_gpu_DriverNative_setBatchOuterLoops",
    "ac_solver_gpu_BatchReadbackNative_readBatchNewtonLoopIterations",
    "ac_solver_gpu_BatchReadbackNative_readBatchSolveCount",
    "ac_solver_gpu_BatchReadbackNative_readBatchTargets",
    "ac_solver_gpu_BatchReadbackNative_readBatchRowModes",
    "ac_solver_gpu_BatchReadbackNative_readBatchDistributedSlackGeneratorMove",
    "ac_solver_gpu_BatchReadbackNative_readBatchSlackRetainedShare",
    "ac_solver_gpu_BatchReadbackNative_readBatchSlackAbsorbed",
    "ac_solver_gpu_BatchReadbackNative_readBatchOuterLoopStats",
    "ac_solver_gpu_BatchReadbackNative_readBatchLastConvergedState",
    "ac_solver_gpu_NewtonSettingsNative_setBatchX0Seeds",
    "ac_solver_gpu_NewtonSettingsNative_setBatchRowCriteria",
    "ac_solver_gpu_NewtonSettingsNative_setBatchRowCriteriaAlternate",
    "ac_solver_gpu_NewtonSettingsNative_setBatchActiveRowCounts",
    "ac_solver_gpu_NewtonSettingsNative_setBatchFrozenRows",
    "ac_solver_gpu_NewtonSettingsNative_setBatchLineSearch",
    "ac_solver_gpu_NewtonSettingsNative_setBatchLoopTraceSlot",
    "ac_outerloop_gpu_DistributedSlackNative_setBatchDistributedSlackGeneratorAnchors",
    "ac_outerloop_gpu_DistributedSlackNative_setBatchSlackOnlyAnchor",
    "ac_outerloop_gpu_ReactiveLimitsNative_setBatchForcedTargetQPre",
    "ac_outerloop_gpu_ReactiveLimitsNative_setBatchReactiveLimitSeedTargetQ",
    "ac_outerloop_gpu_ReactiveLimitsNative_readBatchReactiveLimitsFinalState",
]

_vp, _i32, _i64, _f64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double


class FakeJvm:
    """A JNIEnv whose functions live in Python: arrays and classes are handles into a table of Python objects."""

    SLOTS = {"FindClass": 6, "ThrowNew": 14, "DeleteLocalRef": 23, "GetArrayLength": 171, "NewObjectArray": 172,
             "GetObjectArrayElement": 173, "SetObjectArrayElement": 174, "NewIntArray": 179, "NewDoubleArray": 182,
             "GetBooleanArrayRegion": 199, "GetByteArrayRegion": 200, "GetIntArrayRegion": 203,
             "GetDoubleArrayRegion": 206, "SetIntArrayRegion": 211, "SetDoubleArrayRegion": 214,
             "ExceptionCheck": 228}

    def __init__(self):
        self.objects = {}
        self.next = 0x1000
        self.exception = None
        self.calls = {k: 0 for k in self.SLOTS}
        cb = {
            "FindClass": ctypes.CFUNCTYPE(_vp, _vp, ctypes.c_char_p)(self._find_class),
            "ThrowNew": ctypes.CFUNCTYPE(_i32, _vp, _vp, ctypes.c_char_p)(self._throw_new),
            "DeleteLocalRef": ctypes.CFUNCTYPE(None, _vp, _vp)(self._delete),
            "GetArrayLength": ctypes.CFUNCTYPE(_i32, _vp, _vp)(self._length),
            "NewObjectArray": ctypes.CFUNCTYPE(_vp, _vp, _i32, _vp, _vp)(self._new_object_array),
            "GetObjectArrayElement": ctypes.CFUNCTYPE(_vp, _vp, _vp, _i32)(self._get_element),
            "SetObjectArrayElement": ctypes.CFUNCTYPE(None, _vp, _vp, _i32, _vp)(self._set_element),
            "NewIntArray": ctypes.CFUNCTYPE(_vp, _vp, _i32)(lambda e, n: self._new_array(np.zeros(n, np.int32))),
            "NewDoubleArray": ctypes.CFUNCTYPE(_vp, _vp, _i32)(lambda e, n: self._new_array(np.zeros(n))),
            "GetBooleanArrayRegion": ctypes.CFUNCTYPE(None, _vp, _vp, _i32, _i32, _vp)(self._get_region),
            "GetByteArrayRegion": ctypes.CFUNCTYPE(None, _vp, _vp, _i32, _i32, _vp)(self._get_region),
            "GetIntArrayRegion": ctypes.CFUNCTYPE(None, _vp, _vp, _i32, _i32, _vp)(self._get_region),
            "GetDoubleArrayRegion": ctypes.CFUNCTYPE(None, _vp, _vp, _i32, _i32, _vp)(self._get_region),
            "SetIntArrayRegion": ctypes.CFUNCTYPE(None, _vp, _vp, _i32, _i32, _vp)(self._set_region),
            "SetDoubleArrayRegion": ctypes.CFUNCTYPE(None, _vp, _vp, _i32, _i32, _vp)(self._set_region),
            "ExceptionCheck": ctypes.CFUNCTYPE(ctypes.c_uint8, _vp)(lambda e: 1 if self.exception else 0),
        }
        self._callbacks = cb
        self.table = (_vp * 235)()
        for name, idx in self.SLOTS.items():
            self.table[idx] = ctypes.cast(cb[name], _vp)
        self._table_ptr = _vp(ctypes.addressof(self.table))
        self.env = ctypes.pointer(self._table_ptr)       # JNIEnv*: points at the pointer to the table

    # -- objects -------------------------------------------------------------------------------------------------
    def _new(self, obj):
        h = self.next
        self.next += 16
        self.objects[h] = obj
        return h

    def _new_array(self, a):
        return self._new(a)

    def array(self, a, dtype):
        """A Java array of `a` (None: a null reference)."""
        return None if a is None else self._new(np.ascontiguousarray(a, dtype=dtype))

    def object_array(self, rows):
        return self._new([self._new(np.ascontiguousarray(r, dtype=np.uint8)) for r in rows])

    def value(self, h):
        return self.objects[h]

    # -- JNI functions -------------------------------------------------------------------------------------------
    def _find_class(self, env, name):
        return self._new(("class", name.decode()))

    def _throw_new(self, env, cls, msg):
        self.exception = (self.objects[cls][1], msg.decode())
        return 0

    def _delete(self, env, h):
        pass

    def _length(self, env, h):
        return len(self.objects[h])

    def _new_object_array(self, env, n, cls, init):
        return self._new([init] * n)

    def _get_element(self, env, h, i):
        return self.objects[h][i] or 0

    def _set_element(self, env, h, i, v):
        self.objects[h][i] = v

    def _get_region(self, env, h, start, n, buf):
        a = self.objects[h][start:start + n]
        ctypes.memmove(buf, a.ctypes.data, a.nbytes)

    def _set_region(self, env, h, start, n, buf):
        a = self.objects[h]
        ctypes.memmove(a[start:start + n].ctypes.data, buf, n * a.itemsize)

    def take_exception(self):
        e, self.exception = self.exception, None
        return e


@pytest.fixture(scope="module")
def jni(engine_lib):
    if not os.path.exists(JNI_LIB):
        from olfgpu import native  # noqa: F401  (the engine library is built by the engine_lib fixture)
        import importlib.util
        spec = importlib.util.spec_from_file_location("olfgpu_build", os.path.join(ROOT, "olf-gpu_b200", "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    return ctypes.CDLL(JNI_LIB)


def _fn(lib, name, restype, n_args):
    f = getattr(lib, PREFIX + name)
    f.restype = restype
    return f


def test_jni_library_exports_the_hot_set(jni):
    for name in HOT_SET:
        assert hasattr(jni, PREFIX + name), name


def test_readbacks_of_a_null_handle_are_null(jni):
    """BatchReadbackNative on handle 0 returns null without raising, as the reference's read-backs do
    (batch_readback_jni.cu:16-18, 36-38, 103-116); no GPU is touched."""
    jvm = FakeJvm()
    for name in ("readBatchTargets", "readBatchRowModes", "readBatchDistributedSlackGeneratorMove",
                 "readBatchSlackRetainedShare", "readBatchSlackAbsorbed", "readBatchOuterLoopStats"):
        f = _fn(jni, "ac_solver_gpu_BatchReadbackNative_" + name, _vp, 0)
        f.argtypes = [_vp, _vp, _i64]
        assert f(jvm.env, None, 0) is None
    f = _fn(jni, "ac_solver_gpu_BatchReadbackNative_readBatchLastConvergedState", _vp, 0)
    f.argtypes = [_vp, _vp, _i64, _i32]
    assert f(jvm.env, None, 0, 0) is None
    f = _fn(jni, "ac_outerloop_gpu_ReactiveLimitsNative_readBatchReactiveLimitsFinalState", _vp, 0)
    f.argtypes = [_vp, _vp, _i64]
    assert f(jvm.env, None, 0) is None
    for name, res in (("readBatchNewtonLoopIterations", _i32), ("readBatchSolveCount", _i64)):
        f = _fn(jni, "ac_solver_gpu_BatchReadbackNative_" + name, res, 0)
        f.argtypes = [_vp, _vp, _i64]
        assert f(jvm.env, None, 0) == -1
    assert jvm.take_exception() is None


def _create_structure(jni, jvm, p, extra=None):
    """StructureNative.createStructure with the reference's 33 array arguments; `extra` replaces some by name."""
    args = {"cbP": jvm.array(p.cb_params.reshape(-1), np.float64), "cbI": jvm.array(p.cb_idx.reshape(-1), np.int32),
            "obP": jvm.array(p.ob_params.reshape(-1), np.float64), "obI": jvm.array(p.ob_idx.reshape(-1), np.int32),
            "shP": jvm.array(p.sh_params.reshape(-1), np.float64), "shI": jvm.array(p.sh_idx.reshape(-1), np.int32)}
    names = ["cbP", "cbI", "obP", "obI", "shP", "shI", "hvdcP", "hvdcI", "dqE", "dqS", "dqW", "dqR", "dqK", "zibP",
             "zibI", "drR", "drC", "drK", "dbR", "dbC", "dbK", "phaseControlSide", "lmP", "lmI", "rrGroupStart",
             "rrCandidateRows", "obAltDest", "zibAltDest", "rrDepBaseGroup", "rrBaseTargetRow", "rrDepGroupOfRow",
             "identityRows"]
    args["phaseControlSide"] = jvm.array(-np.ones(p.n_cb), np.int32)
    args["rrGroupStart"] = jvm.array([0], np.int32)
    args["obAltDest"] = jvm.array(-np.ones(2 * p.n_ob), np.int32)
    args["identityRows"] = jvm.array(p.identity_rows, np.int32)
    for k, v in (extra or {}).items():
        args[k] = v
    f = _fn(jni, "ac_equations_vector_gpu_StructureNative_createStructure", _i64, 0)
    f.argtypes = [_vp, _vp, _i32] + [_vp] * len(names)
    return f(jvm.env, None, p.n, *[args.get(k) for k in names])


def test_create_structure_through_jni_matches_the_c_abi(jni):
    from olfgpu import native
    g, p = grid("grid118")
    jvm = FakeJvm()
    h = _create_structure(jni, jvm, p)
    assert jvm.take_exception() is None
    assert h != 0
    L = native.load()
    info = np.zeros(9, np.int32)
    ops = _i64(0)
    assert L.olfgpu_structure_info(h, info.ctypes.data_as(native._ip), ctypes.byref(ops)) == 0
    ref = native.Structure(p, ordering=native.PLAN_DEFAULT)
    assert info[0] == ref.n and info[1] == ref.nnz and info[3] == ref.n_lu_blocks and ops.value == ref.block_ops
    # the reference-compatible structure is the same whatever the plan
    ex = {k: np.zeros(ref.export()[k].shape, np.int32) for k in ("row_map", "row_ptr", "col_idx", "diag_pos")}
    L.olfgpu_structure_export(h, *[ex[k].ctypes.data_as(native._ip) for k in ("row_map", "row_ptr", "col_idx",
                                                                             "diag_pos")], None, None, None)
    for k, v in ex.items():
        assert np.array_equal(v, ref.export()[k]), k
    d = _fn(jni, "ac_equations_vector_gpu_StructureNative_destroyStructure", None, 0)
    d.argtypes = [_vp, _vp, _i64]
    d(jvm.env, None, h)
    d(jvm.env, None, 0)                                  # a handle of 0 is a no-op


@pytest.mark.parametrize("name,value", [
    ("hvdcI", np.arange(4)), ("dqE", np.arange(1)), ("zibI", np.zeros(11)), ("drR", np.arange(1)),
    ("lmI", np.zeros(2)), ("rrGroupStart", np.array([0, 2])), ("phaseControlSide", np.full(186, 3)),
])
def test_create_structure_rejects_unsupported_families(jni, name, value):
    g, p = grid("grid118")
    jvm = FakeJvm()
    arr = jvm.array(value, np.int32)
    h = _create_structure(jni, jvm, p, {name: arr})
    assert h == 0
    cls, msg = jvm.take_exception()
    assert cls == "java/lang/RuntimeException"
    assert "not supported" in msg


def test_linear_solver_settings_round_trip(jni):
    jvm = FakeJvm()
    s = _fn(jni, "ac_solver_gpu_NewtonSettingsNative_setLinearSolverSettings", None, 0)
    s.argtypes = [_vp, _vp, _i32, _i32, _i32, _f64, _i32, _i32, _f64, _i32, ctypes.c_uint8]
    s(jvm.env, None, 1, 2, 3, 0.5, 4, 5, 1e-9, 0, 1)
    r = _fn(jni, "ac_solver_gpu_NewtonSettingsNative_readLinearSolverSettings", _vp, 0)
    r.argtypes = [_vp, _vp]
    out = jvm.value(r(jvm.env, None))
    assert np.array_equal(out, [1, 2, 3, 0.5, 4, 5, 1e-9, 0, 1])


def _create_context(jni, jvm, s_handle, ns, rl=None, flags=None):
    f = _fn(jni, "ac_solver_gpu_BatchSolveNative_createBatchContext", _i64, 0)
    f.argtypes = [_vp, _vp, _i64, _i32, _i32] + [_vp] * 9 + [_i32, _f64] + [_vp] * 3 + [_i32] + [_vp] * 2 + [_f64] * 2
    a = [None] * 5
    if rl is not None:
        a = [jvm.array(rl.voltage_row, np.int32), jvm.array(rl.min_q, np.float64), jvm.array(rl.max_q, np.float64),
             jvm.array(rl.load_q, np.float64), jvm.array(rl.target_v, np.float64)]
    fl = jvm.array(flags, np.int8) if flags is not None else None
    return f(jvm.env, None, s_handle, ns, 7, *a, fl, None, None, None, -1, 0.0, None, None, None, 0, None, None, 0.0,
             0.0)


def test_create_context_rejects_monitoring_svc_flags(jni):
    g, p = grid("grid300")
    jvm = FakeJvm()
    h = _create_structure(jni, jvm, p)
    flags = np.zeros(p.rl.voltage_row.shape[0], np.int8)
    flags[1] = 1
    c = _create_context(jni, jvm, h, 4, rl=p.rl, flags=flags)
    assert c == 0
    assert "voltage-monitoring SVC" in jvm.take_exception()[1]


def _solve(jni, jvm, ctx, p, dis, x0_full=None, max_iter=15, tol=1e-8, unsupported=None):
    """BatchSolveNative.solveBatchContext with the reference's argument list."""
    f = _fn(jni, "ac_solver_gpu_BatchSolveNative_solveBatchContext", _vp, 0)
    f.argtypes = ([_vp, _vp, _i64] + [_vp] * 6 + [_vp] * 14 + [_i32, _f64, _f64, _f64, _f64, _i32, _f64, _f64] +
                  [_vp] * 7 + [_i32] * 5 + [_vp] * 2 + [_i32])
    ov = [None] * 13
    for k, v in (unsupported or {}).items():
        ov[k] = v
    h = f(jvm.env, None, ctx, jvm.array(p.x_base, np.float64), jvm.array(p.target, np.float64), None,
          jvm.array(p.base_row_mode, np.int32), jvm.object_array(dis), jvm.array(np.zeros(0), np.int32),
          jvm.array(np.zeros(0), np.float64), *ov, max_iter, tol, 1e-4, 1e-6, 0.0, 0, 0.1, 0.17, None,
          None if x0_full is None else jvm.array(x0_full.reshape(-1), np.float64), None, None, None, None, None, 20,
          3, 0, 0, 0, None, None, 0)
    if not h:
        return None
    return np.stack([jvm.value(r) for r in jvm.value(h)])


@pytest.mark.gpu
def test_solve_through_jni_equals_the_c_abi(jni):
    """createStructure -> createBatchContext -> setBatchReactiveLimitStrongestPvKeys -> solveBatchContext through the
    JNI table gives, bit for bit, what the engine's own entry gives on the same structure plan and schedule."""
    from olfgpu import native, synthetic
    g, p = grid("grid300")
    outs = synthetic.draw_outages(g, 40, seed=303)
    dis = p.outage_masks(outs)
    jvm = FakeJvm()
    sh = _create_structure(jni, jvm, p)
    ctx = _create_context(jni, jvm, sh, outs.shape[0], rl=p.rl)
    assert ctx != 0, jvm.take_exception()
    # without the forced-PV keys a solve with reactive-limit entries is refused (batch_solve_jni.cu:103-111)
    assert _solve(jni, jvm, ctx, p, dis) is None
    assert "forced-PV election keys" in jvm.take_exception()[1]
    keys = _fn(jni, "ac_outerloop_gpu_ReactiveLimitsNative_setBatchReactiveLimitStrongestPvKeys", None, 0)
    keys.argtypes = [_vp, _vp, _i64, _vp, _vp, _vp, _vp]
    r = p.rl
    keys(jvm.env, None, ctx, jvm.array(r.nom_v, np.float64), jvm.array(r.p_row, np.int32),
         jvm.array(r.static_p, np.float64), jvm.array(r.id_rank, np.int32))
    assert jvm.take_exception() is None
    got = _solve(jni, jvm, ctx, p, dis)
    assert got is not None, jvm.take_exception()
    s = native.Structure(p, ordering=native.PLAN_DEFAULT)
    c = native.BatchContext(s, outs.shape[0], rl=p.rl)
    c.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
    ref = c.solve(p.x_base, p.target, p.base_row_mode, dis)
    assert np.array_equal(got, ref)
    # the readbacks
    it = _fn(jni, "ac_solver_gpu_BatchReadbackNative_readBatchNewtonLoopIterations", _i32, 0)
    it.argtypes = [_vp, _vp, _i64]
    assert it(jvm.env, None, ctx) > 0
    cnt = _fn(jni, "ac_solver_gpu_BatchReadbackNative_readBatchSolveCount", _i64, 0)
    cnt.argtypes = [_vp, _vp, _i64]
    assert cnt(jvm.env, None, ctx) == 1
    # the per-scenario targets and row modes as the solve ended (the reactive-limit loop rewrote some), [scenarios x n]
    tg = _fn(jni, "ac_solver_gpu_BatchReadbackNative_readBatchTargets", _vp, 0)
    tg.argtypes = [_vp, _vp, _i64]
    rm = _fn(jni, "ac_solver_gpu_BatchReadbackNative_readBatchRowModes", _vp, 0)
    rm.argtypes = [_vp, _vp, _i64]
    targets = jvm.value(tg(jvm.env, None, ctx))
    modes = jvm.value(rm(jvm.env, None, ctx))
    assert jvm.take_exception() is None
    assert np.array_equal(targets.reshape(outs.shape[0], p.n), c.read_targets())
    assert np.array_equal(modes.reshape(outs.shape[0], p.n), c.read_row_modes())
    assert (modes.reshape(outs.shape[0], p.n) != p.base_row_mode).any()
    assert tg(jvm.env, None, 0) is None and rm(jvm.env, None, 0) is None
    # an unsupported override fails as a RuntimeException naming it
    bad = _solve(jni, jvm, ctx, p, dis, unsupported={0: jvm.array([1], np.int32)})
    assert bad is None and "distributedSlackOverrideBus" in jvm.take_exception()[1]
    d = _fn(jni, "ac_solver_gpu_BatchSolveNative_destroyBatchContext", None, 0)
    d.argtypes = [_vp, _vp, _i64]
    d(jvm.env, None, ctx)


@pytest.mark.gpu
def test_spi_path_settings_seeds_and_reactive_limit_state(jni):
    """The other native methods GpuNewtonRaphson / GpuBatchChunkSolver call on every run, through the JNI table on a
    reactive-limit context: the reactive-limit final state agrees with the row modes read back and with the C ABI; the
    settings clear on null and refuse inputs of families the engine does not model, naming them; start seeds
    (setBatchX0Seeds) equal a full per-scenario start through the C ABI and are consumed by that solve."""
    from olfgpu import native, synthetic
    g, p = grid("grid300")
    outs = synthetic.draw_outages(g, 40, seed=303)
    dis = p.outage_masks(outs)
    ns, n = outs.shape[0], p.n
    jvm = FakeJvm()
    sh = _create_structure(jni, jvm, p)
    ctx = _create_context(jni, jvm, sh, ns, rl=p.rl)
    assert ctx != 0, jvm.take_exception()
    keys = _fn(jni, "ac_outerloop_gpu_ReactiveLimitsNative_setBatchReactiveLimitStrongestPvKeys", None, 0)
    keys.argtypes = [_vp, _vp, _i64, _vp, _vp, _vp, _vp]
    r = p.rl
    keys(jvm.env, None, ctx, jvm.array(r.nom_v, np.float64), jvm.array(r.p_row, np.int32),
         jvm.array(r.static_p, np.float64), jvm.array(r.id_rank, np.int32))
    got = _solve(jni, jvm, ctx, p, dis)
    assert got is not None, jvm.take_exception()

    def call(cls, name, restype, argtypes, *args):
        f = _fn(jni, cls + "_" + name, restype, 0)
        f.argtypes = [_vp, _vp, _i64] + argtypes
        return f(jvm.env, None, ctx, *args)

    # the reactive-limit state: limit type in the low bits, switch count above; at a limit exactly where the entry's
    # voltage row was read back as an equation row
    st = jvm.value(call("ac_outerloop_gpu_ReactiveLimitsNative", "readBatchReactiveLimitsFinalState", _vp, []))
    nrl = r.voltage_row.shape[0]
    st = st.reshape(ns, nrl)
    modes = jvm.value(call("ac_solver_gpu_BatchReadbackNative", "readBatchRowModes", _vp, [])).reshape(ns, n)
    kind, switches = st & 7, st >> 3
    assert set(np.unique(kind).tolist()) <= {0, 1, 2} and (kind > 0).any() and (switches >= (kind > 0)).all()
    assert np.array_equal(kind > 0, modes[:, r.voltage_row] == 1)
    out = np.zeros((2, nrl), np.int32)
    cnt = ctypes.c_int(0)
    two = np.array([9, 4], np.int32)
    lib = native.load()
    assert lib.olfgpu_read_reactive_limits_state(ctx, 2, two.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                 ctypes.byref(cnt)) == 0
    assert cnt.value == nrl and np.array_equal(out, st[two])
    # settings: null clears, data of an unmodelled family is refused by name
    call("ac_solver_gpu_NewtonSettingsNative", "setBatchRowCriteria", None, [_vp, _vp], None, None)
    call("ac_outerloop_gpu_DistributedSlackNative", "setBatchDistributedSlackGeneratorAnchors", None,
         [_vp, _vp, _vp], None, jvm.array(np.zeros(0), np.float64), None)
    call("ac_solver_gpu_NewtonSettingsNative", "setBatchActiveRowCounts", None, [_vp],
         jvm.array(np.full(ns, n), np.int32))
    call("ac_outerloop_gpu_DistributedSlackNative", "setBatchSlackOnlyAnchor", None, [_vp],
         jvm.array(np.ones(ns), np.float64))
    assert jvm.take_exception() is None
    call("ac_solver_gpu_NewtonSettingsNative", "setBatchRowCriteria", None, [_vp, _vp],
         jvm.array(np.ones(n), np.float64), jvm.array(np.ones(n), np.float64))
    assert "per-equation-type" in jvm.take_exception()[1]
    call("ac_outerloop_gpu_DistributedSlackNative", "setBatchDistributedSlackGeneratorAnchors", None,
         [_vp, _vp, _vp], jvm.array(np.ones(ns), np.float64), None, None)
    assert "per-generator" in jvm.take_exception()[1]
    call("ac_solver_gpu_NewtonSettingsNative", "setBatchActiveRowCounts", None, [_vp],
         jvm.array(np.full(ns, n - 2), np.int32))
    assert "active equation count" in jvm.take_exception()[1]
    call("ac_solver_gpu_NewtonSettingsNative", "setBatchLineSearch", None, [_i32, _f64], 5, 0.5)
    assert "LINE_SEARCH" in jvm.take_exception()[1]
    for name in ("readBatchOuterLoopStats", "readBatchSlackAbsorbed", "readBatchSlackRetainedShare",
                 "readBatchDistributedSlackGeneratorMove"):
        assert call("ac_solver_gpu_BatchReadbackNative", name, _vp, []) is None
    # start seeds: two scenarios start off the base state; equal to the same start given in full through the C ABI,
    # and consumed by that solve (the next one starts from the base again)
    eq = np.flatnonzero(p.base_row_mode == 1)           # equation rows: their start moves the whole trajectory
    idx = np.array([3 * n + eq[1], 7 * n + eq[5]], np.int32)
    val = np.array([p.x_base[eq[1]] + 2e-3, p.x_base[eq[5]] - 2e-3])
    call("ac_solver_gpu_NewtonSettingsNative", "setBatchX0Seeds", None, [_vp, _vp], jvm.array(idx, np.int32),
         jvm.array(val, np.float64))
    seeded = _solve(jni, jvm, ctx, p, dis)
    assert seeded is not None, jvm.take_exception()
    full = np.tile(p.x_base, (ns, 1))
    full.reshape(-1)[idx] = val
    c = native.BatchContext(native.Structure(p, ordering=native.PLAN_DEFAULT), ns, rl=p.rl)
    c.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
    assert np.array_equal(seeded, c.solve(p.x_base, p.target, p.base_row_mode, dis, x0_full=full))
    assert not np.array_equal(seeded, got)
    assert np.array_equal(_solve(jni, jvm, ctx, p, dis), got)
    call("ac_solver_gpu_NewtonSettingsNative", "setBatchX0Seeds", None, [_vp, _vp], jvm.array([ns * n], np.int32),
         jvm.array([1.0], np.float64))
    assert _solve(jni, jvm, ctx, p, dis) is None and "setBatchX0Seeds index" in jvm.take_exception()[1]
    d = _fn(jni, "ac_solver_gpu_BatchSolveNative_destroyBatchContext", None, 0)
    d.argtypes = [_vp, _vp, _i64]
    d(jvm.env, None, ctx)


@pytest.mark.gpu
def test_bank_slots_and_states_left_on_the_device(jni):
    """beginBatchInstall puts the scenarios of a solve into chosen bank slots; the result rows come in installation
    order (readBatchHandedBackSlots), equal to solving those scenarios alone; with setBatchStatesToHost(false) the rows
    carry [iterations, norm, status] only."""
    from olfgpu import native, synthetic
    g, p = grid("grid118")
    outs = synthetic.outage_candidates(g)[:10]
    dis = p.outage_masks(outs)
    jvm = FakeJvm()
    sh = _create_structure(jni, jvm, p)
    ctx = _create_context(jni, jvm, sh, 16)
    begin = _fn(jni, "ac_solver_gpu_BatchSolveNative_beginBatchInstall", None, 0)
    begin.argtypes = [_vp, _vp, _i64, _vp]
    slots = np.array([7, 2, 15, 0, 9, 4, 11, 3, 8, 1], np.int32)
    begin(jvm.env, None, ctx, jvm.array(slots, np.int32))
    assert jvm.take_exception() is None
    got = _solve(jni, jvm, ctx, p, dis)
    assert got is not None, jvm.take_exception()
    hb = _fn(jni, "ac_solver_gpu_BatchSolveNative_readBatchHandedBackSlots", _vp, 0)
    hb.argtypes = [_vp, _vp, _i64]
    assert np.array_equal(jvm.value(hb(jvm.env, None, ctx)), slots)
    alone = native.BatchContext(native.Structure(p, ordering=native.PLAN_DEFAULT), 10)
    alone.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
    ref = alone.solve(p.x_base, p.target, p.base_row_mode, dis)
    assert np.array_equal(got, ref)
    # a slot twice is refused
    begin(jvm.env, None, ctx, jvm.array([1, 1], np.int32))
    assert "installed twice" in jvm.take_exception()[1]
    # states left on the device: rows of three
    sth = _fn(jni, "ac_solver_gpu_BatchSolveNative_setBatchStatesToHost", None, 0)
    sth.argtypes = [_vp, _vp, _i64, ctypes.c_uint8]
    sth(jvm.env, None, ctx, 0)
    begin(jvm.env, None, ctx, jvm.array(slots, np.int32))
    tails = _solve(jni, jvm, ctx, p, dis)
    assert tails.shape == (10, 3)
    assert np.array_equal(tails, ref[:, -3:])
