"""ctypes binding of the engine's C ABI (``include/olfgpu_b200.h``), shaped like the reference's Java facades
(``StructureNative``, ``BatchSolveNative``, ``NewtonSettingsNative``).

The binding loads ``lib/libolfgpu_b200.so`` built in-tree; there is no fallback: a missing library is an error.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "lib", "libolfgpu_b200.so")

# Linear-solve modes (codes/gpu_linear_solve_mode.cuh:10-12)
UBATCH, ROBUST, BATCHED_LU = 3, 6, 7
# Statuses (codes/gpu_ac_solver_status.cuh:10-15)
CONVERGED, MAX_ITERATION_REACHED, UNREALISTIC_STATE = 0, 1, 2
DIVERGED, REJECTED, LINEAR_SOLVE_FAILED = -1, -2, -3
STATUS_NAMES = {0: "CONVERGED", 1: "MAX_ITERATION_REACHED", 2: "UNREALISTIC_STATE", -1: "DIVERGED", -2: "REJECTED",
                -3: "LINEAR_SOLVE_FAILED"}
# Precision of the linear solves
FP64, MIXED = 0, 1

_i64 = ctypes.c_int64
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_fp = ctypes.POINTER(ctypes.c_float)

EXPORTS = ["olfgpu_last_error", "olfgpu_create_structure", "olfgpu_destroy_structure", "olfgpu_structure_info",
           "olfgpu_structure_export", "olfgpu_recommend_batch_size", "olfgpu_create_batch_context",
           "olfgpu_destroy_batch_context", "olfgpu_set_linear_solver_settings", "olfgpu_solve_batch_context",
           "olfgpu_last_solve_stats", "olfgpu_debug_fill", "olfgpu_debug_linear_solve", "olfgpu_set_schedule",
           "olfgpu_get_schedule", "olfgpu_linear_solve_noalloc", "olfgpu_stage_batch_context",
           "olfgpu_create_multi_context", "olfgpu_destroy_multi_context", "olfgpu_set_multi_schedule",
           "olfgpu_get_multi_schedule", "olfgpu_solve_multi_context", "olfgpu_set_fallback_start",
           "olfgpu_last_fallbacks", "olfgpu_set_phase_timing", "olfgpu_last_phase_times", "olfgpu_structure_levels",
           "olfgpu_set_device_start", "olfgpu_set_mixed_precision_controls", "olfgpu_last_fp64_refactors",
           "olfgpu_solve_batch_context_full", "olfgpu_set_realistic_check", "olfgpu_set_refinement_bound",
           "olfgpu_set_fp64_restart", "olfgpu_structure_subtrees", "olfgpu_create_structure_full",
           "olfgpu_create_batch_context_full", "olfgpu_set_reactive_limit_strongest_pv_keys",
           "olfgpu_begin_batch_install", "olfgpu_read_handed_back_slots", "olfgpu_set_states_to_host",
           "olfgpu_states_to_host", "olfgpu_read_batch_states", "olfgpu_set_outer_loops", "olfgpu_context_info",
           "olfgpu_linear_solve_transposed", "olfgpu_screen_violations", "olfgpu_last_slack_distribution_failures",
           "olfgpu_set_start_polish", "olfgpu_set_mixed_precision_policy", "olfgpu_last_fp64_iterations",
           "olfgpu_set_device_loop", "olfgpu_read_batch_targets", "olfgpu_read_batch_row_modes",
           "olfgpu_structure_check_plan", "olfgpu_read_reactive_limits_state"]
# The arrays of BatchSolveNative.solveBatchContext this engine rejects when non-empty, in the reference's order
UNSUPPORTED_SOLVE_ARRAYS = [
    "distributedSlackOverrideBus", "distributedSlackOverrideFactorDelta", "distributedSlackOverrideBaseTargetPDelta",
    "distributedSlackOverrideMaxDelta", "distributedSlackOverrideMinDelta", "distributedSlackBusAnchorShift",
    "slackBusAnchorShift", "reactiveLimitTargetVOverrideScenarioEntry", "reactiveLimitTargetVOverrideValue",
    "reactiveLimitDeltaOverrideScenarioEntry", "reactiveLimitDeltaOverrideValues",
    "reactiveCapabilityCurveOverrideScenarioCurve", "reactiveCapabilityCurveOverrideStepScale"]
_INT_SOLVE_ARRAYS = {"distributedSlackOverrideBus", "reactiveLimitTargetVOverrideScenarioEntry",
                     "reactiveLimitDeltaOverrideScenarioEntry", "reactiveCapabilityCurveOverrideScenarioCurve"}
# State-vector scaling modes (codes/gpu_state_vector_scaling_mode.cuh) and variable types (gpu_ac_variable_type.cuh)
SVS_NONE, SVS_LINE_SEARCH, SVS_MAX_VOLTAGE_CHANGE = 0, 1, 2
MIXED_REFINE, MIXED_FP64_NEAR = 0, 1
VAR_BUS_V, VAR_BUS_PHI = 0, 1
# Schedules of the Newton iterations (LEVELS_SHARED: the level schedule with the narrow factorization levels in
# shared memory; LEVELS_SHARED_ALL: the solves' narrow levels too; SUBTREES: LEVELS_SHARED_ALL with the wide levels'
# independent subtrees in one launch per phase)
LEVELS, PERSISTENT, COOPERATIVE, LEVELS_SHARED, LEVELS_SHARED_ALL, SUBTREES, AUTOTUNE = 0, 1, 2, 3, 4, 5, -1
# Structure orderings (0 minimum degree, 1 nested dissection, 2 natural) and the deferred-L plan flag
MIN_DEGREE, NESTED_DISSECTION, NATURAL, MIN_DEGREE_SHALLOW, PLAN_DEFERRED_L, PLAN_DENSE_FRONT = 0, 1, 2, 3, 8, 16
# The fastest measured plan: minimum degree relaxed toward a shallow elimination tree, with the dense front
PLAN_DEFAULT = PLAN_DENSE_FRONT | MIN_DEGREE_SHALLOW


class NativeError(RuntimeError):
    pass


_lib = None


def load(path: str = LIB_PATH):
    """Load the engine library (no fallback: raises when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise NativeError(f"engine library not built: {path} (run olf-gpu_b200/build.py)")
    L = ctypes.CDLL(path)
    L.olfgpu_last_error.restype = ctypes.c_char_p
    L.olfgpu_create_structure.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _ip, ctypes.c_int, _dp, _ip, ctypes.c_int,
                                          _dp, _ip, ctypes.c_int, _ip, ctypes.c_int, ctypes.POINTER(_i64)]
    L.olfgpu_destroy_structure.argtypes = [_i64]
    L.olfgpu_structure_info.argtypes = [_i64, _ip, ctypes.POINTER(_i64)]
    L.olfgpu_structure_export.argtypes = [_i64, _ip, _ip, _ip, _ip, _ip, _ip, _ip]
    L.olfgpu_recommend_batch_size.argtypes = [_i64, ctypes.c_int, ctypes.c_int, _ip]
    L.olfgpu_create_batch_context.argtypes = [_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip, _dp, _dp, _dp, _dp,
                                              _dp, _ip, _dp, _ip, ctypes.POINTER(_i64)]
    L.olfgpu_destroy_batch_context.argtypes = [_i64]
    L.olfgpu_set_linear_solver_settings.argtypes = [_i64, ctypes.c_int, ctypes.c_int]
    L.olfgpu_solve_batch_context.argtypes = [_i64, _dp, _dp, _dp, _ip, ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int,
                                             _u8p, ctypes.c_int, _ip, _dp, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_int, ctypes.c_int, _dp]
    L.olfgpu_stage_batch_context.argtypes = L.olfgpu_solve_batch_context.argtypes[:-1]
    _ci, _cd = ctypes.c_int, ctypes.c_double
    L.olfgpu_solve_batch_context_full.argtypes = (
        [_i64, _dp, _ci, _dp, _ci, _ip, _ci, _ip, _ci, _u8p, _ci, _ci, _ip, _ci, _dp, _ci,
         _ip, _ci, _dp, _ci, _dp, _ci, _dp, _ci, _dp, _ci, _dp, _ci, _dp, _ci,    # distributed-slack overrides
         _ip, _ci, _dp, _ci, _ip, _ci, _dp, _ci, _ip, _ci, _dp, _ci,              # reactive-limit overrides
         _ci, _cd, _cd, _cd, _cd, _ci, _cd, _cd, _ip, _ci, _dp, _ci,
         _ip, _ci, _dp, _ci, _ip, _ci, _ip, _ci, _dp, _ci,
         _ci, _ci, _ci, _ci, _ci, _ip, _ci, _ip, _ci, _ci, _dp])
    L.olfgpu_create_batch_context_full.argtypes = (
        [_i64, _ci, _ci, _ip, _ci, _dp, _ci, _dp, _ci, _dp, _ci, _dp, _ci, ctypes.POINTER(ctypes.c_byte), _ci, _dp, _ci,
         _ip, _ci, _dp, _ci, _ci, _cd, _dp, _ci, _dp, _ci, _dp, _ci, _ci, _dp, _ci, _dp, _ci, _cd, _cd,
         ctypes.POINTER(_i64)])
    L.olfgpu_last_slack_distribution_failures.argtypes = [_i64, _u8p, _ip]
    L.olfgpu_set_reactive_limit_strongest_pv_keys.argtypes = [_i64, _dp, _ip, _dp, _ip, _ci]
    L.olfgpu_set_realistic_check.argtypes = [_i64, _u8p, _cd, _cd, _ci]
    L.olfgpu_set_refinement_bound.argtypes = [_i64, _cd]
    L.olfgpu_set_fp64_restart.argtypes = [_i64, _ci]
    L.olfgpu_set_start_polish.argtypes = [_i64, _cd]
    L.olfgpu_set_mixed_precision_policy.argtypes = [_i64, _ci]
    L.olfgpu_set_device_loop.argtypes = [_i64, _ci]
    L.olfgpu_last_fp64_iterations.argtypes = [_i64, _ip]
    L.olfgpu_structure_subtrees.argtypes = [_i64, ctypes.POINTER(_i64)]
    L.olfgpu_linear_solve_transposed.argtypes = [_i64, _dp, _dp, _dp, _ci, _dp, _dp]
    L.olfgpu_screen_violations.argtypes = [_i64, _ci, _ip, _ip, _ip, _ip, _ip, _dp, _ci, _ip, _dp, _dp, _ci, _cd, _cd,
                                           _cd, _ci, _ip, _ip]
    L.olfgpu_read_batch_states.argtypes = [_i64, _ci, _ip, _dp]
    L.olfgpu_read_batch_targets.argtypes = [_i64, _ci, _ip, _dp]
    L.olfgpu_read_reactive_limits_state.argtypes = [_i64, _ci, _ip, _ip, _ip]
    L.olfgpu_structure_check_plan.argtypes = [_i64, _ci, ctypes.POINTER(_i64), ctypes.c_char_p, _ci]
    L.olfgpu_read_batch_row_modes.argtypes = [_i64, _ci, _ip, _ip]
    L.olfgpu_begin_batch_install.argtypes = [_i64, _ip, _ci]
    L.olfgpu_read_handed_back_slots.argtypes = [_i64, _ip, _ci, _ip]
    L.olfgpu_set_states_to_host.argtypes = [_i64, _ci]
    L.olfgpu_states_to_host.argtypes = [_i64, _ip]
    L.olfgpu_set_outer_loops.argtypes = [_i64, _ci, _ci]
    L.olfgpu_context_info.argtypes = [_i64, _ip, _ip, _ip, _ip, _ip, ctypes.POINTER(_i64)]
    L.olfgpu_create_multi_context.argtypes = [ctypes.c_int, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]
    L.olfgpu_destroy_multi_context.argtypes = [_i64]
    L.olfgpu_set_multi_schedule.argtypes = [_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.olfgpu_get_multi_schedule.argtypes = [_i64, _ip, _ip, _ip, ctypes.c_int, _dp, _ip]
    L.olfgpu_solve_multi_context.argtypes = [_i64, ctypes.POINTER(_dp), _fp]
    L.olfgpu_structure_levels.argtypes = [_i64, _ip, _ip, _ip, ctypes.POINTER(_i64)]
    L.olfgpu_set_phase_timing.argtypes = [_i64, ctypes.c_int]
    L.olfgpu_last_phase_times.argtypes = [_i64, _dp]
    L.olfgpu_set_fallback_start.argtypes = [_i64, ctypes.c_int]
    L.olfgpu_set_device_start.argtypes = [_i64, ctypes.c_void_p]
    L.olfgpu_set_mixed_precision_controls.argtypes = [_i64, ctypes.c_double, ctypes.c_double]
    L.olfgpu_last_fp64_refactors.argtypes = [_i64, _u8p, _ip]
    L.olfgpu_last_fallbacks.argtypes = [_i64, _u8p, _ip]
    L.olfgpu_last_solve_stats.argtypes = [_i64, _fp, _ip, _ip]
    L.olfgpu_debug_fill.argtypes = [_i64, _dp, _dp, _ip, _u8p, _dp, _dp]
    L.olfgpu_debug_linear_solve.argtypes = [_i64, _dp, _dp, ctypes.c_int, _dp]
    L.olfgpu_set_schedule.argtypes = [_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.olfgpu_get_schedule.argtypes = [_i64, _ip, _ip, _ip, ctypes.c_int, _dp, _ip]
    L.olfgpu_linear_solve_noalloc.argtypes = [_i64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_int, ctypes.c_void_p]
    for name in EXPORTS:
        getattr(L, name).restype = ctypes.c_char_p if name == "olfgpu_last_error" else ctypes.c_int
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        raise NativeError(load().olfgpu_last_error().decode())


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _p(a):
    if a is None:
        return None
    if a.dtype == np.float64:
        return a.ctypes.data_as(_dp)
    if a.dtype == np.int32:
        return a.ctypes.data_as(_ip)
    if a.dtype == np.uint8:
        return a.ctypes.data_as(_u8p)
    if a.dtype == np.float32:
        return a.ctypes.data_as(_fp)
    raise TypeError(a.dtype)


class Structure:
    """StructureNative: the shared structure built once per packed network."""

    def __init__(self, packed, ordering: int = 0):
        L = load()
        self.packed = packed
        keep = [_c(packed.cb_params, np.float64), _c(packed.cb_idx, np.int32), _c(packed.ob_params, np.float64),
                _c(packed.ob_idx, np.int32), _c(packed.sh_params, np.float64), _c(packed.sh_idx, np.int32),
                _c(packed.identity_rows, np.int32)]
        h = _i64(0)
        _check(L.olfgpu_create_structure(packed.n, packed.n_cb, _p(keep[0]), _p(keep[1]), packed.n_ob, _p(keep[2]),
                                         _p(keep[3]), packed.n_sh, _p(keep[4]), _p(keep[5]), keep[6].shape[0],
                                         _p(keep[6]), ordering, ctypes.byref(h)))
        self.handle = h.value
        info = np.zeros(9, np.int32)
        ops = _i64(0)
        _check(L.olfgpu_structure_info(self.handle, _p(info), ctypes.byref(ops)))
        (self.n, self.nnz, self.n_bus, self.n_lu_blocks, self.factor_levels, self.forward_levels,
         self.backward_levels, self.n_elements, self.n_a_blocks) = [int(v) for v in info]
        self.block_ops = int(ops.value)

    def close(self):
        if getattr(self, "handle", 0):
            load().olfgpu_destroy_structure(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def export(self):
        p = self.packed
        out = dict(row_map=np.zeros(self.n, np.int32), row_ptr=np.zeros(self.n + 1, np.int32),
                   col_idx=np.zeros(self.nnz, np.int32), diag_pos=np.zeros(self.n, np.int32),
                   cb_dest=np.zeros(p.n_cb * 28, np.int32), ob_dest=np.zeros(p.n_ob * 8, np.int32),
                   sh_dest=np.zeros(p.n_sh * 5, np.int32))
        _check(load().olfgpu_structure_export(self.handle, *[_p(out[k]) for k in (
            "row_map", "row_ptr", "col_idx", "diag_pos", "cb_dest", "ob_dest", "sh_dest")]))
        return out

    def levels(self):
        """Block-LU schedule: (factor level pointers, block updates per factor level, forward / backward level
        pointers)."""
        f = np.zeros(self.factor_levels + 1, np.int32)
        fw = np.zeros(self.forward_levels + 1, np.int32)
        bw = np.zeros(self.backward_levels + 1, np.int32)
        ops = np.zeros(self.factor_levels, np.int64)
        _check(load().olfgpu_structure_levels(self.handle, _p(f), _p(fw), _p(bw),
                                              ops.ctypes.data_as(ctypes.POINTER(_i64))))
        return f, ops, fw, bw

    def subtrees(self) -> dict:
        """The subtree bins of the wide levels (schedule SUBTREES), planned and checked on the host."""
        st = (_i64 * 6)()
        _check(load().olfgpu_structure_subtrees(self.handle, st))
        return {"bins": int(st[0]) // 100, "phases": int(st[0]) % 100, "bin_blocks": int(st[1]),
                "max_bin_levels": int(st[2]), "top_wide_blocks": int(st[3]), "bin_positions": int(st[4]),
                "wide_levels": int(st[5])}

    def check_plan(self, planted_fault: int = 0):
        """(violations, first violation) of the host check of the block-LU plan: closure of the symbolic
        factorization, every level task reading only blocks of strictly earlier levels, both sweeps likewise.
        planted_fault 1..3 checks a copy with one planted error (tests of the check itself)."""
        v = _i64(0)
        msg = ctypes.create_string_buffer(512)
        _check(load().olfgpu_structure_check_plan(self.handle, planted_fault, ctypes.byref(v), msg, 512))
        return int(v.value), msg.value.decode()

    def recommend_batch_size(self, max_cap: int, mode: int = BATCHED_LU) -> int:
        b = ctypes.c_int(0)
        _check(load().olfgpu_recommend_batch_size(self.handle, max_cap, mode, ctypes.byref(b)))
        return int(b.value)

    def linear_solve_noalloc(self, n_scenarios: int, csr_vals_ptr: int, rhs_ptr: int, out_ptr: int,
                             precision: int = FP64, stream: int = 0):
        """olfgpu_linear_solve_noalloc on caller-owned device buffers (raw device addresses); enqueues and returns."""
        _check(load().olfgpu_linear_solve_noalloc(self.handle, n_scenarios, ctypes.c_void_p(csr_vals_ptr),
                                                  ctypes.c_void_p(rhs_ptr), ctypes.c_void_p(out_ptr), precision,
                                                  ctypes.c_void_p(stream)))

    @property
    def lu_bytes_per_scenario(self) -> int:
        return self.n_lu_blocks * 4 * 8


class BatchContext:
    """BatchSolveNative: a bank of ``n_scenarios`` lanes on one structure."""

    def __init__(self, structure: Structure, n_scenarios: int, mode: int = BATCHED_LU, rl=None, ds=None):
        """``rl``: reactive-limit tables (packing.ReactiveLimits); ``ds``: bus-level distributed-slack participants
        (packing.DistributedSlack, static factors), which go through olfgpu_create_batch_context_full."""
        L = load()
        self.structure = structure
        self.n_scenarios = n_scenarios
        h = _i64(0)
        if ds is not None:
            self._ds = [_c(ds.row, np.int32), _c(ds.factor, np.float64), _c(ds.base_target, np.float64),
                        _c(ds.max_delta, np.float64), _c(ds.min_delta, np.float64)]
            d = self._ds
            nd = int(d[0].size)
            if rl is not None:
                self._rl = [_c(rl.voltage_row, np.int32), _c(rl.min_q, np.float64), _c(rl.max_q, np.float64),
                            _c(rl.load_q, np.float64), _c(rl.target_v, np.float64)]
                r = self._rl
                nr = int(r[0].size)
                rl_args = [_p(r[0]), nr, _p(r[1]), nr, _p(r[2]), nr, _p(r[3]), nr, _p(r[4]), nr]
            else:
                rl_args = [None, 0] * 5
            _check(L.olfgpu_create_batch_context_full(
                structure.handle, n_scenarios, mode, *rl_args, None, 0, None, 0,
                _p(d[0]), nd, _p(d[1]), nd, int(ds.slack_row), float(ds.slack_target_p), _p(d[2]), nd, _p(d[3]), nd,
                _p(d[4]), nd, 0, None, 0, None, 0, 0.0, 0.0, ctypes.byref(h)))
            self.handle = h.value
            if rl is not None:       # ReactiveLimitsNative.setBatchReactiveLimitStrongestPvKeys
                self._keys = [_c(rl.nom_v, np.float64), _c(rl.p_row, np.int32), _c(rl.static_p, np.float64),
                              _c(rl.id_rank, np.int32)]
                k = self._keys
                _check(L.olfgpu_set_reactive_limit_strongest_pv_keys(self.handle, _p(k[0]), _p(k[1]), _p(k[2]),
                                                                      _p(k[3]), int(k[0].size)))
            return
        if rl is not None:
            self._rl = [_c(rl.voltage_row, np.int32), _c(rl.min_q, np.float64), _c(rl.max_q, np.float64),
                        _c(rl.load_q, np.float64), _c(rl.target_v, np.float64), _c(rl.nom_v, np.float64),
                        _c(rl.p_row, np.int32), _c(rl.static_p, np.float64), _c(rl.id_rank, np.int32)]
            r = self._rl
            _check(L.olfgpu_create_batch_context(structure.handle, n_scenarios, mode, r[0].shape[0], *[_p(a) for a in r],
                                                 ctypes.byref(h)))
        else:
            _check(L.olfgpu_create_batch_context(structure.handle, n_scenarios, mode, 0, None, None, None, None, None,
                                                 None, None, None, None, ctypes.byref(h)))
        self.handle = h.value

    def close(self):
        if getattr(self, "handle", 0):
            load().olfgpu_destroy_batch_context(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_linear_solver_settings(self, precision: int = FP64, refinement_steps: int = 1):
        _check(load().olfgpu_set_linear_solver_settings(self.handle, precision, refinement_steps))

    def set_schedule(self, schedule: int, lanes_per_tile: int = 2, threads: int = 512):
        _check(load().olfgpu_set_schedule(self.handle, schedule, lanes_per_tile, threads))

    def schedule(self):
        """(schedule, lanes per tile, threads) in force and the autotuner's timings [(schedule, lanes, threads, ms)]."""
        sc, la, th, nr = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        res = np.zeros(4 * 32)
        _check(load().olfgpu_get_schedule(self.handle, ctypes.byref(sc), ctypes.byref(la), ctypes.byref(th), 32,
                                          _p(res), ctypes.byref(nr)))
        tuning = [tuple(res[4 * i:4 * i + 4]) for i in range(min(nr.value, 32))]
        return (sc.value, la.value, th.value), tuning

    def solve(self, x0_base, target_base, base_row_mode, disabled, x0_full=None, row_mode_entries=None,
              target_override_index=None, target_override_value=None, max_iter: int = 15, tol: float = 1e-8,
              reactive_limit_tol: float = 1e-4, max_outer: int = 20, max_pq_pv_switch: int = 3,
              out: Optional[np.ndarray] = None, conv_eps_per_eq: float = 0.0, svs_mode: int = SVS_NONE,
              max_dv: float = 0.1, max_dphi: float = 0.17453292519943295, var_type=None,
              skip_reactive_limits: bool = False, unsupported: Optional[dict] = None,
              pause_at_ended: int = 0, slack_dist_tol: float = 1e-6,
              reject_slack_distribution_failure: bool = False) -> np.ndarray:
        """Per scenario [x(n), iterations, ||F||inf, status] through the full reference-shaped entry
        (BatchSolveNative.solveBatchContext, olfgpu_solve_batch_context_full).  ``unsupported`` maps the name of an
        argument in UNSUPPORTED_SOLVE_ARRAYS to an array passed as given (the engine rejects non-empty ones)."""
        n = self.structure.n
        disabled = _c(disabled, np.uint8)
        ns = disabled.shape[0]
        x0b = None if x0_base is None else _c(x0_base, np.float64)
        x0f = None if x0_full is None else _c(x0_full, np.float64)
        tb = _c(target_base, np.float64)
        bm = _c(base_row_mode, np.int32)
        rme = _c(np.zeros(0) if row_mode_entries is None else row_mode_entries, np.int32).reshape(-1)
        toi = _c(np.zeros(0) if target_override_index is None else target_override_index, np.int32)
        tov = _c(np.zeros(0) if target_override_value is None else target_override_value, np.float64)
        vt = None if var_type is None else _c(var_type, np.int32)
        extra = []
        unsupported = unsupported or {}
        for name in UNSUPPORTED_SOLVE_ARRAYS:
            a = unsupported.get(name)
            if a is None:
                extra += [None, 0]
            else:
                a = _c(a, np.int32 if name in _INT_SOLVE_ARRAYS else np.float64)
                extra += [_p(a) if a.size else None, int(a.size)]
                self._keep_unsupported = a
        if out is None:
            out = np.zeros((ns, n + 3))
        ln = lambda a: 0 if a is None else int(a.size)
        _check(load().olfgpu_solve_batch_context_full(
            self.handle, _p(x0b), ln(x0b), _p(tb), ln(tb), _p(rme) if rme.size else None, int(rme.size), _p(bm), ln(bm),
            _p(disabled), ns, disabled.shape[1], _p(toi) if toi.size else None, int(toi.size),
            _p(tov) if tov.size else None, int(tov.size), *extra, max_iter, tol, reactive_limit_tol, slack_dist_tol,
            conv_eps_per_eq, svs_mode, max_dv, max_dphi, _p(vt), ln(vt), _p(x0f), ln(x0f),
            None, 0, None, 0, None, 0, None, 0, None, 0,
            max_outer, max_pq_pv_switch, 1 if reject_slack_distribution_failure else 0,
            1 if skip_reactive_limits else 0, 0, None, 0, None, 0, pause_at_ended,
            _p(out)))
        return out

    def solve_simple(self, x0_base, target_base, base_row_mode, disabled, x0_full=None, row_mode_entries=None,
                     target_override_index=None, target_override_value=None, max_iter: int = 15, tol: float = 1e-8,
                     reactive_limit_tol: float = 1e-4, max_outer: int = 20, max_pq_pv_switch: int = 3,
                     out: Optional[np.ndarray] = None) -> np.ndarray:
        """The same solve through olfgpu_solve_batch_context (the short argument list)."""
        args, keep = self._request(x0_base, target_base, base_row_mode, disabled, x0_full, row_mode_entries,
                                   target_override_index, target_override_value, max_iter, tol, reactive_limit_tol,
                                   max_outer, max_pq_pv_switch)
        if out is None:
            out = np.zeros((keep[0].shape[0], self.structure.n + 3))
        _check(load().olfgpu_solve_batch_context(self.handle, *args, _p(out)))
        return out

    def last_slack_distribution_failures(self) -> np.ndarray:
        """Per scenario of the last solve, 1 where the distributed slack could not place the whole mismatch."""
        out = np.zeros(self.n_scenarios, np.uint8)
        cnt = ctypes.c_int(0)
        _check(load().olfgpu_last_slack_distribution_failures(self.handle, _p(out), ctypes.byref(cnt)))
        return out

    def read_targets(self, slots=None) -> np.ndarray:
        """BatchReadbackNative.readBatchTargets: [slots][n] targets as the last solve ended with them (default: the
        whole bank)."""
        slots = _c(np.arange(self.n_scenarios) if slots is None else slots, np.int32)
        out = np.zeros((slots.size, self.structure.n))
        _check(load().olfgpu_read_batch_targets(self.handle, int(slots.size), _p(slots), _p(out)))
        return out

    def read_row_modes(self, slots=None) -> np.ndarray:
        """BatchReadbackNative.readBatchRowModes: [slots][n] row modes as the last solve ended with them."""
        slots = _c(np.arange(self.n_scenarios) if slots is None else slots, np.int32)
        out = np.zeros((slots.size, self.structure.n), np.int32)
        _check(load().olfgpu_read_batch_row_modes(self.handle, int(slots.size), _p(slots), _p(out)))
        return out

    def set_outer_loops(self, distributed_slack: bool = True, reactive_limits: bool = True):
        """DriverNative.setBatchOuterLoops: each outer loop on or off for the following solves."""
        _check(load().olfgpu_set_outer_loops(self.handle, 1 if distributed_slack else 0, 1 if reactive_limits else 0))

    def set_realistic_check(self, row_checked=None, min_v: float = 0.0, max_v: float = 0.0, enabled: bool = True):
        """ReactiveLimitsNative.setBatchRealisticCheck: rows [n] whose converged voltage must lie in [min_v, max_v]."""
        rc = None if row_checked is None else _c(row_checked, np.uint8)
        self._row_checked = rc
        _check(load().olfgpu_set_realistic_check(self.handle, _p(rc), min_v, max_v, 1 if enabled else 0))

    def set_refinement_bound(self, correction_bound: float = 1e-11):
        """Mixed precision: a scenario near convergence refines until its correction max |d| <= correction_bound."""
        _check(load().olfgpu_set_refinement_bound(self.handle, correction_bound))

    def set_start_polish(self, ratio: float = 1e-2):
        """Fallback mode: a scenario converged from its own start above ratio * tol takes one more Newton step."""
        _check(load().olfgpu_set_start_polish(self.handle, ratio))

    def set_fp64_restart(self, enable: bool = True):
        """Mixed precision: a scenario whose solve fails restarts once in FP64 (on by default)."""
        _check(load().olfgpu_set_fp64_restart(self.handle, 1 if enable else 0))

    def stage(self, x0_base, target_base, base_row_mode, disabled, x0_full=None, row_mode_entries=None,
              target_override_index=None, target_override_value=None, max_iter: int = 15, tol: float = 1e-8,
              reactive_limit_tol: float = 1e-4, max_outer: int = 20, max_pq_pv_switch: int = 3) -> None:
        """Validates and uploads a request without running it (run by MultiContext.solve)."""
        args, keep = self._request(x0_base, target_base, base_row_mode, disabled, x0_full, row_mode_entries,
                                   target_override_index, target_override_value, max_iter, tol, reactive_limit_tol,
                                   max_outer, max_pq_pv_switch)
        _check(load().olfgpu_stage_batch_context(self.handle, *args))

    def _request(self, x0_base, target_base, base_row_mode, disabled, x0_full, row_mode_entries, target_override_index,
                 target_override_value, max_iter, tol, reactive_limit_tol, max_outer, max_pq_pv_switch):
        disabled = _c(disabled, np.uint8)
        ns = disabled.shape[0]
        x0b = None if x0_base is None else _c(x0_base, np.float64)
        x0f = None if x0_full is None else _c(x0_full, np.float64)
        tb = _c(target_base, np.float64)
        bm = _c(base_row_mode, np.int32)
        rme = _c(np.zeros(0) if row_mode_entries is None else row_mode_entries, np.int32).reshape(-1)
        toi = _c(np.zeros(0) if target_override_index is None else target_override_index, np.int32)
        tov = _c(np.zeros(0) if target_override_value is None else target_override_value, np.float64)
        args = (_p(x0b), _p(x0f), _p(tb), _p(bm), rme.shape[0] // 3, _p(rme) if rme.size else None, ns,
                disabled.shape[1], _p(disabled), toi.shape[0], _p(toi) if toi.size else None,
                _p(tov) if tov.size else None, max_iter, tol, reactive_limit_tol, max_outer, max_pq_pv_switch)
        return args, (disabled, x0b, x0f, tb, bm, rme, toi, tov)

    def set_phase_timing(self, enable: bool = True):
        """Level schedule: launch each iteration phase by phase between CUDA events (diagnostics)."""
        _check(load().olfgpu_set_phase_timing(self.handle, 1 if enable else 0))

    def last_phase_times(self) -> dict:
        """Milliseconds per phase of the last solve (summed over its iterations), iterations and factorized lanes."""
        o = np.zeros(8)
        _check(load().olfgpu_last_phase_times(self.handle, _p(o)))
        keys = ["fill", "test", "factor", "solve", "refine", "step"]
        d = {k: float(v) for k, v in zip(keys, o[:6])}
        d["iterations"] = int(o[6])
        d["factorized_lanes"] = int(o[7])
        return d

    def set_mixed_precision_policy(self, policy: int = 0):
        """0 MIXED_REFINE: FP32 LU + FP64 refinement near convergence; 1 MIXED_FP64_NEAR: iterations with a scenario
        near convergence run in FP64."""
        _check(load().olfgpu_set_mixed_precision_policy(self.handle, policy))

    def set_device_loop(self, enable: bool = True):
        """The whole Newton loop as one graph launch (conditional graph nodes; level schedules)."""
        _check(load().olfgpu_set_device_loop(self.handle, 1 if enable else 0))

    def last_fp64_iterations(self) -> int:
        v = ctypes.c_int(0)
        _check(load().olfgpu_last_fp64_iterations(self.handle, ctypes.byref(v)))
        return v.value

    def set_mixed_precision_controls(self, refine_below: float = 1e-2, growth_limit: float = 1e4):
        """Mixed precision: refinement only below refine_below; FP64 refactor above growth_limit pivot growth."""
        _check(load().olfgpu_set_mixed_precision_controls(self.handle, refine_below, growth_limit))

    def last_fp64_refactors(self) -> np.ndarray:
        """Indices of the scenarios whose last solve was flagged for FP64 refactors."""
        f = np.zeros(self.n_scenarios, np.uint8)
        k = ctypes.c_int(0)
        _check(load().olfgpu_last_fp64_refactors(self.handle, _p(f), ctypes.byref(k)))
        return np.flatnonzero(f)

    def set_device_start(self, x0_full_device=None):
        """Per-scenario start states from a device array [nS, n] float64 (a torch CUDA tensor) for the following
        solves; None switches back to the host x0_full argument.  Keep the tensor alive while it is set."""
        ptr = None if x0_full_device is None else ctypes.c_void_p(x0_full_device.data_ptr())
        self._device_start = x0_full_device
        _check(load().olfgpu_set_device_start(self.handle, ptr))

    def set_fallback_start(self, enable: bool = True):
        """Scenarios that fail from x0_full restart once from x0_base inside the same solve."""
        _check(load().olfgpu_set_fallback_start(self.handle, 1 if enable else 0))

    def last_fallbacks(self) -> np.ndarray:
        """Indices of the scenarios the last solve restarted from the base start."""
        f = np.zeros(self.n_scenarios, np.uint8)
        k = ctypes.c_int(0)
        _check(load().olfgpu_last_fallbacks(self.handle, _p(f), ctypes.byref(k)))
        return np.flatnonzero(f)

    def last_stats(self):
        ms = ctypes.c_float(0)
        it = ctypes.c_int(0)
        tot = np.zeros(self.n_scenarios, np.int32)
        _check(load().olfgpu_last_solve_stats(self.handle, ctypes.byref(ms), ctypes.byref(it), _p(tot)))
        return float(ms.value), int(it.value), tot

    def debug_fill(self, x_full, target_base, base_row_mode, disabled):
        s = self.structure
        ns = self.n_scenarios
        J = np.zeros((ns, s.nnz))
        F = np.zeros((ns, s.n))
        xf, tb, bm, dis = (_c(x_full, np.float64), _c(target_base, np.float64), _c(base_row_mode, np.int32),
                           _c(disabled, np.uint8))
        _check(load().olfgpu_debug_fill(self.handle, _p(xf), _p(tb), _p(bm), _p(dis), _p(J), _p(F)))
        return J, F

    def linear_solve_transposed(self, csr_vals, rhs=None, rhs_t=None, precision: int = FP64):
        """BatchedLuNative.factorizeAndSolveTransposed: one factorization of each J, then J x = rhs and J^T y = rhs_t
        on its factors; returns (x, y) (None where the right-hand side is None)."""
        s = self.structure
        v = _c(csr_vals, np.float64)
        r = None if rhs is None else _c(rhs, np.float64)
        rt = None if rhs_t is None else _c(rhs_t, np.float64)
        x = None if r is None else np.zeros((self.n_scenarios, s.n))
        y = None if rt is None else np.zeros((self.n_scenarios, s.n))
        _check(load().olfgpu_linear_solve_transposed(self.handle, _p(v), _p(r), _p(rt), precision, _p(x), _p(y)))
        return x, y

    def screen_violations(self, elem_id, group_ptr, group_side, group_qty, lim_ptr, lim_threshold, bus_vrow=None,
                          bus_high=None, bus_low=None, realistic: bool = False, min_v: float = 0.0, max_v: float = 0.0,
                          band: float = 1e-7, capacity: int = 64):
        """Violation candidates of the last solve (olfgpu_screen_violations): per scenario the sorted record ids, and
        the per-scenario counts (above capacity: truncated)."""
        a = [_c(v, np.int32) for v in (elem_id, group_ptr, group_side, group_qty, lim_ptr)]
        lt = _c(lim_threshold, np.float64)
        nb = 0 if bus_vrow is None else len(bus_vrow)
        br = _c(np.zeros(0) if bus_vrow is None else bus_vrow, np.int32)
        bh = _c(np.zeros(0) if bus_high is None else bus_high, np.float64)
        bl = _c(np.zeros(0) if bus_low is None else bus_low, np.float64)
        rec = np.zeros((self.n_scenarios, capacity), np.int32)
        cnt = np.zeros(self.n_scenarios, np.int32)
        _check(load().olfgpu_screen_violations(self.handle, len(elem_id), *[_p(v) if v.size else None for v in a],
                                               _p(lt) if lt.size else None, nb, _p(br) if nb else None,
                                               _p(bh) if nb else None, _p(bl) if nb else None, 1 if realistic else 0,
                                               min_v, max_v, band, capacity, _p(rec), _p(cnt)))
        return [list(rec[s, :min(cnt[s], capacity)]) for s in range(self.n_scenarios)], cnt

    def debug_linear_solve(self, csr_vals, rhs, precision: int = FP64):
        s = self.structure
        out = np.zeros((self.n_scenarios, s.n))
        v, r = _c(csr_vals, np.float64), _c(rhs, np.float64)
        _check(load().olfgpu_debug_linear_solve(self.handle, _p(v), _p(r), precision, _p(out)))
        return out


class MultiContext:
    """Batch contexts of different grids run by one persistent launch (olfgpu_solve_multi_context)."""

    def __init__(self, contexts):
        self.contexts = list(contexts)
        h = _i64(0)
        arr = (_i64 * len(self.contexts))(*[c.handle for c in self.contexts])
        _check(load().olfgpu_create_multi_context(len(self.contexts), arr, ctypes.byref(h)))
        self.handle = h.value

    def close(self):
        if getattr(self, "handle", 0):
            load().olfgpu_destroy_multi_context(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_schedule(self, lanes_per_tile: int, threads: int = 256, order: int = 0):
        """lanes_per_tile -1: the next solve autotunes (tile lanes x threads x member order)."""
        _check(load().olfgpu_set_multi_schedule(self.handle, lanes_per_tile, threads, order))

    def schedule(self):
        """(lanes per tile, threads, order) in force and the autotuner's timings [(lanes, threads, order, ms)]."""
        la, th, od, nr = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        res = np.zeros(4 * 64)
        _check(load().olfgpu_get_multi_schedule(self.handle, ctypes.byref(la), ctypes.byref(th), ctypes.byref(od), 64,
                                                _p(res), ctypes.byref(nr)))
        return (la.value, th.value, od.value), [tuple(res[4 * i:4 * i + 4]) for i in range(min(nr.value, 64))]

    def solve(self, outs=None):
        """Runs every member's staged batch; returns (per member [nS][n + 3] results, device ms)."""
        if outs is None:
            outs = [np.zeros((c.n_scenarios, c.structure.n + 3)) for c in self.contexts]
        ptrs = (_dp * len(outs))(*[o.ctypes.data_as(_dp) for o in outs])
        ms = ctypes.c_float(0)
        _check(load().olfgpu_solve_multi_context(self.handle, ptrs, ctypes.byref(ms)))
        return outs, float(ms.value)
