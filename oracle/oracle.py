"""ORACLE -- test infrastructure only (the tests, the smoke check and the benchmark's CPU-baseline leg).

ctypes wrapper over ``oracle/lib/liboracle.so`` (the C restatement of the reference path, ``olf_oracle.c``) and, when
they were built here from the reference's own sources (``oracle/ref/Makefile``), ``oracle/_ref/libolfref.so`` (the
reference's host structure code and generated formula headers) and ``oracle/_ref/libolfreflu.so`` (the reference's
host LU).  None of these libraries is ever on the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libolfref.so")
REF_LU_LIB = os.path.join(HERE, "_ref", "libolfreflu.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def reference_root(reference: Optional[str] = None) -> Optional[str]:
    """Where the reference sources lie: the argument, else $OLF_REFERENCE, else the default the recipe in
    ``oracle/ref/Makefile`` names; None when no reference tree is there (the glue is then not built)."""
    ref = reference or os.environ.get("OLF_REFERENCE")
    if not ref:
        out = subprocess.run(["make", "-s", "-C", os.path.join(HERE, "ref"), "print-ref"], capture_output=True,
                             text=True)
        ref = out.stdout.strip() if out.returncode == 0 else ""
    return ref if ref and os.path.isdir(os.path.join(ref, "native", "cuda")) else None


def build(reference: Optional[str] = None) -> None:
    """Compile the oracle (and, when the reference sources are present, the reference glue)."""
    subprocess.check_call(["make", "-s", "-C", HERE])
    ref = reference_root(reference)
    if ref:
        subprocess.check_call(["make", "-s", "-C", os.path.join(HERE, "ref"), f"REF={ref}"])


def _arr(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    return a


def _ptr(a):
    if a.dtype == np.float64:
        return a.ctypes.data_as(_dp)
    if a.dtype == np.int32:
        return a.ctypes.data_as(_ip)
    if a.dtype == np.uint8:
        return a.ctypes.data_as(_u8p)
    raise TypeError(a.dtype)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.oracle_structure_build.restype = ctypes.c_void_p
        L.oracle_structure_build.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _ip, ctypes.c_int, _dp, _ip, ctypes.c_int,
                                             _dp, _ip, ctypes.c_int, _ip, ctypes.c_char_p]
        L.oracle_structure_free.argtypes = [ctypes.c_void_p]
        L.oracle_structure_nnz.argtypes = [ctypes.c_void_p]
        L.oracle_structure_export.argtypes = [ctypes.c_void_p, _ip, _ip, _ip, _ip, _ip, _ip, _ip]
        L.oracle_fill.argtypes = [ctypes.c_void_p, _dp, _dp, _ip, _u8p, _dp, _dp]
        L.oracle_solver_new.restype = ctypes.c_void_p
        L.oracle_solver_new.argtypes = [ctypes.c_void_p]
        L.oracle_solver_free.argtypes = [ctypes.c_void_p]
        L.oracle_solve_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_int, _dp, _ip, _u8p, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, _dp]
        L.oracle_solve_batch_ex.argtypes = L.oracle_solve_batch.argtypes[:-1] + [ctypes.c_void_p, _dp]
        L.oracle_solve_batch_ds.argtypes = L.oracle_solve_batch.argtypes[:-1] + [ctypes.c_void_p, ctypes.c_void_p, _dp]
        L.oracle_solve_batch_final.argtypes = L.oracle_solve_batch_ds.argtypes + [_dp, _ip]
        L.oracle_linear_solve.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        L.oracle_linear_solve_transposed.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        L.oracle_closed_branch.argtypes = [_dp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_double, _dp]
        L.oracle_open_branch.argtypes = [_dp, ctypes.c_double, ctypes.c_double, _dp]
        L.oracle_shunt.argtypes = [_dp, ctypes.c_double, _dp]
        _lib = L
    return _lib


class _Rl(ctypes.Structure):
    _fields_ = [("n_rl", ctypes.c_int), ("voltage_row", _ip), ("min_q", _dp), ("max_q", _dp), ("load_q", _dp),
                ("target_v", _dp), ("nom_v", _dp), ("static_p", _dp), ("p_row", _ip), ("id_rank", _ip)]


class _Ds(ctypes.Structure):
    _fields_ = [("n_ds", ctypes.c_int), ("row", _ip), ("factor", _dp), ("base", _dp), ("max_delta", _dp),
                ("min_delta", _dp), ("slack_row", ctypes.c_int), ("slack_target_p", ctypes.c_double),
                ("dist_tol", ctypes.c_double), ("reject", ctypes.c_int)]


class _Opts(ctypes.Structure):
    _fields_ = [("conv_eps_per_eq", ctypes.c_double), ("svs_mode", ctypes.c_int), ("max_dv", ctypes.c_double),
                ("max_dphi", ctypes.c_double), ("var_type", _ip), ("v_check", _u8p), ("min_v", ctypes.c_double),
                ("max_v", ctypes.c_double)]


class Structure:
    """The oracle's structure and solver over one packed network (``olfgpu.packing.Packed``)."""

    def __init__(self, packed):
        L = lib()
        self.p = packed
        self._keep = [_arr(packed.cb_params, np.float64), _arr(packed.cb_idx, np.int32),
                      _arr(packed.ob_params, np.float64), _arr(packed.ob_idx, np.int32),
                      _arr(packed.sh_params, np.float64), _arr(packed.sh_idx, np.int32),
                      _arr(packed.identity_rows, np.int32)]
        k = self._keep
        err = ctypes.create_string_buffer(256)
        self.h = L.oracle_structure_build(packed.n, packed.n_cb, _ptr(k[0]), _ptr(k[1]), packed.n_ob, _ptr(k[2]),
                                          _ptr(k[3]), packed.n_sh, _ptr(k[4]), _ptr(k[5]), k[6].shape[0], _ptr(k[6]),
                                          err)
        if not self.h:
            raise RuntimeError("oracle structure: " + err.value.decode())
        self.nnz = L.oracle_structure_nnz(self.h)
        self.solver = L.oracle_solver_new(self.h)

    def close(self):
        if self.h:
            lib().oracle_solver_free(self.solver)
            lib().oracle_structure_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def export(self):
        n, p = self.p.n, self.p
        out = dict(row_map=np.zeros(n, np.int32), row_ptr=np.zeros(n + 1, np.int32),
                   col_idx=np.zeros(self.nnz, np.int32), diag_pos=np.zeros(n, np.int32),
                   cb_dest=np.zeros(p.n_cb * 28, np.int32), ob_dest=np.zeros(p.n_ob * 8, np.int32),
                   sh_dest=np.zeros(p.n_sh * 5, np.int32))
        lib().oracle_structure_export(self.h, *[_ptr(out[k]) for k in ("row_map", "row_ptr", "col_idx", "diag_pos",
                                                                       "cb_dest", "ob_dest", "sh_dest")])
        return out

    def fill(self, x, target, mode, disabled=None):
        vals = np.zeros(self.nnz)
        F = np.zeros(self.p.n)
        x, target, mode = _arr(x, np.float64), _arr(target, np.float64), _arr(mode, np.int32)
        dis = None if disabled is None else _arr(disabled, np.uint8)
        lib().oracle_fill(self.h, _ptr(x), _ptr(target), _ptr(mode), None if dis is None else _ptr(dis),
                          _ptr(vals), _ptr(F))
        return vals, F

    def linear_solve(self, vals, b):
        z = np.zeros(self.p.n)
        vals, b = _arr(vals, np.float64), _arr(b, np.float64)
        rc = lib().oracle_linear_solve(self.solver, _ptr(vals), _ptr(b), _ptr(z))
        if rc != 0:
            raise RuntimeError("oracle LU: singular")
        return z

    def linear_solve_transposed(self, vals, b):
        """z with J^T z = b (J given by its CSR values)."""
        z = np.zeros(self.p.n)
        vals, b = _arr(vals, np.float64), _arr(b, np.float64)
        rc = lib().oracle_linear_solve_transposed(self.solver, _ptr(vals), _ptr(b), _ptr(z))
        if rc != 0:
            raise RuntimeError("oracle LU: singular")
        return z

    def solve_batch(self, x0, disabled, max_iter=15, tol=1e-8, target=None, mode=None, reactive_limits=False,
                    rl_tol=1e-4, max_outer=20, max_switch=3, threads=0, conv_eps_per_eq=0.0, svs_mode=0,
                    max_dv=0.1, max_dphi=0.17453292519943295, var_type=None, v_check=None, min_v=0.0, max_v=0.0,
                    distributed_slack=None, slack_dist_tol=1e-6, reject_slack_distribution_failure=False,
                    final_equations=False):
        """Per scenario [x(n), iterations, ||F||inf, status]; x0 is [n] (shared) or [nS, n].  conv_eps_per_eq > 0:
        OLF's 2-norm stopping test; svs_mode 2: MAX_VOLTAGE_CHANGE with var_type [n]; v_check [n]: the realistic-voltage
        rows checked against [min_v, max_v] at convergence; distributed_slack (packing.DistributedSlack): the bus-level
        distributed-slack outer loop, before the reactive-limit check.  final_equations: also return each scenario's
        targets and row modes as its solve ended with them ([nS][n] each), as (rows, targets, modes)."""
        p = self.p
        disabled = _arr(disabled, np.uint8)
        ns = disabled.shape[0]
        x0 = _arr(x0, np.float64)
        stride = 0 if x0.ndim == 1 else p.n
        target = _arr(p.target if target is None else target, np.float64)
        mode = _arr(p.base_row_mode if mode is None else mode, np.int32)
        out = np.zeros((ns, p.n + 3))
        rl_struct = None
        if reactive_limits and p.rl is not None:
            r = p.rl
            self._rl_keep = [_arr(r.voltage_row, np.int32), _arr(r.min_q, np.float64), _arr(r.max_q, np.float64),
                             _arr(r.load_q, np.float64), _arr(r.target_v, np.float64), _arr(r.nom_v, np.float64),
                             _arr(r.static_p, np.float64), _arr(r.p_row, np.int32), _arr(r.id_rank, np.int32)]
            k = self._rl_keep
            rl_struct = _Rl(k[0].shape[0], _ptr(k[0]), _ptr(k[1]), _ptr(k[2]), _ptr(k[3]), _ptr(k[4]), _ptr(k[5]),
                            _ptr(k[6]), _ptr(k[7]), _ptr(k[8]))
        vt = None if var_type is None else _arr(var_type, np.int32)
        vc = None if v_check is None else _arr(v_check, np.uint8)
        opts = _Opts(conv_eps_per_eq, svs_mode, max_dv, max_dphi, None if vt is None else _ptr(vt),
                     None if vc is None else _ptr(vc), min_v, max_v)
        ds_struct = None
        if distributed_slack is not None:
            d = distributed_slack
            self._ds_keep = [_arr(d.row, np.int32), _arr(d.factor, np.float64), _arr(d.base_target, np.float64),
                             _arr(d.max_delta, np.float64), _arr(d.min_delta, np.float64)]
            k = self._ds_keep
            ds_struct = _Ds(k[0].shape[0], _ptr(k[0]), _ptr(k[1]), _ptr(k[2]), _ptr(k[3]), _ptr(k[4]),
                            int(d.slack_row), float(d.slack_target_p), slack_dist_tol,
                            1 if reject_slack_distribution_failure else 0)
        final_target = np.zeros((ns, p.n)) if final_equations else None
        final_mode = np.zeros((ns, p.n), np.int32) if final_equations else None
        lib().oracle_solve_batch_final(self.solver, ns, _ptr(x0), stride, _ptr(target), _ptr(mode), _ptr(disabled),
                                       disabled.shape[1], max_iter, tol,
                                       ctypes.cast(ctypes.pointer(rl_struct), ctypes.c_void_p) if rl_struct else None,
                                       rl_tol, max_outer, max_switch, threads,
                                       ctypes.cast(ctypes.pointer(opts), ctypes.c_void_p),
                                       ctypes.cast(ctypes.pointer(ds_struct), ctypes.c_void_p) if ds_struct else None,
                                       _ptr(out), None if final_target is None else _ptr(final_target),
                                       None if final_mode is None else _ptr(final_mode))
        if final_equations:
            return out, final_target, final_mode
        return out


def closed_branch(params, v1, r1, v2, a1, ph1, ph2):
    o = np.zeros(28)
    p = _arr(params, np.float64)
    lib().oracle_closed_branch(_ptr(p), v1, r1, v2, a1, ph1, ph2, _ptr(o))
    return o


def open_branch(params, v1, v2):
    o = np.zeros(8)
    p = _arr(params, np.float64)
    lib().oracle_open_branch(_ptr(p), v1, v2, _ptr(o))
    return o


def shunt(params, v):
    o = np.zeros(5)
    p = _arr(params, np.float64)
    lib().oracle_shunt(_ptr(p), v, _ptr(o))
    return o


# ---------------------------------------------------------------------------------------------------------------
# The reference's own host code (built here from its sources), when available.
# ---------------------------------------------------------------------------------------------------------------
_ref = None


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref
    if _ref is None:
        R = ctypes.CDLL(REF_LIB)
        R.olfref_structure.argtypes = [ctypes.c_int, ctypes.c_int, _ip, ctypes.c_int, _ip, ctypes.c_int, _ip,
                                       ctypes.c_int, _ip, _ip, _ip, _ip, _ip, ctypes.c_int, _ip, _ip, _ip, _ip,
                                       ctypes.c_char_p]
        R.olfref_closed_branch.argtypes = [_dp] + [ctypes.c_double] * 6 + [_dp]
        R.olfref_open_branch.argtypes = [_dp, ctypes.c_double, ctypes.c_double, _dp]
        R.olfref_shunt.argtypes = [_dp, ctypes.c_double, _dp]
        _ref = R
    return _ref


def ref_structure(packed):
    """The reference's row map / pattern / destinations / diagonal slots for the packed network."""
    R = ref_lib()
    n = packed.n
    cap = packed.n_cb * 28 + packed.n_ob * 8 + packed.n_sh * 5 + n
    out = dict(row_map=np.zeros(n, np.int32), row_ptr=np.zeros(n + 1, np.int32), col_idx=np.zeros(cap, np.int32),
               diag_pos=np.zeros(n, np.int32), cb_dest=np.zeros(packed.n_cb * 28, np.int32),
               ob_dest=np.zeros(packed.n_ob * 8, np.int32), sh_dest=np.zeros(packed.n_sh * 5, np.int32))
    nnz = ctypes.c_int(0)
    cb, ob, sh, ir = (_arr(packed.cb_idx, np.int32), _arr(packed.ob_idx, np.int32), _arr(packed.sh_idx, np.int32),
                      _arr(packed.identity_rows, np.int32))
    err = ctypes.create_string_buffer(256)
    rc = R.olfref_structure(n, packed.n_cb, _ptr(cb), packed.n_ob, _ptr(ob), packed.n_sh, _ptr(sh), ir.shape[0],
                            _ptr(ir), _ptr(out["row_map"]), ctypes.byref(nnz), _ptr(out["row_ptr"]),
                            _ptr(out["col_idx"]), cap, _ptr(out["cb_dest"]), _ptr(out["ob_dest"]),
                            _ptr(out["sh_dest"]), _ptr(out["diag_pos"]), err)
    if rc != 0:
        raise RuntimeError("reference structure: " + err.value.decode())
    out["col_idx"] = out["col_idx"][:nnz.value].copy()
    return out


def ref_closed_branch(params, v1, r1, v2, a1, ph1, ph2):
    o = np.zeros(28)
    p = _arr(params, np.float64)
    ref_lib().olfref_closed_branch(_ptr(p), v1, r1, v2, a1, ph1, ph2, _ptr(o))
    return o


def ref_open_branch(params, v1, v2):
    o = np.zeros(8)
    p = _arr(params, np.float64)
    ref_lib().olfref_open_branch(_ptr(p), v1, v2, _ptr(o))
    return o


def ref_shunt(params, v):
    o = np.zeros(5)
    p = _arr(params, np.float64)
    ref_lib().olfref_shunt(_ptr(p), v, _ptr(o))
    return o


_ref_lu = None


def ref_lu_available() -> bool:
    return os.path.exists(REF_LU_LIB)


def ref_lu_lib():
    global _ref_lu
    if _ref_lu is None:
        R = ctypes.CDLL(REF_LU_LIB)
        R.olfref_lu_plan.restype = ctypes.c_void_p
        R.olfref_lu_plan.argtypes = [ctypes.c_int, _ip, _ip, _ip, _ip, ctypes.c_char_p]
        R.olfref_lu_free.argtypes = [ctypes.c_void_p]
        R.olfref_lu_solve.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        R.olfref_lu_solve_transposed.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        _ref_lu = R
    return _ref_lu


class RefLu:
    """The reference's own host LU on one CSR pattern: the fast engine's plan (scalar_lu_plan.cu) on its
    minimum-degree order (minimum_degree.cu), factorized and solved by the one-lane ports of
    native/host/lu_transposed_check.cpp:74-145 (static pivots; a clamped pivot or an oversized multiplier counts as
    trouble)."""

    def __init__(self, row_ptr, col_idx):
        R = ref_lu_lib()
        self.row_ptr = _arr(row_ptr, np.int32)
        self.col_idx = _arr(col_idx, np.int32)
        self.n = self.row_ptr.shape[0] - 1
        nnz_lu, levels = ctypes.c_int(0), ctypes.c_int(0)
        err = ctypes.create_string_buffer(256)
        self.h = R.olfref_lu_plan(self.n, _ptr(self.row_ptr), _ptr(self.col_idx), ctypes.byref(nnz_lu),
                                  ctypes.byref(levels), err)
        if not self.h:
            raise RuntimeError("reference LU plan: " + err.value.decode())
        self.nnz_lu, self.levels = nnz_lu.value, levels.value

    def solve(self, vals, b):
        """(x, trouble) with A x = b; A by its CSR values in the pattern's order."""
        x = np.zeros(self.n)
        vals, b = _arr(vals, np.float64), _arr(b, np.float64)
        trouble = ref_lu_lib().olfref_lu_solve(self.h, _ptr(vals), _ptr(b), _ptr(x))
        if trouble < 0:
            raise RuntimeError("reference LU: solve failed")
        return x, trouble

    def solve_transposed(self, vals, b):
        """(x, trouble) with A^T x = b on the same factors: the reference's transposed solve."""
        x = np.zeros(self.n)
        vals, b = _arr(vals, np.float64), _arr(b, np.float64)
        trouble = ref_lu_lib().olfref_lu_solve_transposed(self.h, _ptr(vals), _ptr(b), _ptr(x))
        if trouble < 0:
            raise RuntimeError("reference LU: transposed solve failed")
        return x, trouble

    def __del__(self):
        try:
            if self.h:
                ref_lu_lib().olfref_lu_free(self.h)
                self.h = None
        except Exception:
            pass


def ref_component_fill(packed, ref_struct, x, target, mode, disabled=None):
    """J values and F of one scenario assembled from the reference's OWN components only: its generated formula
    headers per element (``ref_closed_branch`` / ``ref_open_branch`` / ``ref_shunt``) scattered through its own
    role-folded destinations (``ref_structure``: a J slot >= 0, an F row as -2 - row, -1 skipped), F starting at
    -target, an outaged element skipped, and FIXED_VARIABLE rows (mode 0) replaced by the identity row with
    F = x - target (fill_launch.cu:82-126).  Elements in packing order, outputs in table order."""
    p = packed
    rp, dp = ref_struct["row_ptr"], ref_struct["diag_pos"]
    vals = np.zeros(rp[-1])
    F = -np.asarray(target, dtype=np.float64).copy()

    def scatter(out, dest):
        for k, d in enumerate(dest):
            if d >= 0:
                vals[d] += out[k]
            elif d <= -2:
                F[-2 - d] += out[k]

    for e in range(p.n_cb):
        if disabled is not None and disabled[e]:
            continue
        par, q = p.cb_params[e], p.cb_idx[e]
        r1 = x[q[9]] if q[9] >= 0 else par[6]
        a1 = x[q[8]] if q[8] >= 0 else par[7]
        scatter(ref_closed_branch(par, x[q[5]], r1, x[q[7]], a1, x[q[4]], x[q[6]]),
                ref_struct["cb_dest"][e * 28:(e + 1) * 28])
    for e in range(p.n_ob):
        if disabled is not None and disabled[p.n_cb + e]:
            continue
        par, q = p.ob_params[e], p.ob_idx[e]
        v1 = x[q[4]] if q[4] >= 0 else 1.0
        v2 = x[q[5]] if q[5] >= 0 else 1.0
        scatter(ref_open_branch(par, v1, v2), ref_struct["ob_dest"][e * 8:(e + 1) * 8])
    for e in range(p.n_sh):
        if disabled is not None and disabled[p.n_cb + p.n_ob + e]:
            continue
        par, q = p.sh_params[e], p.sh_idx[e]
        scatter(ref_shunt(par, x[q[2]]), ref_struct["sh_dest"][e * 5:(e + 1) * 5])
    for r in np.flatnonzero(np.asarray(mode) == 0):
        vals[rp[r]:rp[r + 1]] = 0.0
        vals[dp[r]] = 1.0
        F[r] = x[r] - target[r]
    return vals, F


def newton_with(fill, solve, x0, max_iter=15, tol=1e-8):
    """One plain Newton-Raphson solve (no outer loops) over a given fill ``fill(x) -> (vals, F)`` and linear solver
    ``solve(vals, rhs) -> dx``, under the rules of newton_iteration.cu:276-397 as the oracle's ``newton()`` states them:
    at least one iteration; converged when max |F| < tol before the budget; a non-finite mismatch is DIVERGED; the
    budget spent is MAX_ITERATION_REACHED; a failed factorization is LINEAR_SOLVE_FAILED (the linear-solve guard and
    the bad-last-solve reject are left out: they never act on a scenario that converges).  Returns [x(n), iterations,
    ||F||inf, status] with the oracle's status codes, the row layout of ``Structure.solve_batch``.  With the
    reference's own formulas, scatter map and host LU plugged in, it is the trajectory the tests pin the oracle
    against."""
    converged, max_iter_reached, diverged, linear_solve_failed = 0, 1, -1, -3
    x = np.array(x0, dtype=np.float64, copy=True)
    status, it, nrm = linear_solve_failed, 0, float("nan")
    for it in range(max_iter + 1):
        vals, F = fill(x)
        if not np.all(np.isfinite(F)):
            nrm, status = float("nan"), diverged
            break
        nrm = float(np.max(np.abs(F)))
        if it > 0 and nrm < tol and it < max_iter:
            status = converged
            break
        if it == max_iter:
            status = max_iter_reached
            break
        try:
            dx = solve(vals, -F)
        except RuntimeError:
            status = linear_solve_failed
            break
        x += dx
    return np.concatenate([x, [it, nrm, status]])


# ---------------------------------------------------------------------------------------------------------------
# Violation screening (sa/olf_gpu_violations.cu:160-361), restated over host states.
# ---------------------------------------------------------------------------------------------------------------
def branch_flows(packed, x, element):
    """(p1, q1, v1, p2, q2, v2) of one branch element at the states x [nS, n]: closed branches with the closed-branch
    terms (closed_branch.cuh:161-229), open-ended ones with the connected side's open-branch terms (open_branch.cuh:
    65-87), NaN on an open side."""
    ns = x.shape[0]
    nan = np.full(ns, np.nan)
    if element < packed.n_cb:
        y, g1, g2, b1, b2, ksi, r1, a1 = packed.cb_params[element]
        ix = packed.cb_idx[element]
        ph1, v1, ph2, v2 = x[:, ix[4]], x[:, ix[5]], x[:, ix[6]], x[:, ix[7]]
        sk, ck = np.sin(ksi), np.cos(ksi)
        t1, t2 = ksi - a1 - ph1 + ph2, ksi + a1 + ph1 - ph2
        p1 = r1 * v1 * (g1 * r1 * v1 + y * r1 * v1 * sk - y * v2 * np.sin(t1))
        q1 = r1 * v1 * (-b1 * r1 * v1 + y * r1 * v1 * ck - y * v2 * np.cos(t1))
        p2 = v2 * (g2 * v2 - y * r1 * v1 * np.sin(t2) + y * v2 * sk)
        q2 = v2 * (-b2 * v2 - y * r1 * v1 * np.cos(t2) + y * v2 * ck)
        return p1, q1, v1, p2, q2, v2
    e = element - packed.n_cb
    y, ksi, g1, b1, g2, b2, r1 = packed.ob_params[e]
    ix = packed.ob_idx[e]
    sk, ck = np.sin(ksi), np.cos(ksi)
    p1 = q1 = v1 = p2 = q2 = v2 = nan
    if ix[4] >= 0:
        v1 = x[:, ix[4]]
        d2 = (g2 + y * sk) ** 2 + (-b2 + y * ck) ** 2
        p1 = r1 * r1 * v1 * v1 * (g1 + y * y * g2 / d2 + (b2 * b2 + g2 * g2) * y * sk / d2)
        q1 = -r1 * r1 * v1 * v1 * (b1 + y * y * b2 / d2 - (b2 * b2 + g2 * g2) * y * ck / d2)
    if ix[5] >= 0:
        v2 = x[:, ix[5]]
        d1 = (g1 + y * sk) ** 2 + (-b1 + y * ck) ** 2
        p2 = v2 * v2 * (g2 + y * y * g1 / d1 + (b1 * b1 + g1 * g1) * y * sk / d1)
        q2 = -v2 * v2 * (b2 + y * y * b1 / d1 - (b1 * b1 + g1 * g1) * y * ck / d1)
    return p1, q1, v1, p2, q2, v2


def screen_violations(packed, x, disabled, elem_id, group_ptr, group_side, group_qty, lim_ptr, lim_threshold,
                      bus_vrow, bus_high, bus_low, realistic=False, min_v=0.0, max_v=0.0, band=1e-7, values=None):
    """Per scenario the sorted candidate ids of the screen (the engine's numbering; see include/olfgpu_b200.h).  With
    `values` (a list) it also collects (scenario, limit id, value, threshold) of every comparison, for margins."""
    ns = x.shape[0]
    n_lim = int(lim_ptr[-1]) if len(lim_ptr) else 0
    out = [[] for _ in range(ns)]
    for r, e in enumerate(elem_id):
        p1, q1, v1, p2, q2, v2 = branch_flows(packed, x, int(e))
        off = disabled[:, int(e)] != 0
        for g in range(group_ptr[r], group_ptr[r + 1]):
            p, q, v = (p1, q1, v1) if group_side[g] == 1 else (p2, q2, v2)
            with np.errstate(invalid="ignore", divide="ignore"):
                val = [np.hypot(p, q) / v, np.abs(p), np.sqrt(p * p + q * q)][group_qty[g]]
            for s in range(ns):
                if off[s] or np.isnan(val[s]):
                    continue
                for l in range(lim_ptr[g], lim_ptr[g + 1]):
                    t = lim_threshold[l]
                    if values is not None:
                        values.append((s, l, float(val[s]), float(t)))
                    if val[s] > t - abs(t) * band:
                        out[s].append(l)
                        if val[s] > t + abs(t) * band:
                            break
    nb = len(bus_vrow)
    for i in range(nb):
        if bus_vrow[i] < 0:
            continue
        vv = x[:, bus_vrow[i]]
        for s in range(ns):
            if vv[s] > bus_high[i] - abs(bus_high[i]) * band:
                out[s].append(n_lim + 2 * i)
            if vv[s] < bus_low[i] + abs(bus_low[i]) * band:
                out[s].append(n_lim + 2 * i + 1)
            if realistic and (vv[s] < min_v or vv[s] > max_v):
                out[s].append(n_lim + 2 * nb + i)
    return [sorted(o) for o in out]
