"""ORACLE -- test infrastructure only (the tests, the smoke check and the benchmark's CPU-baseline leg).

ctypes wrapper over ``oracle/lib/liboracle.so`` (the C restatement of the reference path, ``olf_oracle.c``) and, when
it was built here from the reference's own sources, ``oracle/_ref/libolfref.so`` (the reference's host structure code
and generated formula headers).  Neither library is ever on the product path.
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
        L.oracle_linear_solve.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        L.oracle_closed_branch.argtypes = [_dp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_double, _dp]
        L.oracle_open_branch.argtypes = [_dp, ctypes.c_double, ctypes.c_double, _dp]
        L.oracle_shunt.argtypes = [_dp, ctypes.c_double, _dp]
        _lib = L
    return _lib


class _Rl(ctypes.Structure):
    _fields_ = [("n_rl", ctypes.c_int), ("voltage_row", _ip), ("min_q", _dp), ("max_q", _dp), ("load_q", _dp),
                ("target_v", _dp), ("nom_v", _dp), ("static_p", _dp), ("p_row", _ip), ("id_rank", _ip)]


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

    def solve_batch(self, x0, disabled, max_iter=15, tol=1e-8, target=None, mode=None, reactive_limits=False,
                    rl_tol=1e-4, max_outer=20, max_switch=3, threads=0, conv_eps_per_eq=0.0, svs_mode=0,
                    max_dv=0.1, max_dphi=0.17453292519943295, var_type=None, v_check=None, min_v=0.0, max_v=0.0):
        """Per scenario [x(n), iterations, ||F||inf, status]; x0 is [n] (shared) or [nS, n].  conv_eps_per_eq > 0:
        OLF's 2-norm stopping test; svs_mode 2: MAX_VOLTAGE_CHANGE with var_type [n]; v_check [n]: the realistic-voltage
        rows checked against [min_v, max_v] at convergence."""
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
        lib().oracle_solve_batch_ex(self.solver, ns, _ptr(x0), stride, _ptr(target), _ptr(mode), _ptr(disabled),
                                    disabled.shape[1], max_iter, tol,
                                    ctypes.cast(ctypes.pointer(rl_struct), ctypes.c_void_p) if rl_struct else None,
                                    rl_tol, max_outer, max_switch, threads,
                                    ctypes.cast(ctypes.pointer(opts), ctypes.c_void_p), _ptr(out))
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
