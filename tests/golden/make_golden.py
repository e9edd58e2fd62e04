"""Generates the committed golden fixtures of this folder from the reference project (run where its sources are).

  formulas.npz           seeded inputs and, per family, the outputs obtained by evaluating the reference's frozen
                         formula manifests (codegen/golden/{closed_branch,open_branch,shunt}.golden.json, the bodies
                         codegen/java2cuda/prove.py checks at 1e-12) and by calling the reference's generated headers
                         (native/cuda/equations/generated/*.cuh) compiled into oracle/_ref.
  structure_<grid>.npz   the packed arrays of a synthetic grid and the reference's own row map, CSR pattern, diagonal
                         slots and role-folded scatter map for them (native/cuda/structure/csr_pattern.cu and the
                         structure_build.cuh templates, compiled into oracle/_ref).
  newton_<grid>.npz      Newton-Raphson solves of a synthetic grid's base case (flat start) and of seeded N-1 outages
                         (base-case start) assembled only from the reference's own components: its generated formula
                         headers, its row map / pattern / scatter map, and its host LU (the fast engine's plan on its
                         minimum-degree order with the one-lane factorization and solve of
                         native/host/lu_transposed_check.cpp, compiled into oracle/_ref/libolfreflu.so), under the
                         Newton rules of newton_iteration.cu:276-397; plus linear systems J x = b and J^T x = b at
                         perturbed states solved by that LU (its transposed solve: lu/transposed_solve.cuh's row bodies).

Usage:  python tests/golden/make_golden.py [/root/reference]
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "olf-gpu_b200"))

from oracle import oracle as O  # noqa: E402
from olfgpu import packing, synthetic  # noqa: E402

CB_ORDER = ["p1", "dp1dv1", "dp1dv2", "dp1dph1", "dp1dph2", "dp1da1", "dp1dr1", "q1", "dq1dv1", "dq1dv2", "dq1dph1",
            "dq1dph2", "dq1da1", "dq1dr1", "p2", "dp2dv1", "dp2dv2", "dp2dph1", "dp2dph2", "dp2da1", "dp2dr1", "q2",
            "dq2dv1", "dq2dv2", "dq2dph1", "dq2dph2", "dq2da1", "dq2dr1"]
OB_ORDER = ["p2", "dp2dv2", "q2", "dq2dv2", "p1", "dp1dv1", "q1", "dq1dv1"]
SH_ORDER = ["p", "dpdv", "q", "dqdv", "dqdb"]
# the operating ranges the reference's proof samples (codegen/java2cuda/prove.py:66-75)
RANGES = {"v1": (0.9, 1.1), "v2": (0.9, 1.1), "r1": (0.9, 1.1), "ph1": (-0.5, 0.5), "ph2": (-0.5, 0.5),
          "a1": (-0.3, 0.3), "ksi": (1.2, 1.9), "y": (10.0, 50.0), "g1": (-0.1, 0.1), "g2": (-0.1, 0.1),
          "b1": (-0.1, 0.1), "b2": (-0.1, 0.1)}
SAMPLES = 200


def _methods(path):
    """The manifest's methods as Python callables (the bodies are plain arithmetic expressions)."""
    d = json.load(open(path))
    ns = {"R2": 1.0, "A2": 0.0, "sin": math.sin, "cos": math.cos, "sqrt": math.sqrt}
    for m in d.get("helpers", []) + d["methods"]:
        src = f"def {m['name']}({', '.join(m['params'])}):\n    return {m['body']}\n"
        exec(src, ns)
    return ns


def formulas(ref: str):
    gdir = os.path.join(ref, "codegen", "golden")
    cb = _methods(os.path.join(gdir, "closed_branch.golden.json"))
    ob = _methods(os.path.join(gdir, "open_branch.golden.json"))
    sh = _methods(os.path.join(gdir, "shunt.golden.json"))
    rng = np.random.default_rng(20261203)
    cb_in = np.zeros((SAMPLES, 14))      # y g1 g2 b1 b2 ksi r1 a1 | v1 r1 v2 a1 ph1 ph2
    cb_gold = np.zeros((SAMPLES, 28))
    cb_ref = np.zeros((SAMPLES, 28))
    ob_in = np.zeros((SAMPLES, 9))       # y ksi g1 b1 g2 b2 r1 | v1 v2
    ob_gold = np.zeros((SAMPLES, 8))
    ob_ref = np.zeros((SAMPLES, 8))
    sh_in = np.zeros((SAMPLES, 3))       # g b | v
    sh_gold = np.zeros((SAMPLES, 5))
    sh_ref = np.zeros((SAMPLES, 5))
    u = lambda k: rng.uniform(*RANGES[k])  # noqa: E731
    for i in range(SAMPLES):
        y, g1, g2, b1, b2, ksi, r1, a1 = u("y"), u("g1"), u("g2"), u("b1"), u("b2"), u("ksi"), u("r1"), u("a1")
        v1, v2, ph1, ph2 = u("v1"), u("v2"), u("ph1"), u("ph2")
        cb_in[i] = [y, g1, g2, b1, b2, ksi, r1, a1, v1, r1, v2, a1, ph1, ph2]
        th1 = ksi - a1 + 0.0 - ph1 + ph2
        th2 = ksi + a1 - 0.0 + ph1 - ph2
        env1 = dict(y=y, g1=g1, g2=g2, b1=b1, b2=b2, v1=v1, r1=r1, v2=v2, sinKsi=math.sin(ksi), cosKsi=math.cos(ksi),
                    sinTheta=math.sin(th1), cosTheta=math.cos(th1))
        env2 = dict(env1, sinTheta=math.sin(th2), cosTheta=math.cos(th2))
        for k, name in enumerate(CB_ORDER):
            f = cb[name]
            env = env1 if name in CB_ORDER[:14] else env2
            cb_gold[i, k] = f(*[env[a] for a in f.__code__.co_varnames[:f.__code__.co_argcount]])
        cb_ref[i] = O.ref_closed_branch(cb_in[i, :8], v1, r1, v2, a1, ph1, ph2)
        oy, oksi, og1, ob1, og2, ob2, or1 = u("y"), u("ksi"), u("g1"), u("b1"), u("g2"), u("b2"), u("r1")
        ov1, ov2 = u("v1"), u("v2")
        ob_in[i] = [oy, oksi, og1, ob1, og2, ob2, or1, ov1, ov2]
        env = dict(y=oy, cosKsi=math.cos(oksi), sinKsi=math.sin(oksi), g1=og1, b1=ob1, g2=og2, b2=ob2, v1=ov1, v2=ov2,
                   r1=or1)
        for k, name in enumerate(OB_ORDER):
            f = ob[name]
            ob_gold[i, k] = f(*[env[a] for a in f.__code__.co_varnames[:f.__code__.co_argcount]])
        ob_ref[i] = O.ref_open_branch(ob_in[i, :7], ov1, ov2)
        sg, sb, sv = u("g1"), u("b1"), u("v1")
        sh_in[i] = [sg, sb, sv]
        env = dict(v=sv, g=sg, b=sb)
        for k, name in enumerate(SH_ORDER):
            f = sh[name]
            sh_gold[i, k] = f(*[env[a] for a in f.__code__.co_varnames[:f.__code__.co_argcount]])
        sh_ref[i] = O.ref_shunt(sh_in[i, :2], sv)
    np.savez_compressed(os.path.join(HERE, "formulas.npz"), cb_in=cb_in, cb_gold=cb_gold, cb_ref=cb_ref, ob_in=ob_in,
                        ob_gold=ob_gold, ob_ref=ob_ref, sh_in=sh_in, sh_gold=sh_gold, sh_ref=sh_ref)


def structures():
    for name in ("grid118", "grid300"):
        g = synthetic.build(name)
        p = packing.pack(g)
        ref = O.ref_structure(p)
        np.savez_compressed(os.path.join(HERE, f"structure_{name}.npz"), n=p.n, cb_params=p.cb_params,
                            cb_idx=p.cb_idx, ob_params=p.ob_params, ob_idx=p.ob_idx, sh_params=p.sh_params,
                            sh_idx=p.sh_idx, **{"ref_" + k: v for k, v in ref.items()})


NEWTON_OUTAGES = 24


def newton_fixtures():
    """newton_<grid>.npz: the packed arrays, each scenario's start and outage mask, the reference-component Newton rows
    [x(n), iterations, ||F||inf, status], and three linear systems with the reference LU's solutions."""
    for name in ("grid118", "grid300"):
        g = synthetic.build(name)
        p = packing.pack(g)
        rs = O.ref_structure(p)
        lu = O.RefLu(rs["row_ptr"], rs["col_idx"])
        outs = synthetic.draw_outages(g, NEWTON_OUTAGES, seed=20261203)
        dis = np.concatenate([np.zeros((1, p.n_elements), np.uint8), p.outage_masks(outs)])
        x0 = np.tile(p.x_base, (dis.shape[0], 1))
        x0[0] = p.x_flat                                 # the base case from a flat start, then the N-1 outages
        rows = np.stack([O.newton_with(
            lambda x, k=k: O.ref_component_fill(p, rs, x, p.target, p.base_row_mode, dis[k]),
            lambda v, b: lu.solve(v, b)[0], x0[k]) for k in range(dis.shape[0])])
        rng = np.random.default_rng(7)
        lin_vals, lin_b, lin_x, lin_xt, lin_trouble = [], [], [], [], []
        for _ in range(3):
            x = p.x_base.copy()
            x[0::2] += rng.uniform(-0.02, 0.02, p.n_bus)
            x[1::2] += rng.uniform(-0.02, 0.02, p.n_bus)
            vals, _F = O.ref_component_fill(p, rs, x, p.target, p.base_row_mode)
            b = rng.standard_normal(p.n)
            xr, trouble = lu.solve(vals, b)
            xt, _ = lu.solve_transposed(vals, b)
            lin_vals.append(vals), lin_b.append(b), lin_x.append(xr), lin_xt.append(xt), lin_trouble.append(trouble)
        np.savez_compressed(os.path.join(HERE, f"newton_{name}.npz"), n=p.n, cb_params=p.cb_params, cb_idx=p.cb_idx,
                            ob_params=p.ob_params, ob_idx=p.ob_idx, sh_params=p.sh_params, sh_idx=p.sh_idx,
                            identity_rows=p.identity_rows, target=p.target, base_row_mode=p.base_row_mode,
                            row_ptr=rs["row_ptr"], col_idx=rs["col_idx"], x0=x0, disabled=dis, ref_rows=rows,
                            lin_vals=np.array(lin_vals), lin_b=np.array(lin_b), lin_x=np.array(lin_x),
                            lin_xt=np.array(lin_xt),
                            lin_trouble=np.array(lin_trouble), ref_nnz_lu=lu.nnz_lu, ref_levels=lu.levels)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else O.reference_root()
    if not ref:
        sys.exit("no reference tree: pass its path or set OLF_REFERENCE")
    O.build(ref)
    formulas(ref)
    structures()
    newton_fixtures()
    print("fixtures written to", HERE)
