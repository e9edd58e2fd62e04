"""Packed arrays of one network, in the layout the reference's Java extraction hands to its native library.

Mirrors, for the element families of the synthetic grids:

* ``GpuAcFamilyPacker.java:140-181`` -- closed branch ``{y, g1, g2, b1, b2, ksi, r1, a1}`` with 12 indices
  ``{P1, Q1, P2, Q2, ph1, v1, ph2, v2, a1col, r1col, altQ1, altQ2}``; open branch ``{y, ksi, g1, b1, g2, b2, r1}``
  with 6 indices ``{P1, Q1, P2, Q2, v1, v2}`` (-1 on the open side); fixed shunt ``{g, b}`` with 5 indices
  ``{P, Q, v, bcol, altQ}``.
* the stable-row numbering (``StableRowIndexing.java:30``; ``ExtractionColumns.java:53-62``): bus b owns variable
  column 2b (BUS_PHI) and 2b+1 (BUS_V); its P balance sits on row 2b and its Q balance on row 2b+1.
* the activation (``GpuAcActivationExtractor.java:84-272``): slack PHI row and PV V rows hold identities
  (``GpuRowMode.FIXED_VARIABLE``), every other row its power equation (``EQUATION``); targets are the net injections
  (P rows, PQ Q rows), the voltage set points (PV V rows) and the slack angle.
* the reactive-limit entries (``ReactiveLimitsPacker.java:76``): per voltage-controlling bus its V row, Q limits, load
  Q and voltage target, plus the forced-PV election keys (nominal V, target-P row, id rank).
* the pi model (``SimplePiModel``; ``GpuBatchSideOpen.java:59-60``): y = 1/|z|, ksi = atan2(r, x).

The disabled mask of a scenario follows the element order closed, open, shunt (``BatchSolveNative.java:81-83``).
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np

from .synthetic import Grid

# Row modes (GpuRowMode.java / native gpu_row_mode.cuh)
FIXED_VARIABLE = 0
EQUATION = 1
BUS_TARGET_Q = 4

# Variable types of the MAX_VOLTAGE_CHANGE step clamp, by OLF's AcVariableType ordinal
# (codes/gpu_ac_variable_type.cuh): 0 BUS_V (voltage magnitude), 1 BUS_PHI (angle)
VAR_V = 0
VAR_PHI = 1


@dataclasses.dataclass
class ReactiveLimits:
    voltage_row: np.ndarray      # int32 [nRl]   the bus's V row (2b+1)
    min_q: np.ndarray            # float64 [nRl] generator Q limits (pu)
    max_q: np.ndarray
    load_q: np.ndarray           # load Q at the bus (q_gen = q_flows + load_q)
    target_v: np.ndarray         # voltage set point restored on a switch back to PV
    nom_v: np.ndarray            # election key 1: nominal voltage (higher stays PV)
    p_row: np.ndarray            # election key 2: the bus's P row (its target P is read live)
    static_p: np.ndarray         # ... or this value when p_row < 0
    id_rank: np.ndarray          # election key 3: lower id rank wins


@dataclasses.dataclass
class DistributedSlack:
    """Bus-level distributed-slack participants with static factors (the reference's GpuDistributedSlackFactorMode
    STATIC, DistributedSlackNative tables): per participating bus its P row, factor, base target P and the bounds of
    its target's move; the slack bus's angle row, whose closed-branch P is compared with slack_target_p."""
    row: np.ndarray              # int32 [nDs]  the bus's P row (2b)
    factor: np.ndarray           # float64 [nDs] participation factor (normalised by the engine)
    base_target: np.ndarray      # float64 [nDs] target P before any distribution
    max_delta: np.ndarray        # float64 [nDs] largest upward move of the target
    min_delta: np.ndarray        # float64 [nDs] largest downward move (<= 0)
    slack_row: int
    slack_target_p: float


def distributed_slack(g: Grid, p: "Packed") -> DistributedSlack:
    """Generator buses other than the slack share the slack's mismatch in proportion to their Pmax, within
    [0, Pmax] of generation (the P_MAX balance type with static factors)."""
    nb = g.n_bus
    pmax = np.zeros(nb)
    pgen = np.zeros(nb)
    np.add.at(pmax, g.gen_bus, g.gen_pmax)
    np.add.at(pgen, g.gen_bus, g.gen_p)
    buses = np.array(sorted(set(int(b) for b in g.gen_bus) - {int(g.slack)}), dtype=np.int64)
    rows = (2 * buses).astype(np.int32)
    slack_p = pgen[g.slack] - float(g.load_p[g.load_bus == g.slack].sum())
    return DistributedSlack(row=rows, factor=pmax[buses].copy(), base_target=p.target[rows].copy(),
                            max_delta=pmax[buses] - pgen[buses], min_delta=-pgen[buses],
                            slack_row=int(2 * g.slack), slack_target_p=float(slack_p))


@dataclasses.dataclass
class Packed:
    n: int
    cb_params: np.ndarray        # float64 [nCb, 8]
    cb_idx: np.ndarray           # int32   [nCb, 12]
    ob_params: np.ndarray        # float64 [nOb, 7]
    ob_idx: np.ndarray           # int32   [nOb, 6]
    sh_params: np.ndarray        # float64 [nSh, 2]
    sh_idx: np.ndarray           # int32   [nSh, 5]
    identity_rows: np.ndarray    # int32   [k]
    x_flat: np.ndarray           # flat start (V = 1 or the set point, angles 0)
    x_base: Optional[np.ndarray]  # base-case solution (the N-1 warm start), when known
    target: np.ndarray           # float64 [n]
    base_row_mode: np.ndarray    # int32 [n]
    var_type: np.ndarray         # int32 [n]
    rl: Optional[ReactiveLimits]
    n_bus: int

    @property
    def n_cb(self) -> int:
        return int(self.cb_idx.shape[0])

    @property
    def n_ob(self) -> int:
        return int(self.ob_idx.shape[0])

    @property
    def n_sh(self) -> int:
        return int(self.sh_idx.shape[0])

    @property
    def n_elements(self) -> int:
        return self.n_cb + self.n_ob + self.n_sh

    def outage_masks(self, branches: np.ndarray) -> np.ndarray:
        """uint8 [nS, nElements]: scenario s disables closed-branch element ``branches[s]``."""
        m = np.zeros((branches.shape[0], self.n_elements), dtype=np.uint8)
        m[np.arange(branches.shape[0]), branches] = 1
        return m


def pi_model(r, x):
    """SimplePiModel's admittance magnitude and angle: y = 1/|z|, ksi = atan2(r, x)."""
    return 1.0 / np.hypot(r, x), np.arctan2(r, x)


def pack(g: Grid, with_reactive_limits: Optional[bool] = None) -> Packed:
    nb = g.n_bus
    n = 2 * nb
    p_row = 2 * np.arange(nb)
    q_row = 2 * np.arange(nb) + 1
    phi_col = p_row
    v_col = q_row
    y, ksi = pi_model(g.r, g.x)
    bh = g.b / 2
    cb_params = np.stack([y, np.zeros_like(y), np.zeros_like(y), bh, bh, ksi, g.ratio, np.zeros_like(y)], axis=1)
    f, t = g.f, g.t
    m1 = -np.ones_like(f)
    cb_idx = np.stack([p_row[f], q_row[f], p_row[t], q_row[t], phi_col[f], v_col[f], phi_col[t], v_col[t],
                       m1, m1, m1, m1], axis=1).astype(np.int32)
    nob = g.open_bus.shape[0]
    oy, oksi = pi_model(g.open_r, g.open_x)
    obh = g.open_b / 2
    ob_params = np.stack([oy, oksi, np.zeros(nob), obh, np.zeros(nob), obh, np.ones(nob)], axis=1) if nob else \
        np.zeros((0, 7))
    ob_idx = np.zeros((nob, 6), dtype=np.int32)
    for k in range(nob):
        b = int(g.open_bus[k])
        if g.open_side[k] == 1:                       # side 2 open: p1/q1 at bus1, variable v1
            ob_idx[k] = [p_row[b], q_row[b], -1, -1, v_col[b], -1]
        else:                                         # side 1 open: p2/q2 at bus2, variable v2
            ob_idx[k] = [-1, -1, p_row[b], q_row[b], -1, v_col[b]]
    nsh = g.shunt_bus.shape[0]
    sh_params = np.stack([g.shunt_g, g.shunt_b], axis=1) if nsh else np.zeros((0, 2))
    sb = g.shunt_bus
    sh_idx = np.stack([p_row[sb], q_row[sb], v_col[sb], -np.ones(nsh, dtype=np.int64),
                       -np.ones(nsh, dtype=np.int64)], axis=1).astype(np.int32) if nsh else \
        np.zeros((0, 5), dtype=np.int32)

    target = np.zeros(n)
    np.add.at(target, p_row[g.gen_bus], g.gen_p)
    np.add.at(target, p_row[g.load_bus], -g.load_p)
    np.add.at(target, q_row[g.load_bus], -g.load_q)
    mode = np.full(n, EQUATION, dtype=np.int32)
    mode[v_col[g.gen_bus]] = FIXED_VARIABLE
    target[v_col[g.gen_bus]] = g.gen_vset
    mode[phi_col[g.slack]] = FIXED_VARIABLE
    target[phi_col[g.slack]] = 0.0
    var_type = np.tile(np.array([VAR_PHI, VAR_V], dtype=np.int32), nb)
    x_flat = np.zeros(n)
    x_flat[1::2] = 1.0
    x_flat[v_col[g.gen_bus]] = g.gen_vset
    x_base = None
    if g.base_vm is not None:
        x_base = np.zeros(n)
        x_base[0::2] = g.base_va
        x_base[1::2] = g.base_vm
    rl = None
    use_rl = g.spec.q_limits if with_reactive_limits is None else with_reactive_limits
    if use_rl:
        load_q_bus = np.zeros(nb)
        np.add.at(load_q_bus, g.load_bus, g.load_q)
        gb = g.gen_bus
        rl = ReactiveLimits(
            voltage_row=v_col[gb].astype(np.int32),
            min_q=np.where(np.isfinite(g.gen_minq), g.gen_minq, -1e30),
            max_q=np.where(np.isfinite(g.gen_maxq), g.gen_maxq, 1e30),
            load_q=load_q_bus[gb],
            target_v=g.gen_vset.copy(),
            nom_v=np.full(gb.shape[0], 400.0),
            p_row=p_row[gb].astype(np.int32),
            static_p=g.gen_p.copy(),
            id_rank=np.arange(gb.shape[0], dtype=np.int32),
        )
    return Packed(n, np.ascontiguousarray(cb_params), cb_idx, np.ascontiguousarray(ob_params), ob_idx,
                  np.ascontiguousarray(sh_params), sh_idx, np.zeros(0, dtype=np.int32), x_flat, x_base, target,
                  mode, var_type, rl, nb)
