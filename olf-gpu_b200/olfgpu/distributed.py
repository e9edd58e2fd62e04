"""Multi-GPU N-1: scenarios shard across ranks with no collective on the data path (each rank holds a replica of the
structure and solves its own scenarios); the results are gathered to rank 0 on the host, in request order.

The reference is single-GPU; its scenarios are independent units (one disabled mask per scenario,
``branch_fill.cu:133``), so sharding them is exact.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

import numpy as np


def shard(n_items: int, rank: int, world: int, costs: Optional[Sequence[float]] = None) -> np.ndarray:
    """Indices of the items rank `rank` solves: round-robin over the items sorted by decreasing predicted cost
    (stable), so every rank gets a similar share of slow scenarios."""
    order = np.arange(n_items) if costs is None else np.argsort(-np.asarray(costs, dtype=float), kind="stable")
    return np.sort(order[rank::world])


def solve_sharded(solve: Callable[[np.ndarray], np.ndarray], outages: Sequence[int], rank: int, world: int,
                  costs: Optional[Sequence[float]] = None):
    """Every rank solves its shard with `solve` (outages -> per-scenario result rows); rank 0 returns all rows in
    request order, the other ranks None.  The gather is a host-side object gather over the process group."""
    import torch.distributed as dist
    outages = np.asarray(outages)
    idx = shard(outages.shape[0], rank, world, costs)
    local = solve(outages[idx]) if idx.size else None
    parts = [None] * world if rank == 0 else None
    dist.gather_object((idx, local), parts, dst=0)
    if rank != 0:
        return None
    rows = None
    for ix, res in parts:
        if res is None:
            continue
        if rows is None:
            rows = np.zeros((outages.shape[0],) + res.shape[1:], dtype=res.dtype)
        rows[ix] = res
    return rows
