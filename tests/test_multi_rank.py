"""World-size-2 gloo runs of the sharded N-1 path: the host logic with the oracle as the per-rank solver (CPU), and
the engine itself on the GPU in each rank."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "olf-gpu_b200"))
    sys.path.insert(0, os.path.join(root, "tests"))
    import datetime
    import torch.distributed as dist
    from conftest import grid
    from olfgpu import distributed, synthetic
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    g, p = grid("grid118")
    outs = synthetic.outage_candidates(g)[:25]
    st = O.Structure(p)
    rows = distributed.solve_sharded(lambda o: st.solve_batch(p.x_base, p.outage_masks(o), threads=1), outs, rank,
                                     world, costs=np.arange(outs.shape[0])[::-1])
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        q.put(rows)


def test_two_ranks_reassemble_the_single_rank_result(oracle_mod):
    from conftest import grid
    from olfgpu import synthetic
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    rows = q.get(timeout=120)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    g, p = grid("grid118")
    outs = synthetic.outage_candidates(g)[:25]
    ref = oracle_mod.Structure(p).solve_batch(p.x_base, p.outage_masks(outs), threads=1)
    assert np.array_equal(rows, ref)


def test_shards_cover_every_scenario_once():
    from olfgpu.distributed import shard
    for world in (1, 2, 3, 8):
        got = np.sort(np.concatenate([shard(101, r, world, costs=np.random.default_rng(world).random(101))
                                      for r in range(world)]))
        assert np.array_equal(got, np.arange(101))


def _engine_worker(rank, world, port, q):
    """One rank: the engine's own batch context on the GPU, its shard of the outages, the gather and a max-over-ranks
    reduction of the device time over the gloo process group (host-side collectives; no kernel waits on another
    rank)."""
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "olf-gpu_b200"))
    sys.path.insert(0, os.path.join(root, "tests"))
    import datetime
    import torch
    import torch.distributed as dist
    from conftest import grid
    from olfgpu import distributed, native, synthetic
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 90, seed=55)
    s = native.Structure(p, native.PLAN_DENSE_FRONT)
    timing = {}

    def solve(o):
        ctx = native.BatchContext(s, o.shape[0])
        ctx.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
        ctx.set_device_loop(True)
        r = ctx.solve(p.x_base, p.target, p.base_row_mode, p.outage_masks(o))
        timing["ms"] = ctx.last_stats()[0]
        ctx.close()
        return r

    rows = distributed.solve_sharded(solve, outs, rank, world)
    t = torch.tensor([timing["ms"]], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        q.put((rows, float(t[0]), timing["ms"]))


@pytest.mark.gpu
def test_two_engine_ranks_reassemble_the_single_process_result(engine_lib):
    """Two processes, each with the engine's contexts on the GPU inside a torch.distributed (gloo) process group,
    solve their shards; rank 0's gathered rows equal one process solving the whole batch bit for bit, and the reduced
    device time is the maximum over the ranks."""
    from conftest import grid
    from olfgpu import native, synthetic
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_engine_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    rows, ms_max, ms0 = q.get(timeout=300)
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    assert ms_max >= ms0 > 0
    g, p = grid("grid2000")
    outs = synthetic.draw_outages(g, 90, seed=55)
    s = native.Structure(p, native.PLAN_DENSE_FRONT)
    c = native.BatchContext(s, outs.shape[0])
    c.set_schedule(native.LEVELS_SHARED_ALL, 0, 256)
    ref = c.solve(p.x_base, p.target, p.base_row_mode, p.outage_masks(outs))
    assert np.array_equal(rows, ref)
