"""World-size-2 gloo run of the sharded N-1 host path (CPU; the per-rank solver is the oracle)."""
import os
import socket

import numpy as np
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
