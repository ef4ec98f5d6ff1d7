"""Multi-process plumbing on CPU (gloo, world size 2).

The path shards by particles: every rank integrates its own seed set (the benchmark's weak
scaling) and only the timing / work figures are combined, as the slowest rank's time and
the summed particle-steps.  No GPU is touched here.
"""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    from pygranite_b200 import workloads as W
    # each rank builds its own shard of the workload (seed = rank)
    _, _, seeds = W.config2(n_particles=64, n_snapshots=2, grid=(4, 6, 6), steps=10, seed=rank)
    t, ps = bench.combine_ranks(dist, 10.0 * (rank + 1), 1000 + rank, "cpu")
    out.put((rank, t, ps, float(seeds[0, 0])))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_reduction_and_sharding():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # slowest rank's time, summed work, on every rank
    assert all(r[1] == pytest.approx(20.0) and r[2] == 2001 for r in res)
    # the shards differ (independent seed sets)
    assert res[0][3] != res[1][3]
