"""Replica logic of bench.py on two CPU ranks (gloo): each rank's share of
independent problems, whole-job totals and the max-over-ranks time.  No
data-path collective exists; these are the only cross-rank steps."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    from neko_b200 import workloads
    specs = workloads.uneven_specs(37, seed=4)
    mine = bench.shard(specs, rank, world)
    t = 1.0 + rank  # this rank's device time
    tmax = bench.max_over_ranks(t, world)
    n_all = bench.sum_over_ranks(len(mine), world)
    bench.barrier(world)
    q.put((rank, [sp["rhs_seed"] for sp in mine], tmax, n_all))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_sharding_and_reductions():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from neko_b200 import workloads
    seeds = [sp["rhs_seed"] for sp in workloads.uneven_specs(37, seed=4)]
    got = sorted(s for _, mine, _, _ in out for s in mine)
    assert got == sorted(seeds)  # every problem on exactly one rank
    for rank, mine, tmax, n_all in out:
        assert tmax == 2.0 and n_all == 37
        assert len(mine) in (18, 19)
