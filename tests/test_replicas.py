"""The multi-GPU path of the benchmark is replicas only: every rank multiplies
its own operands, no collective touches the data, and the device time is the
max over ranks.  This runs that host logic as two gloo ranks on the CPU."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t = bench.max_over_ranks(10.0 + rank, dist, torch.device("cpu"))
    seeds = bench.replica_seeds(rank)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, t, seeds))


def test_two_replicas_max_time_and_distinct_operands():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [11.0, 11.0]          # both ranks see the slowest
    assert got[0][2] != got[1][2]                        # independent operands


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, None) == 3.5
