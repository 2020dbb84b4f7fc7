"""The multi-GPU path of bench.py is replicas only: each rank runs its own
solve and the job reports cells x steps x ranks over the slowest rank's time.
This runs that aggregation with world_size 2 over gloo on CPU."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, ms_per_rank, out):
    import datetime
    import sys

    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    m = bench.reduce_max(ms_per_rank[rank], dist, "cpu")
    out[rank] = (m, bench.replica_throughput(world, 1000, 10, m))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        ms = [40.0, 50.0]
        mp.start_processes(_worker, args=(2, _free_port(), ms, out), nprocs=2, join=True,
                           start_method="spawn")
        res = dict(out)
    assert res[0] == res[1]
    m, v = res[0]
    assert m == 50.0
    assert v == pytest.approx(2 * 1000 * 10 / 0.05 / 1e6)
