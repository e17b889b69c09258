"""The multi-GPU path of the bench: independent replicas, timed as the max over ranks.

The path shards into independent alignments with no data-path exchange, so N GPUs run
N replicas; the only collective is the max over ranks of the timed seconds.  Checked
here with two gloo ranks on the CPU.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        seconds = 1.0 + rank  # rank 1 is the slow one
        m = bench.max_over_ranks_of(seconds, dist, "cpu")
        out[rank] = (m, bench.replica_throughput(world, 320, m))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1] == (2.0, 320.0)


def test_single_process_has_no_reduction():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks_of(3.5, None, "cpu") == 3.5
    assert bench.replica_throughput(1, 320, 0.5) == pytest.approx(640.0)
