"""Multi-rank replicas on CPU (gloo, world size 2): the bench's max-over-ranks
timing and whole-job throughput, with no data-path collective."""
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


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    local = 1.0 + rank          # rank 1 is the slow replica
    slow = bench.slowest_rank(local, world, "cpu")
    out[rank] = (slow, bench.replica_throughput(5, world, slow))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        slow, value = res[r]
        assert slow == pytest.approx(2.0)
        assert value == pytest.approx(world * 5 / 2.0)
