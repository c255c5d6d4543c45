"""CPU test of the multi-GPU path of bench.py with two gloo ranks: every rank is an independent replica; the job
time is the slowest rank's, the throughput counts the work of all ranks (no other data crosses ranks)."""
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


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    ms_local = [40.0, 55.0][rank]
    n_local = [1000, 3000][rank]
    ms, value = bench.replica_throughput(ms_local, n_local, steps=10, dist=dist, device="cpu")
    out[rank] = (ms, value)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_throughput_two_gloo_ranks():
    world = 2
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    for r in range(world):
        ms, value = out[r]
        assert ms == 55.0
        assert value == pytest.approx((1000 + 3000) * 10 / 0.055)


def test_replica_throughput_single_process():
    sys.path.insert(0, ROOT)
    import bench
    ms, value = bench.replica_throughput(20.0, 500, steps=4)
    assert ms == 20.0 and value == pytest.approx(500 * 4 / 0.02)
