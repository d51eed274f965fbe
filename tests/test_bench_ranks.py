"""bench.py's multi-rank arithmetic (one replica per rank, max over ranks,
whole-job throughput) on two gloo ranks on the CPU."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
    m = bench.max_over_ranks(ms, device="cpu")
    out[rank] = (m, bench.replica_throughput(world, 1000, 4, m))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_throughput():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = 29500 + os.getpid() % 2000
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    assert out[0] == out[1]
    m, v = out[0]
    assert m == 15.0
    assert v == pytest.approx(2 * 1000 * 4 / 15e-3)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, device="cpu") == 3.5
    assert bench.replica_throughput(1, 10, 2, 4.0) == pytest.approx(5000.0)
