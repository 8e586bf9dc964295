"""The multi-GPU form of bench.py is replicas only: every rank runs its own
build, and the job's time is the slowest rank's.  The rank logic (max over
ranks, whole-job throughput) runs here as two gloo processes on the CPU."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    slowest = bench.max_over_ranks(1.0 + rank, dist)  # rank 1 is the slow one
    q.put((rank, slowest, bench.replica_throughput(1e9, world, slowest)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for rank, slowest, gteps in out:
        assert slowest == 2.0
        assert gteps == pytest.approx(1.0)  # 2 replicas x 1e9 edges in 2 s


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.replica_throughput(2e9, 1, 2.0) == pytest.approx(1.0)
