"""The replica bookkeeping of ``bench.py --gpus N`` on the CPU.

The solver path does not shard: with N GPUs the bench runs N independent
replicas of the same workload, one process per GPU, with no data-path
collective.  What the ranks share is the bookkeeping: a barrier around the
timed region, the maximum of the per-rank device times, and the whole-job
rate (the steps of all ranks over the slowest rank's time).  These run here
on world size 2 over gloo, with rank-dependent times."""
import os
import socket
import sys
from datetime import timedelta

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        sys.path.insert(0, ROOT)
        import bench
        bench.rank_barrier(dist)
        ms = 100.0 * (rank + 1)  # the last rank is the slowest
        ms_max = bench.max_over_ranks(dist, ms, device="cpu")
        rate = bench.replica_rate(world, 20, ms_max)
        bench.rank_barrier(dist)
        q.put((rank, ms_max, rate))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted(q.get(timeout=120) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    assert [r for r, _, _ in got] == [0, 1]
    for _, ms_max, rate in got:
        assert ms_max == 200.0
        # 2 ranks x 20 steps over the slowest rank's 0.2 s
        assert rate == pytest.approx(200.0)


def test_one_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    bench.rank_barrier(None)
    assert bench.max_over_ranks(None, 3.5) == 3.5
    assert bench.replica_rate(1, 10, 500.0) == pytest.approx(20.0)
