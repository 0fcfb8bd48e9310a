"""The multi-GPU path of the benchmark on CPU: two gloo ranks (world size 2).

The step does not shard: with N GPUs the benchmark runs N independent
replicas of the workload, one per rank, and reports whole-job MLUPS over the
slowest rank's time. Here two processes stand in for two ranks and check the
max-over-ranks reduction and the aggregate the benchmark prints.
"""

from __future__ import annotations

import datetime
import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        ms = 100.0 * (rank + 1)  # the second rank is the slow one
        slowest = bench.max_over_ranks(ms, world, torch.device("cpu"))
        out.put((rank, slowest, bench.whole_job_mlups(nodes=2**24, steps=50, ms=slowest, world=world)))
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank_and_the_whole_job():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in results] == [200.0, 200.0]
    # two replicas of 2^24 nodes x 50 steps in 0.2 s
    assert results[0][2] == pytest.approx(2 * 2**24 * 50 / 0.2 / 1e6)


def test_one_rank_needs_no_process_group():
    import bench

    assert bench.max_over_ranks(3.5, 1, None) == 3.5
    assert bench.whole_job_mlups(1000, 10, 1.0, 1) == pytest.approx(10.0)
