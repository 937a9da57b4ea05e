"""bench.py on N ranks: every rank times its own decomposition (a replica,
or its shard of the instance batch), the job's time is the maximum over the
ranks, and the whole-job rate counts every rank's edges (replicas: m per
rank; shards: the sum of the shards' edges).  Checked here with two gloo
ranks on the CPU (the same collective calls bench.py makes over NCCL on
GPUs); the reference arm runs on rank 0 only.
"""
import argparse
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r timed 100 + 10 r ms for the device steps and 200 - 10 r ms end to end
        got = bench.max_over_ranks([100.0 + 10 * rank, 200.0 - 10 * rank], world, "cpu")
        # and rank r holds a shard of 1000 + r edges: the job's edges are their sum
        got += bench.sum_over_ranks([1000.0 + rank], world, "cpu")
        out.put((rank, got))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_agree_on_the_slowest_replica():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = dict(out.get(timeout=10) for _ in range(world))
    assert res[0] == res[1] == [110.0, 200.0, 2001.0]


def test_job_rate_counts_every_replica():
    import bench

    # 6,242,304 edges, 2 ranks, 10 steps in 220 ms -> 567.5 M edges/s
    assert bench.job_rate(6242304, 2, 10, 220.0) == pytest.approx(6242304 * 2 * 10 / 0.22)
    assert bench.max_over_ranks([3.0, 4.0], 1, "cpu") == [3.0, 4.0]


def test_reference_arm_runs_on_rank_zero_only():
    import bench

    args = argparse.Namespace(steps=1, warmup=0, gpus=2)
    assert bench.reference_arm(args, rank=1) == 0   # returns at once, no work, no output
