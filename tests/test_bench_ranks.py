"""The multi-GPU form of the benchmark, on the CPU with two gloo ranks.

The path does not shard: with N GPUs every rank runs its own replica of the
system, and the job's time is the slowest rank's device time (replicas only).
* ``max_over_ranks`` gives every rank the maximum of the ranks' values;
* ``job_throughput`` counts every rank's bodies over that time;
* the reference arm under a multi-rank launch runs and prints on rank 0 only.
"""
import io
import json
import os
import socket
from contextlib import redirect_stdout
from datetime import timedelta

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        job_ms = bench.max_over_ranks(100.0 + 25.0 * rank, dist, "cpu")  # rank 1 is the slow replica
        value = bench.job_throughput(world, 1000, 10, job_ms)
        q.put((rank, job_ms, value))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    try:
        for _ in range(2):
            rank, job_ms, value = q.get(timeout=120)
            got[rank] = (job_ms, value)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert got[0] == got[1]
    job_ms, value = got[0]
    assert job_ms == 125.0
    assert value == pytest.approx(2 * 1000 * 10 / 0.125)


def test_without_a_process_group_the_value_is_the_rank_s_own():
    import bench
    assert bench.max_over_ranks(42.0, None, "cpu") == 42.0
    assert bench.job_throughput(1, 131072, 100, 555.0) == pytest.approx(131072 * 100 / 0.555)


def test_reference_arm_prints_on_rank_zero_only():
    import bench

    class Args:
        steps, warmup = 1, 0
    out = io.StringIO()
    with redirect_stdout(out):
        bench.run_reference(Args(), rank=1, world=2)
    assert out.getvalue() == ""
    old = bench.SHAPE
    bench.SHAPE = "tetra16"  # a workload without a CPU arm answers with its one-line reason, on rank 0
    try:
        out = io.StringIO()
        with redirect_stdout(out):
            bench.run_reference(Args(), rank=0, world=2)
        line = json.loads(out.getvalue())
        assert line["impl"] == "reference" and "unavailable" in line
    finally:
        bench.SHAPE = old
