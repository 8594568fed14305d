"""The multi-GPU path of bench.py runs replicas: every rank solves its own
copy of the workload and the job is timed by the slowest rank.  This checks
that aggregation on two gloo ranks on the CPU (the GPU box uses NCCL with the
same calls)."""

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
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    ms_local = 100.0 + 25.0 * rank   # rank 1 is the slow one
    ms = bench.max_over_ranks(ms_local, dist, device="cpu")
    out[rank] = (ms, bench.job_throughput(10, world, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_job_throughput_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        ms, thr = out[r]
        assert ms == 125.0                      # the slowest rank's time on every rank
        assert abs(thr - 10 * 2 / 0.125) < 1e-9  # all ranks' steps over that time


def test_single_rank_passthrough():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.job_throughput(20, 1, 500.0) == 40.0
