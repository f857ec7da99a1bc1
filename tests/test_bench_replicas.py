"""bench.py's multi-GPU path (replicas only): the job time is the slowest
rank's, reduced across ranks, and the metric is whole-job MLUPS.  Two gloo
ranks on the CPU stand in for the NCCL ranks of a GPU node."""

import importlib
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    bench = importlib.import_module("bench")
    from datetime import timedelta

    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    try:
        w, r, local = bench.dist_env()
        ms = 100.0 + 25.0 * r  # rank 1 is slower
        ms_max = bench.reduce_max(dist, torch, ms, "cpu")
        q.put((r, w, local, ms_max, bench.job_mlups(w, 2_100_225, 1000, ms_max)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_and_job_metric():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for r, (rank, world, local, ms_max, mlups) in enumerate(res):
        assert (rank, world, local) == (r, 2, r)
        assert ms_max == pytest.approx(125.0)  # every rank reports the slowest
        assert mlups == pytest.approx(2 * 2_100_225 * 1000 / 0.125 / 1e6)


def test_single_process_defaults():
    sys.path.insert(0, ROOT)
    bench = importlib.import_module("bench")
    assert bench.reduce_max(None, torch, 3.5, "cpu") == 3.5
    assert bench.job_mlups(1, 10, 100, 1.0) == pytest.approx(1.0)
