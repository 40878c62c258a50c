"""Multi-GPU bench plumbing (replicas: the operator has no cross-GPU
exchange) on CPU with two gloo ranks: every rank sees the max over ranks of
its timed region, the whole-job value counts all ranks' steps, and the
reference arm runs on rank 0 only."""
import io
import json
import os
import sys
import contextlib

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        ms = 100.0 + 50.0 * rank                  # rank 1 is slower
        mx = bench.reduce_over_ranks(ms, dist, "cpu")
        mn = bench.reduce_over_ranks(ms, dist, "cpu", "min")
        val = bench.replica_throughput(10, world, mx)

        class A:
            workload = "2d128x1"
            steps = 1
            warmup = 0
            gpus = world
        out = io.StringIO()
        with contextlib.redirect_stdout(out):
            if rank != 0:
                bench.run_reference_arm(A, rank)   # must return silently
        q.put((rank, mx, mn, val, out.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregation_on_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q))
             for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, mn, val, out in res:
        assert mx == 150.0 and mn == 100.0
        assert abs(val - 2 * 10 / 0.150) < 1e-9
        assert out == ""
