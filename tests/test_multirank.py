"""The multi-rank (replicas) plumbing of bench.py on CPU: two gloo ranks."""

from __future__ import annotations

import datetime
import os
import pathlib
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank times its own replica; the job's time is the slowest rank's
        got = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
        out.put((rank, got))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: 15.0, 1: 15.0}


def test_max_over_ranks_single_process():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5


def test_reference_arm_runs_on_rank_zero_only(capsys):
    """Under torchrun the other ranks of the CPU reference arm exit without work."""
    sys.path.insert(0, str(ROOT))
    import argparse

    import bench

    bench.reference_arm(argparse.Namespace(steps=1, warmup=0, gpus=2), rank=1, world=2)
    assert capsys.readouterr().out == ""


if __name__ == "__main__":
    pytest.main([__file__])
