"""The N > 1 plumbing of bench.py (independent replicas, one per GPU) on two
CPU ranks over gloo: the max-over-ranks timing, the barrier, and that only
rank 0 of the reference arm runs and prints."""
from __future__ import annotations

import os
import socket
import sys

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        bench.barrier(world)
        slowest = bench.max_over_ranks(world, 10.0 + rank)      # per-rank "ms per step"
        value = world * 1000.0 / slowest                         # whole-job solves/s, as the bench reports it
        bench.barrier(world)
        out.put((rank, slowest, value))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_replica():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert [g[1] for g in got] == [11.0, 11.0]
    assert got[0][2] == pytest.approx(2 * 1000.0 / 11.0)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    import argparse

    sys.path.insert(0, ROOT)
    import bench

    args = argparse.Namespace(gpus=2, steps=1, warmup=3)
    bench.run_reference(args, 2, 1)   # rank 1: no work, no output
    assert capsys.readouterr().out == ""
