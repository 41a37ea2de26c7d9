"""The multi-process side of bench.py on CPU (gloo, world size 2): the
barrier and the max-over-ranks reduction that time N replicas, and the
reference arm's rule that only rank 0 works."""
import argparse
import os
import socket

import pytest

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        got = bench.max_over_ranks(1.5 + rank, world)
        bench.barrier(world)
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world_2():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 2.5), (1, 2.5)]


def test_single_rank_is_identity():
    assert bench.max_over_ranks(3.25, 1) == 3.25


def test_reference_arm_other_ranks_do_no_work(monkeypatch):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = argparse.Namespace(size=8192, ref_rows=32, steps=1, warmup=3)
    assert bench.reference_arm(args) == 0
