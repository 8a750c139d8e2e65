"""bench.py's multi-rank arithmetic on CPU: two gloo ranks (the GPU run uses
the same code over NCCL, one process per GPU)."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # each rank timed its own steps; the job's time is the slowest rank's
        ms = bench.max_over_ranks(torch, dist, 10.0 + 5.0 * rank)
        q.put((rank, ms, bench.whole_job_rate(world, 65536, 300, ms)))
    finally:
        dist.destroy_process_group()


def test_slowest_rank_sets_the_whole_job_rate():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, ms, rate in got:
        assert ms == 15.0
        assert rate == pytest.approx(2 * 65536 * 300 / 0.015)


def test_single_process_needs_no_group():
    assert bench.max_over_ranks(torch, None, 3.5) == 3.5
    assert bench.whole_job_rate(1, 100, 10, 1000.0) == pytest.approx(1000.0)
