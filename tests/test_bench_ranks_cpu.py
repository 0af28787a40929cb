"""bench.py's multi-rank plumbing on the CPU: two gloo ranks (127.0.0.1), each
with its own timing, agree on the slowest rank's time through max_over_ranks
and report the whole job's rate (both replicas' point-updates over that time);
a single rank needs no process group. The GPU arm runs the same two functions
with NCCL."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        ms = bench.max_over_ranks(torch, dist, world, 100.0 + 25.0 * rank, "cpu")
        rate = bench.whole_job_rate(1000, 10, world, ms)
        out.put((rank, ms, rate))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [125.0, 125.0]
    assert all(g[2] == pytest.approx(1000 * 10 * 2 / 0.125) for g in got)


def test_single_rank_needs_no_group():
    assert bench.max_over_ranks(torch, None, 1, 42.5, "cpu") == 42.5
    assert bench.whole_job_rate(31457280, 20, 1, 1000.0) == 31457280 * 20
