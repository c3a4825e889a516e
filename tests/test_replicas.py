"""Multi-GPU form of the benchmark: N independent replicas (one grid per rank, no
data-path collective).  The only collectives are the barrier and the max-over-ranks
of the device time; they are exercised here with two `gloo` ranks on the CPU."""
from __future__ import annotations

import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

import bench  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, times: list, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        dist.barrier()
        ms_max = bench.max_over_ranks(times[rank], dist, "cpu")
        dist.barrier()
        out.put((rank, ms_max, bench.job_value(1000, 10, world, ms_max)))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    world, times = 2, [12.5, 17.25]
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, times, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, ms_max, value in res:
        assert ms_max == max(times)
        # whole-job throughput: every rank's cells x steps over the slowest rank's time
        assert value == pytest.approx(1000 * 10 * world / (max(times) / 1e3))


def test_single_process_needs_no_collective():
    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0
    assert bench.job_value(100, 2, 1, 1000.0) == pytest.approx(200.0)
