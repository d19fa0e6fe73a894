"""The multi-GPU path is replicas (no data-path collective): bench.py
reports the units all ranks processed over the slowest rank's device time.
Two gloo ranks on the CPU check that reduction (job_rate)."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms, rate = bench.job_rate(10.0 + 5.0 * rank, 100.0 * (rank + 1), dist, "cpu")
        out.put((rank, ms, rate))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_job_rate_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, rate in got:
        assert ms == 15.0  # the slowest rank's time
        assert abs(rate - 300.0 / 0.015) < 1e-6  # all ranks' units over it


def test_job_rate_single_process():
    import bench
    ms, rate = bench.job_rate(20.0, 1000.0, None, "cpu")
    assert ms == 20.0 and rate == 1000.0 / 0.02
