"""Multi-process host logic of a multi-GPU bench run, on CPU with gloo.

A run on N GPUs is N independent replicas (one process per GPU); what the
ranks share is the timing: every rank takes the slowest rank's time, and the
whole-job rate counts every rank's cells.  Two ranks here stand in for two
GPUs: each reports a different time, and both must see the maximum and the
same whole-job rate.
"""
import os
import socket
import sys
from datetime import timedelta

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        m = bench.max_over_ranks(ms, dist, device="cpu")
        rate = bench.whole_job_rate(world, 1000, 4, m)
        dist.barrier()
        q.put((rank, m, rate))
    finally:
        dist.destroy_process_group()


def test_ranks_report_the_slowest_time_and_the_whole_job_rate():
    mp = pytest.importorskip("torch.multiprocessing")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        got = sorted(q.get(timeout=120) for _ in range(world))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0] * world
    for rank, m, rate in got:
        assert m == 15.0
        assert rate == world * 1000 * 4 / (15.0 * 1e-3)


def test_single_process_needs_no_group():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, None) == 12.5
    assert bench.whole_job_rate(1, 256 ** 3, 100, 2700.0) == 256 ** 3 * 100 / 2.7
