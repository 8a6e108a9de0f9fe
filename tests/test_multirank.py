"""The multi-rank path of bench.py (replicas, one per GPU) on CPU: two gloo
ranks reduce their timings to the maximum and report the whole-job rate."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms, ms_e2e = bench.max_over_ranks([1.0 + rank, 10.0 * (rank + 1)], "cpu")
        rate = bench.whole_job_rate(world, 1000, 4, 10, ms)
        q.put((rank, ms, ms_e2e, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, ms_e2e, rate in got:
        assert ms == 2.0 and ms_e2e == 20.0
        # 2 ranks x 1000 DOF x 4 stages x 10 steps in 2 ms
        assert rate == pytest.approx(2 * 1000 * 4 * 10 / 2e-3)


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks([3.0, 4.0], "cpu") == [3.0, 4.0]
    assert bench.whole_job_rate(1, 10, 4, 5, 1000.0) == pytest.approx(200.0)
