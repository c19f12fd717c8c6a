"""bench.py's replica timing with two ranks on the CPU (gloo): every rank's device time enters
the job time as the maximum over ranks, and the whole-job rate counts the units of all ranks."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        rate, max_ms = bench.job_rate(100.0 * (rank + 1), 3, world, torch, torch.device("cpu"), dist)
        e2e, e2e_max = bench.job_rate(40.0 + rank, 1, world, torch, torch.device("cpu"), dist)
        out.put((rank, rate, max_ms, e2e, e2e_max))
    finally:
        dist.destroy_process_group()


def test_job_rate_is_max_over_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for rank, rate, max_ms, e2e, e2e_max in res:
        assert max_ms == 200.0 and abs(rate - 2 * 3 / 0.2) < 1e-9
        assert e2e_max == 41.0 and abs(e2e - 2 / 0.041) < 1e-9


def test_single_rank_needs_no_process_group():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    rate, max_ms = bench.job_rate(250.0, 5, 1, torch, torch.device("cpu"), None)
    assert max_ms == 250.0 and abs(rate - 20.0) < 1e-12
