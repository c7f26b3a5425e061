"""Multi-rank bench path on CPU: two gloo ranks (127.0.0.1) each report their
own device time; the job's time is the slowest rank's and its throughput
counts every replica's triangles (bench.py's replicas-only scaling)."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as tdist
    import bench
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = 1.5 + rank  # rank 1 is the slow one
        t = bench.max_over_ranks(mine, "cpu")
        out[rank] = (t, bench.job_value(world, 1000, 3, t))
    finally:
        tdist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        t, v = out[r]
        assert t == pytest.approx(2.5)
        assert v == pytest.approx(2 * 1000 * 3 / 2.5)
