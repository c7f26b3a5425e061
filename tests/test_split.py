"""Replicas over several GPUs: the split of independent graphs
(nucleus34_split_plan) and its merge, on the CPU.

- The plan covers every graph exactly once, is deterministic, and stays
  within the greedy longest-processing-time bound (4/3 of the optimum, which
  is at least the largest cost and the mean load).
- Two gloo ranks (127.0.0.1) each derive the same plan from the same inputs
  without exchanging it, decompose their own share (here with the CPU oracle
  standing in for the device, so no GPU is needed), and all_gather the
  results; every graph's k then equals the oracle's on the whole set and
  comes from exactly one rank."""
import hashlib
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_plan_covers_balances_and_repeats(n34):
    rng = np.random.default_rng(3)
    for count, parts in ((0, 3), (1, 4), (7, 3), (500, 8), (4096, 2)):
        costs = (rng.pareto(1.2, count) * 1000).astype(np.uint64) + 1
        part_of, load = n34.split_plan(costs, parts)
        assert part_of.shape == (count,) and np.all(part_of < parts)
        got = np.zeros(parts, np.uint64)
        np.add.at(got, part_of.astype(np.int64), costs)
        assert np.array_equal(got, load)
        if count:
            opt_lb = max(int(costs.max()), int(costs.sum()) / parts)
            assert int(load.max()) <= 4 / 3 * opt_lb + 1
        again, _ = n34.split_plan(costs, parts)
        assert np.array_equal(part_of, again)


def test_plan_rejects_zero_parts(n34):
    with pytest.raises(n34.Nucleus34Error) as ei:
        n34.split_plan([1, 2, 3], 0)
    assert ei.value.code == n34.E_INVALID


def test_graph_cost_is_edges_plus_out_wedges(n34):
    s, t = n34.gen_rmat(9, 8, 2)
    g = n34.graph_from_edges(s, t)
    D = g.D.astype(np.int64)
    assert n34.graph_cost(g) == g.m + int((D * (D - 1) // 2).sum())


def _graphs(n34):
    out = []
    for i in range(12):
        if i % 3 == 0:
            s, t = n34.gen_rmat(7 + i % 4, 8 + i, 100 + i)
        elif i % 3 == 1:
            s, t = n34.gen_ws(300 + 50 * i, 10, 0.1, 200 + i)
        else:
            s, t = n34.gen_rgg(1500 + 100 * i, 20.0, 300 + i)
        out.append(n34.graph_from_edges(s, t))
    return out


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    for p in (os.path.join(ROOT, "gpu-nucleus34_b200"), os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    from datetime import timedelta
    import torch.distributed as tdist
    import nucleus34 as n34
    import oracle
    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        graphs = _graphs(n34)
        part_of, _ = n34.split_plan([n34.graph_cost(g) for g in graphs], world)
        mine = {}
        for i, g in enumerate(graphs):
            if part_of[i] == rank:
                o = oracle.decompose(g)
                mine[i] = (rank, int(o.T), hashlib.sha256(o.k.astype(np.int32).tobytes()).hexdigest())
        gathered = [None] * world
        tdist.all_gather_object(gathered, mine)
        if rank == 0:
            merged = {}
            for part in gathered:
                for i, v in part.items():
                    assert i not in merged, "a graph was decomposed by two ranks"
                    merged[i] = v
            out["merged"] = merged
            out["plan"] = [int(x) for x in part_of]
    finally:
        tdist.destroy_process_group()


def test_two_gloo_ranks_split_and_merge(n34, oracle):
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
        p.join(300)
        assert p.exitcode == 0
    graphs = _graphs(n34)
    merged, plan = out["merged"], out["plan"]
    assert sorted(merged) == list(range(len(graphs)))
    assert {r for r, _, _ in merged.values()} == {0, 1}
    for i, g in enumerate(graphs):
        o = oracle.decompose(g)
        rank, T, kh = merged[i]
        assert rank == plan[i]
        assert T == o.T and kh == hashlib.sha256(o.k.astype(np.int32).tobytes()).hexdigest()
