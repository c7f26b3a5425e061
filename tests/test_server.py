"""Serving loop (nucleus34_server_*): requests submitted concurrently are
batched into shared passes; each request's triangles, counts and k must equal
the graph decomposed alone (bit for bit), whether it ran alone or in a mix,
and a request for its clique list is served by the direct variant."""
import threading

import numpy as np
import pytest

from test_batch import _mixed_graphs

pytestmark = pytest.mark.gpu


def test_requests_alone_and_in_a_mix_give_the_same_results(n34, oracle):
    graphs = _mixed_graphs(n34, 40, 11)
    alone = [n34.decompose(g, variant="ondemand", n_quds=0) for g in graphs]
    with n34.Server(workers=2, max_batch_graphs=16) as srv:
        # the mix: all submitted at once from two threads
        ids = [None] * len(graphs)

        def submit(lo, hi):
            for i in range(lo, hi):
                ids[i] = srv.submit(graphs[i], triangles=True)

        th = [threading.Thread(target=submit, args=(0, 20)), threading.Thread(target=submit, args=(20, 40))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        passes = set()
        for i, rid in enumerate(ids):
            info = srv.wait(rid, timeout_ms=120000)
            passes.add(info["pass"])
            assert info["status"] == 0 and not info["direct"]
            assert info["triangle_count"] == alone[i].result["triangle_count"]
            assert info["four_clique_count"] == alone[i].result["four_clique_count"]
            assert info["k_max"] == alone[i].result["k_max"]
            assert info["k_avg"] == alone[i].result["k_avg"]
            k, tris = srv.copy_k(rid, info["triangle_count"], with_tris=True)
            assert np.array_equal(k, alone[i].k) and np.array_equal(tris, alone[i].tris)
            srv.release(rid)
        assert len(passes) < len(graphs)  # requests shared passes
        # one request alone
        rid = srv.submit(graphs[3])
        info = srv.wait(rid)
        assert np.array_equal(srv.copy_k(rid, info["triangle_count"]), alone[3].k)
        # routed to the direct variant: the clique list comes back
        rid = srv.submit(graphs[0], cliques=True)
        info = srv.wait(rid)
        assert info["direct"]
        o = oracle.decompose(graphs[0], quds_cap=5)
        assert np.array_equal(srv.copy_k(rid, info["triangle_count"]), o.k)
        q = srv.copy_quds(rid, 0, min(5, info["four_clique_count"]))
        assert np.array_equal(q, o.quds[: len(q)])
        st = srv.stats()
        assert st["served"] == len(graphs) + 2 and st["pending"] == 0


def test_server_reports_request_errors_and_timeouts(n34):
    with n34.Server(workers=1, mem_budget_bytes=8 << 20) as srv:
        a, b = n34.gen_rmat(14, 16, 1)
        rid = srv.submit(n34.graph_from_edges(a, b))
        with pytest.raises(n34.Nucleus34Error) as ei:
            srv.wait(rid)
        assert ei.value.code == n34.E_OOM_BUDGET
        with pytest.raises(n34.Nucleus34Error) as ei:
            srv.wait(12345)
        assert ei.value.code == n34.E_INVALID


def test_concurrent_contexts_give_sequential_results(n34):
    """Two contexts decomposing at the same time (separate streams sharing the
    SMs) produce the sequential results: kernels whose blocks start in
    several waves must not depend on which blocks started first."""
    specs = [("rmat", 14, 16, 21), ("rgg", 60000, 40.0, 22), ("rmat", 15, 12, 23), ("ws", 40000, 10, 24)]
    graphs = []
    for kind, x, y, s in specs:
        if kind == "rmat":
            a, b = n34.gen_rmat(x, y, s)
        elif kind == "rgg":
            a, b = n34.gen_rgg(x, y, s)
        else:
            a, b = n34.gen_ws(x, y, 0.1, s)
        graphs.append(n34.graph_from_edges(a, b))
    want = [n34.decompose(g, variant="ondemand", n_quds=0).k for g in graphs]
    errors = []

    def worker(order):
        with n34.Context() as ctx:
            for rep in range(6):
                for i in order:
                    ctx.upload(graphs[i])
                    r = ctx.run("ondemand")
                    if not np.array_equal(ctx.copy_k(int(r["triangle_count"])), want[i]):
                        errors.append((order, rep, i))

    th = [threading.Thread(target=worker, args=([0, 1, 2, 3],)), threading.Thread(target=worker, args=([3, 2, 1, 0],))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors
