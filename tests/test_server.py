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
    with n34.Server(workers=2, max_batch_graphs=16, route=n34.ROUTE_ONDEMAND) as srv:
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


def _estimates(g):
    """The server's admission estimates (server.cu): 40 B per oriented edge
    and 80 B per out-wedge for a pass; the direct variant adds 33 B per
    out-triple (its clique list, incidence and flags)."""
    D = g.D.astype(np.int64)
    w = int((D * (D - 1) // 2).sum())
    t3 = int((D * (D - 1) * (D - 2) // 6).sum())
    on = 40 * g.m + 80 * w
    return on, on + 33 * t3, t3


def test_memory_routing_chooses_the_variant_and_direct_unions_match(n34, oracle):
    """With NUCLEUS34_ROUTE_MEMORY a request is direct when its direct
    estimate is at most budget / direct_div: the small graphs here go direct
    (in shared direct unions, clique lists per request), the larger ones
    on-demand; every result equals the graph decomposed alone."""
    graphs = _mixed_graphs(n34, 24, 5)
    budget = 8 << 30
    div = 2048  # threshold 4 MiB: about two thirds of these graphs go direct
    want_direct = [_estimates(g)[1] <= budget // div and _estimates(g)[2] < 2 ** 32 for g in graphs]
    assert any(want_direct) and not all(want_direct)
    with n34.Server(workers=2, max_batch_graphs=8, mem_budget_bytes=budget, direct_div=div) as srv:
        ids = [srv.submit(g, cliques=False, triangles=True) for g in graphs]
        dgraphs = [g for g, d in zip(graphs, want_direct) if d][:4]
        cid = [srv.submit(g, cliques=True) for g in dgraphs]
        direct_passes = set()
        for i, rid in enumerate(ids):
            info = srv.wait(rid, timeout_ms=300000)
            assert info["status"] == 0
            assert info["direct"] == want_direct[i], i
            if info["direct"]:
                direct_passes.add(info["pass"])
            o = oracle.decompose(graphs[i])
            k, tris = srv.copy_k(rid, info["triangle_count"], with_tris=True)
            assert np.array_equal(k, o.k) and np.array_equal(tris, o.tris)
            assert info["four_clique_count"] == o.Q
        for g, rid in zip(dgraphs, cid):
            info = srv.wait(rid, timeout_ms=300000)
            assert info["direct"]
            o = oracle.decompose(g, quds_cap=1 << 30)
            q = srv.copy_quds(rid, 0, info["four_clique_count"])
            assert np.array_equal(q, o.quds), "a request's clique list from a direct union"
        st = srv.stats()
        assert st["direct_served"] == sum(want_direct) + len(cid)
        assert len(direct_passes) < sum(want_direct)  # direct requests shared passes


def test_two_device_slots_serve_every_request(n34):
    """Workers over two device slots (here both on GPU 0, each with its own
    budget): every request is served once with the result of the graph
    alone."""
    graphs = _mixed_graphs(n34, 16, 9)
    alone = [n34.decompose(g, variant="ondemand", n_quds=0) for g in graphs]
    with n34.Server(workers=1, devices=[0, 0], mem_budget_bytes=6 << 30, route=n34.ROUTE_ONDEMAND) as srv:
        ids = [srv.submit(g) for g in graphs]
        for i, rid in enumerate(ids):
            info = srv.wait(rid, timeout_ms=300000)
            assert np.array_equal(srv.copy_k(rid, info["triangle_count"]), alone[i].k)
        st = srv.stats()
        assert st["devices"] == 2 and st["workers"] == 2 and st["served"] == len(graphs)
        assert st["budget_bytes"] == 2 * (6 << 30)


def test_one_run_at_a_time_serves_every_request(n34, oracle):
    """With concurrent_runs = 1 the workers still build unions and copy
    results concurrently, but one decomposition runs at a time on the slot;
    every request (both variants) gets the result of its graph alone."""
    graphs = _mixed_graphs(n34, 14, 21)
    with n34.Server(workers=3, max_batch_graphs=4, concurrent_runs=1) as srv:
        ids = [srv.submit(g) for g in graphs]
        for g, rid in zip(graphs, ids):
            info = srv.wait(rid, timeout_ms=300000)
            assert np.array_equal(srv.copy_k(rid, info["triangle_count"]), oracle.decompose(g).k)
        st = srv.stats()
        assert st["served"] == len(graphs) and st["passes"] >= len(graphs) // 4


def test_admission_estimates_bound_measured_peaks(n34):
    """The per-edge, per-wedge and per-triple constants bound the measured
    peak device bytes of each variant (the peak counts every allocation of
    the run, the CSR included)."""
    cases = [n34.gen_rmat(s, ef, 3) for s, ef in ((9, 8), (11, 16), (13, 24))] + \
            [n34.gen_rgg(n, d, 4) for n, d in ((5000, 16.0), (40000, 48.0))] + [n34.gen_ws(8000, 10, 0.1, 2)]
    for s, t in cases:
        g = n34.graph_from_edges(s, t)
        on, direct, _ = _estimates(g)
        with n34.Context() as ctx:
            ctx.upload(g)
            r_on = ctx.run("ondemand")
            r_dir = ctx.run("direct")
        assert r_on["peak_device_bytes"] <= on, (g.n, g.m, r_on["peak_device_bytes"], on)
        assert r_dir["peak_device_bytes"] <= direct, (g.n, g.m, r_dir["peak_device_bytes"], direct)
