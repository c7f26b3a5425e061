"""Batched decomposition (nucleus34_batch_decompose): many graphs in one
device pass as their disjoint union. Every graph's triangles, counts, K_max,
K_avg and k must equal its own one-graph decomposition and the oracle, bit
for bit (integer results; K_avg uses the same 64-bit sum / T)."""
import numpy as np
import pytest


def _mixed_graphs(n34, count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        kind = i % 4
        s = n34.splitmix64(seed * 1000 + i) & 0xffffffff
        if kind == 0:
            a, b = n34.gen_rmat(int(rng.integers(6, 11)), int(rng.integers(8, 20)), s)
        elif kind == 1:
            a, b = n34.gen_ws(int(rng.integers(200, 3000)), 10, 0.1, s)
        elif kind == 2:
            a, b = n34.gen_rgg(int(rng.integers(500, 4000)), float(rng.integers(16, 40)), s)
        else:
            a, b = n34.gen_rmat(int(rng.integers(4, 9)), int(rng.integers(4, 12)), s)
        out.append(n34.graph_from_edges(a, b))
    return out


def test_batch_rejects_bad_members_before_any_device_work(n34):
    a, b = n34.gen_rmat(6, 8, 1)
    g = n34.graph_from_edges(a, b)
    bad = n34.HostGraph(g.n, g.m, g.O.copy(), g.D.copy(), g.E.copy())
    bad.E[0] = g.n + 5
    with pytest.raises(n34.Nucleus34Error) as ei:
        n34.batch_decompose([g, bad])
    assert ei.value.code == n34.E_INVALID
    assert "batch graph 1" in n34.last_error()
    with pytest.raises(n34.Nucleus34Error):
        n34.batch_decompose([])


@pytest.mark.gpu
def test_batch_equals_single_graph_runs_and_oracle(n34, oracle):
    graphs = _mixed_graphs(n34, 24, 4)
    # edge cases inside a batch: an empty graph and a triangle-free path
    graphs.insert(5, n34.graph_from_edges(np.zeros(0, np.uint32), np.zeros(0, np.uint32)))
    graphs.insert(9, n34.graph_from_edges(np.arange(0, 50, dtype=np.uint32), np.arange(1, 51, dtype=np.uint32)))
    with n34.batch_decompose(graphs) as b:
        assert b.result["graphs"] == len(graphs)
        tot_t = tot_q = 0
        for i, g in enumerate(graphs):
            one = n34.decompose(g, variant="ondemand", n_quds=0)
            summ = b.summary(i)
            k, tris = b.copy_k(i, with_tris=True)
            assert summ["triangle_count"] == one.result["triangle_count"]
            assert summ["four_clique_count"] == one.result["four_clique_count"]
            assert summ["k_max"] == one.result["k_max"]
            assert summ["k_avg"] == one.result["k_avg"]
            assert np.array_equal(k, one.k)
            assert np.array_equal(tris, one.tris)
            o = oracle.decompose(g, quds_cap=0)
            assert np.array_equal(k, o.k) and summ["four_clique_count"] == o.Q
            tot_t += summ["triangle_count"]
            tot_q += summ["four_clique_count"]
        assert tot_t == b.result["triangle_count"]
        assert tot_q == b.result["four_clique_count"]


@pytest.mark.gpu
def test_batch_cut_into_passes_by_memory_budget(n34):
    """A budget too small for one union cuts the batch into several passes;
    results are unchanged."""
    graphs = _mixed_graphs(n34, 16, 7)
    single = [n34.decompose(g, variant="ondemand", n_quds=0) for g in graphs]
    T = sum(int(d.result["triangle_count"]) for d in single)
    csr = sum(4 * (g.n + 1) + 8 * g.m for g in graphs)
    done = False
    for parts in (4, 3, 2):
        budget = csr + 80 * T // parts + (24 << 20)
        try:
            b = n34.batch_decompose(graphs, mem_budget_bytes=budget)
        except n34.Nucleus34Error as e:
            assert e.code == n34.E_OOM_BUDGET
            continue
        with b:
            assert b.result["chunks"] >= 2
            for i, d in enumerate(single):
                assert np.array_equal(b.copy_k(i), d.k)
                assert b.summary(i)["four_clique_count"] == d.result["four_clique_count"]
        done = True
        break
    assert done


@pytest.mark.gpu
def test_batch_results_moved_to_host_are_unchanged(n34):
    """NUCLEUS34_OPT_HOST_RESULTS moves every finished pass's k and triangle
    lists to host memory; summaries, k and triangle lists are those of the
    device-resident batch, over several passes."""
    graphs = _mixed_graphs(n34, 16, 7)
    single = [n34.decompose(g, variant="ondemand", n_quds=0) for g in graphs]
    T = sum(int(d.result["triangle_count"]) for d in single)
    csr = sum(4 * (g.n + 1) + 8 * g.m for g in graphs)
    budget = csr + 80 * T // 2 + (24 << 20)
    with n34.batch_decompose(graphs, mem_budget_bytes=budget) as dev, \
            n34.batch_decompose(graphs, mem_budget_bytes=budget, flags=n34.OPT_HOST_RESULTS) as host:
        assert host.result["chunks"] == dev.result["chunks"] >= 2
        for i in range(len(graphs)):
            kd, td = dev.copy_k(i, with_tris=True)
            kh, th = host.copy_k(i, with_tris=True)
            assert np.array_equal(kd, kh) and np.array_equal(td, th)
            assert np.array_equal(kh, single[i].k)
            assert host.summary(i) == dev.summary(i)


@pytest.mark.gpu
def test_batch_split_over_device_shares_equals_one_batch(n34):
    """The batched form over several device shares (nucleus34_split_plan,
    here two shares on GPU 0 running at once): every graph's summary, k and
    triangles equal the single batch's."""
    graphs = _mixed_graphs(n34, 32, 13)
    with n34.batch_decompose(graphs) as one, n34.batch_decompose_devices(graphs, [0, 0]) as two:
        assert sorted(two.result["share_graphs"]) == sorted(two.result["share_graphs"]) and \
            sum(two.result["share_graphs"]) == len(graphs) and min(two.result["share_graphs"]) > 0
        for i in range(len(graphs)):
            k1, t1 = one.copy_k(i, with_tris=True)
            k2, t2 = two.copy_k(i, with_tris=True)
            assert np.array_equal(k1, k2) and np.array_equal(t1, t2)
            assert one.summary(i) == two.summary(i)
