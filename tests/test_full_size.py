"""Full-size checks through size-independent properties (the CPU oracle's
bucket peel cannot hold these graphs: it materialises every four-clique).

- The certificate (nucleus34_ctx_verify): per triangle, at least k cliques
  among triangles with k' >= k and at most k cliques alive when its round
  began, one non-decreasing level per round. These hold exactly for the
  (3,4)-nucleus numbers, so zero violations proves every k.
- The four-clique total against an independent CPU count by oriented
  neighbourhoods (oracle.count_k4), for the random geometric graph.

Workloads: R-MAT scale 20 ef 16 seed 2 (the benchmark graph) and the 2D random
geometric graph with 4M points, expected degree 48, seed 3."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _certify(n34, g, variant="ondemand", flags=0):
    with n34.Context(flags=n34.OPT_VERIFIABLE | flags) as ctx:
        ctx.upload(g)
        r = ctx.run(variant)
        viol, checked = ctx.verify()
    return r, viol, checked


@pytest.mark.parametrize("case", [("rmat", 12, 16, 1), ("rgg", 20000, 40, 8), ("ws", 3000, 10, 5)])
@pytest.mark.parametrize("variant", ["ondemand", "direct"])
def test_certificate_on_small_graphs(n34, oracle, case, variant):
    if case[0] == "rmat":
        s, t = n34.gen_rmat(case[1], case[2], case[3])
    elif case[0] == "rgg":
        s, t = n34.gen_rgg(case[1], case[2], case[3])
    else:
        s, t = n34.gen_ws(case[1], case[2], 0.1, case[3])
    g = n34.graph_from_edges(s, t)
    r, viol, checked = _certify(n34, g, variant)
    assert viol == 0 and checked == r["triangle_count"]
    assert r["four_clique_count"] == oracle.count_k4(g)


def test_certificate_stamp_path(n34):
    s, t = n34.gen_rmat(14, 16, 3)
    g = n34.graph_from_edges(s, t)
    r, viol, checked = _certify(n34, g, "ondemand", n34.OPT_STAMP_PEEL)
    assert viol == 0 and checked == r["triangle_count"] > 0


def test_rmat20_benchmark_graph_certified(n34):
    s, t = n34.gen_rmat(20, 16, 2)
    g = n34.graph_from_edges(s, t)
    r, viol, checked = _certify(n34, g)
    # counts and K_max of the reference's own cuNucleus34_ondemand on this graph
    assert r["triangle_count"] == 424141894
    assert r["four_clique_count"] == 17099682515
    assert r["k_max"] == 196
    assert viol == 0 and checked == r["triangle_count"]


def test_rgg4m_certified_and_cliques_counted_independently(n34, oracle):
    s, t = n34.gen_rgg(4000000, 48.0, 3)
    g = n34.graph_from_edges(s, t)
    r, viol, checked = _certify(n34, g)
    assert r["triangle_count"] == 898658078
    assert r["k_max"] == 35
    assert viol == 0 and checked == r["triangle_count"]
    assert r["four_clique_count"] == oracle.count_k4(g)


def test_rgg4m_under_a_40gb_budget_matches_the_uncapped_run(n34):
    """The on-demand config with device memory capped at 40 GB: the library
    switches to its memory-lean layout (entries sorted in place, bitmap
    frontiers, k kept in the support array) and must give the uncapped run's
    results bit for bit, within the cap."""
    s, t = n34.gen_rgg(4000000, 48.0, 3)
    g = n34.graph_from_edges(s, t)
    with n34.Context() as ctx:
        ctx.upload(g)
        free = ctx.run("ondemand")
        k_free = ctx.copy_k(int(free["triangle_count"]))
    budget = 40 * 10**9
    with n34.Context(mem_budget_bytes=budget) as ctx:
        ctx.upload(g)
        lean = ctx.run("ondemand")
        k_lean = ctx.copy_k(int(lean["triangle_count"]))
    assert lean["peak_device_bytes"] <= budget < free["peak_device_bytes"]
    for key in ("triangle_count", "four_clique_count", "k_max", "k_avg"):
        assert lean[key] == free[key], key
    assert np.array_equal(k_lean, k_free)
