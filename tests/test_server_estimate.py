"""The serving loop's admission estimates and variant routing
(nucleus34_server_estimate, the same host function nucleus34_server_submit
uses), on the CPU: the byte formulas against a numpy restatement, the
routing threshold at its exact edge, the 32-bit clique-id bound, and the
request flags."""
import numpy as np
import pytest

from test_batch import _mixed_graphs

# the admission constants of the serving loop: bytes per oriented edge, per
# out-wedge (triangle bound) and, for the direct variant, per out-triple
EDGE, WEDGE, TRIPLE = 40, 80, 33


def _numpy_estimate(g):
    D = g.D[: g.n].astype(np.int64)
    w = int((D * (D - 1) // 2).sum())
    t3 = int((D * (D - 1) * (D - 2) // 6).sum())
    on = EDGE * g.m + WEDGE * w
    return on, on + TRIPLE * t3, w, t3


def test_estimates_match_the_formulas(n34):
    for g in _mixed_graphs(n34, 12, 3):
        on, direct, w, t3 = _numpy_estimate(g)
        e = n34.server_estimate(g, budget=1 << 40)
        assert (e["ondemand_bytes"], e["direct_bytes"], e["triangle_bound"], e["clique_bound"]) == (on, direct, w, t3)


def test_routing_threshold_is_budget_over_direct_div(n34):
    s, t = n34.gen_rmat(10, 16, 4)
    g = n34.graph_from_edges(s, t)
    _, direct, _, _ = _numpy_estimate(g)
    for div in (1, 8, 64):
        # the direct estimate exactly at budget / div goes direct, one byte over does not
        assert n34.server_estimate(g, budget=direct * div, direct_div=div)["direct"]
        assert not n34.server_estimate(g, budget=(direct - 1) * div, direct_div=div)["direct"]
    # direct_div 0 is the default share, 1/64
    assert n34.server_estimate(g, budget=direct * 64)["direct"]
    assert not n34.server_estimate(g, budget=direct * 64 - 64)["direct"]


def test_route_and_request_flags(n34):
    s, t = n34.gen_rmat(9, 8, 2)
    g = n34.graph_from_edges(s, t)
    big = 1 << 50
    assert n34.server_estimate(g, big, route=n34.ROUTE_MEMORY)["direct"]
    assert not n34.server_estimate(g, big, route=n34.ROUTE_ONDEMAND)["direct"]
    # a request for its clique list is direct whatever the route and budget
    assert n34.server_estimate(g, 0, route=n34.ROUTE_ONDEMAND, cliques=True)["direct"]
    assert n34.server_estimate(g, 0, cliques=True)["direct"]
    # the triangle-list flag does not change the variant
    assert not n34.server_estimate(g, 0, triangles=True)["direct"]


def test_clique_bound_beyond_32_bits_stays_on_demand(n34):
    # one source with 3000 out-neighbours: C(3000, 3) = 4.49e9 out-triples,
    # more clique ids than the direct variant's 32 bits hold
    d = 3000
    O = np.zeros(d + 2, np.uint32)
    O[1:] = d
    D = np.zeros(d + 1, np.uint32)
    D[0] = d
    E = np.arange(1, d + 1, dtype=np.uint32)
    g = n34.HostGraph(n=d + 1, m=d, O=O, D=D, E=E)
    e = n34.server_estimate(g, budget=1 << 62, direct_div=1)
    assert e["clique_bound"] == d * (d - 1) * (d - 2) // 6 > 2 ** 32
    assert not e["direct"]
    assert n34.server_estimate(g, budget=0, cliques=True)["direct"]


def test_invalid_inputs_are_rejected(n34):
    s, t = n34.gen_rmat(8, 8, 1)
    g = n34.graph_from_edges(s, t)
    with pytest.raises(n34.Nucleus34Error) as ei:
        n34.server_estimate(g, 1 << 30, route=7)
    assert ei.value.code == n34.E_INVALID
    bad = n34.HostGraph(n=g.n, m=g.m + 1, O=g.O, D=g.D, E=g.E)
    with pytest.raises(n34.Nucleus34Error) as ei:
        n34.server_estimate(bad, 1 << 30)
    assert ei.value.code == n34.E_INVALID
