"""The oriented CSR built on the device from an edge list
(nucleus34_ctx_upload_edges) against the host build of the same list
(nucleus34_graph_from_edges): the same n, m, O, D and E, and the same
decomposition. Inputs cover self-loops, duplicates, reversed duplicates,
isolated ids, hubs with long lists (the segmented sort's three size classes),
an empty list and lists of self-loops only."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def edge_cases(n34):
    rng = np.random.default_rng(7)
    s = rng.integers(0, 3000, 40000).astype(np.uint32)
    d = np.where(rng.random(40000) < 0.05, s, rng.integers(0, 3000, 40000)).astype(np.uint32)
    hub_s = np.zeros(20000, np.uint32)  # one list past the block sort's 8192 entries
    hub_d = rng.integers(1, 30000, 20000).astype(np.uint32)
    return {
        "rmat14": n34.gen_rmat(14, 16, 3),
        "rgg50k": n34.gen_rgg(50000, 24.0, 2),
        "ws4000": n34.gen_ws(4000, 10, 0.1, 9),
        "random_loops_dups": (np.concatenate([s, d[:5000]]), np.concatenate([d, s[:5000]])),
        "hub": (np.concatenate([hub_s, hub_d[:100]]), np.concatenate([hub_d, hub_d[100:200]])),
        "empty": (np.zeros(0, np.uint32), np.zeros(0, np.uint32)),
        "loops_only": (np.arange(10, dtype=np.uint32), np.arange(10, dtype=np.uint32)),
        "single": (np.array([5], np.uint32), np.array([2], np.uint32)),
    }


def test_device_build_equals_host_build(n34):
    for name, (s, d) in edge_cases(n34).items():
        want = n34.graph_from_edges(s, d)
        with n34.Context() as ctx:
            n, m = ctx.upload_edges(s, d)
            got = ctx.copy_csr()
        assert (n, m) == (want.n, want.m), name
        assert np.array_equal(got.O, want.O[: want.n + 1]), name
        assert np.array_equal(got.D, want.D), name
        assert np.array_equal(got.E, want.E), name


def test_decomposition_from_the_device_build(n34):
    s, d = n34.gen_rmat(12, 16, 1)
    g = n34.graph_from_edges(s, d)
    with n34.Context() as a, n34.Context() as b:
        a.upload(g)
        ra = a.run("ondemand")
        b.upload_edges(s, d)
        rb = b.run("ondemand")
        assert ra["triangle_count"] == rb["triangle_count"]
        assert ra["four_clique_count"] == rb["four_clique_count"]
        ka, ta = a.copy_k(ra["triangle_count"], with_tris=True)
        kb, tb = b.copy_k(rb["triangle_count"], with_tris=True)
    assert np.array_equal(ta, tb) and np.array_equal(ka, kb)
