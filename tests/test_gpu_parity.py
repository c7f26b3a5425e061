"""Parity of the CUDA path (through the C-ABI) with the CPU oracle.

Bit-exact: triangle list (canonical (a,b) order), triangle count, four-clique
count, every triangle's k, K_max and K_avg, for both variants."""
import numpy as np
import pytest

import graphs

pytestmark = pytest.mark.gpu

VARIANTS = ["direct", "ondemand"]


def check_against_oracle(n34, oracle, g, variant):
    d = n34.decompose(g, variant=variant, n_quds=5)
    o = oracle.decompose(g, quds_cap=5)
    r = d.result
    assert r["triangle_count"] == o.T
    assert r["four_clique_count"] == o.Q
    assert d.tris.shape == o.tris.shape
    assert np.array_equal(d.tris, o.tris), "canonical triangle list differs"
    assert np.array_equal(d.k, o.k), "per-triangle k differs"
    if o.Q:
        assert r["k_max"] == o.k_max
        assert r["k_avg"] == o.k_avg
        assert r["unpeeled_count"] == 0
    if variant == "direct" and o.Q:
        assert np.array_equal(d.quds, o.quds[: len(d.quds)])
    return d, o


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("name", sorted(graphs.SMALL))
def test_small_known_graphs(n34, oracle, name, variant):
    s, t = graphs.SMALL[name]()
    g = n34.graph_from_edges(s, t)
    d, o = check_against_oracle(n34, oracle, g, variant)
    if name.startswith("K") and "_" not in name:
        n = int(name[1:])
        assert d.result["four_clique_count"] == n * (n - 1) * (n - 2) * (n - 3) // 24
        assert np.all(d.k == n - 3)


@pytest.mark.parametrize("variant", VARIANTS)
def test_c1_rmat12(n34, oracle, variant):
    """R-MAT scale 12, edge factor 16, seed 1 (the plain small configuration)."""
    s, t = n34.gen_rmat(12, 16, 1)
    g = n34.graph_from_edges(s, t)
    d, o = check_against_oracle(n34, oracle, g, variant)
    assert o.T > 400_000 and o.Q > 3_000_000


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("case", [("rmat", 10, 8, 7), ("rmat", 13, 24, 99), ("ws", 5000, 10, 3),
                                  ("rgg", 30000, 32, 5)])
def test_random_graphs(n34, oracle, variant, case):
    kind = case[0]
    if kind == "rmat":
        s, t = n34.gen_rmat(case[1], case[2], case[3])
    elif kind == "ws":
        s, t = n34.gen_ws(case[1], case[2], 0.1, case[3])
    else:
        s, t = n34.gen_rgg(case[1], case[2], case[3])
    g = n34.graph_from_edges(s, t)
    check_against_oracle(n34, oracle, g, variant)


@pytest.mark.parametrize("variant", VARIANTS)
def test_no_triangles_and_empty(n34, oracle, variant):
    for s, t in [graphs.triangle_free(), (np.array([0], np.uint32), np.array([1], np.uint32))]:
        g = n34.graph_from_edges(s, t)
        d = n34.decompose(g, variant=variant)
        assert d.result["triangle_count"] == 0
        assert d.result["four_clique_count"] == 0
        assert len(d.k) == 0


def test_context_reuse_is_deterministic(n34):
    s, t = n34.gen_rmat(11, 16, 5)
    g = n34.graph_from_edges(s, t)
    with n34.Context() as ctx:
        ctx.upload(g)
        outs = []
        for v in ["ondemand", "direct", "ondemand"]:
            r = ctx.run(v)
            k, tris = ctx.copy_k(r["triangle_count"], with_tris=True)
            outs.append((r["four_clique_count"], k, tris))
    for q, k, tris in outs[1:]:
        assert q == outs[0][0]
        assert np.array_equal(k, outs[0][1])
        assert np.array_equal(tris, outs[0][2])


def test_budget_exceeded_is_reported(n34):
    s, t = n34.gen_rmat(12, 16, 1)
    g = n34.graph_from_edges(s, t)
    with pytest.raises(n34.Nucleus34Error) as ei:
        n34.decompose(g, variant="direct", mem_budget_bytes=1 << 20)
    assert ei.value.code == n34.E_OOM_BUDGET


@pytest.mark.parametrize("case", [("rmat", 12, 16, 1), ("rgg", 20000, 40, 8)])
def test_stamp_peel_path_matches(n34, oracle, case):
    """The round-stamp ownership test (used when T >= 2^30) gives the same k."""
    if case[0] == "rmat":
        s, t = n34.gen_rmat(case[1], case[2], case[3])
    else:
        s, t = n34.gen_rgg(case[1], case[2], case[3])
    g = n34.graph_from_edges(s, t)
    d = n34.decompose(g, variant="ondemand", flags=n34.OPT_STAMP_PEEL)
    o = oracle.decompose(g)
    assert np.array_equal(d.k, o.k)
    assert d.result["four_clique_count"] == o.Q


@pytest.mark.parametrize("case", [("rmat", 13, 16, 3), ("rgg", 30000, 40, 9)])
def test_lean_and_profiled_peels_match(n34, oracle, case):
    """In the memory-lean layout (entries sorted in place, entries searched,
    bitmap frontiers, k kept in the support array) and with the per-step
    profiling launches, k is the same."""
    if case[0] == "rmat":
        s, t = n34.gen_rmat(case[1], case[2], case[3])
    else:
        s, t = n34.gen_rgg(case[1], case[2], case[3])
    g = n34.graph_from_edges(s, t)
    o = oracle.decompose(g)
    lean = n34.decompose(g, variant="ondemand", flags=n34.OPT_LEAN_MEMORY)
    assert np.array_equal(lean.k, o.k)
    prof = n34.decompose(g, variant="ondemand", flags=n34.OPT_PROFILE_PEEL)
    assert np.array_equal(prof.k, o.k)
    assert prof.result["t_peel_debit"] > 0


@pytest.mark.parametrize("variant,flags", [("direct", 0x0), ("ondemand", 0x0), ("ondemand", 0x4), ("ondemand", 0x1)])
def test_device_loop_and_host_loop_agree(n34, oracle, variant, flags):
    """The default device loop (one CUDA graph whose while node repeats the
    rounds) and the host-driven replay loop give the oracle's k, in the
    regular, memory-lean and round-stamp peels (the layout flags concern the
    on-demand peel only)."""
    s, t = n34.gen_rmat(12, 16, 4)
    g = n34.graph_from_edges(s, t)
    o = oracle.decompose(g)
    dev = n34.decompose(g, variant=variant, flags=flags)
    host = n34.decompose(g, variant=variant, flags=flags | n34.OPT_HOST_LOOP)
    assert np.array_equal(dev.k, o.k) and np.array_equal(host.k, o.k)
    assert dev.result["peeling_iterations"] == host.result["peeling_iterations"]


def test_listing_chunks_match_one_pass(n34, oracle):
    """With the listing's bit words capped (NUCLEUS34_LIST_CHUNK_WORDS, read
    per call) it counts every chunk of sources first and repeats each chunk's
    bits before its writes; the canonical list is the same, for chunks of
    many sources and for chunks of one."""
    import subprocess
    import sys
    code = ("import sys, json, hashlib; sys.path.insert(0, sys.argv[1]); import nucleus34 as n34\n"
            "s, t = n34.gen_rmat(13, 16, 6); g = n34.graph_from_edges(s, t)\n"
            "d = n34.decompose(g, variant='ondemand', n_quds=0)\n"
            "print(json.dumps([hashlib.sha256(d.tris.tobytes()).hexdigest(), "
            "hashlib.sha256(d.k.tobytes()).hexdigest()]))\n")
    s, t = n34.gen_rmat(13, 16, 6)
    o = oracle.decompose(n34.graph_from_edges(s, t))
    import hashlib
    import json
    import os
    want = [hashlib.sha256(o.tris.astype(np.uint32).tobytes()).hexdigest(),
            hashlib.sha256(o.k.astype(np.int32).tobytes()).hexdigest()]
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gpu-nucleus34_b200")
    for cap in ("4096", "1"):
        env = dict(os.environ, NUCLEUS34_LIST_CHUNK_WORDS=cap)
        r = subprocess.run([sys.executable, "-c", code, pkg], capture_output=True, text=True, timeout=300, env=env)
        assert r.returncode == 0, r.stderr[-2000:]
        assert json.loads(r.stdout.strip().splitlines()[-1]) == want, cap


@pytest.mark.parametrize("case", [("rmat", 14, 16, 2), ("rgg", 40000, 48, 6)])
def test_frontier_ordered_by_c_edge_matches(n34, oracle, case):
    """Large frontiers put in the order of their c-edge entries (instead of
    triangle ids) give the oracle's k; the peel's schedule changes, not its
    result."""
    if case[0] == "rmat":
        s, t = n34.gen_rmat(case[1], case[2], case[3])
    else:
        s, t = n34.gen_rgg(case[1], case[2], case[3])
    g = n34.graph_from_edges(s, t)
    o = oracle.decompose(g)
    d = n34.decompose(g, variant="ondemand", flags=n34.OPT_FRONTIER_BY_C, n_quds=0)
    assert np.array_equal(d.k, o.k)
    # with the sort forced onto every frontier of at least 4096 triangles
    with n34.Context(flags=n34.OPT_FRONTIER_BY_C) as ctx:
        ctx.set_tune({"sort_shift": 31})
        ctx.upload(g)
        r = ctx.run("ondemand")
        assert np.array_equal(ctx.copy_k(r["triangle_count"]), o.k)


@pytest.mark.parametrize("case", [("rmat", 13, 16, 3), ("rgg", 30000, 40, 9)])
def test_chunked_debit_schedule_matches(n34, oracle, case):
    """The default two-kernel debit schedule (a thread per short-list
    triangle, a warp per long one) and the chunked one give the oracle's k."""
    if case[0] == "rmat":
        s, t = n34.gen_rmat(case[1], case[2], case[3])
    else:
        s, t = n34.gen_rgg(case[1], case[2], case[3])
    g = n34.graph_from_edges(s, t)
    o = oracle.decompose(g)
    for fl in (0, n34.OPT_CHUNKED_DEBIT, n34.OPT_CHUNKED_DEBIT | n34.OPT_NO_SMALL_ROUNDS):
        d = n34.decompose(g, variant="ondemand", flags=fl, n_quds=0)
        assert np.array_equal(d.k, o.k), fl


@pytest.mark.parametrize("case", [("rmat", 13, 16, 3), ("rgg", 30000, 40, 9)])
def test_scan_and_pipeline_options_match(n34, oracle, case):
    """The level-change scans (vectorised or one word per thread) and the warp
    debit (static stride, software-pipelined, or claimed from a cursor) give the
    oracle's k, with list frontiers and with the bitmap frontiers of the lean
    layout."""
    if case[0] == "rmat":
        s, t = n34.gen_rmat(case[1], case[2], case[3])
    else:
        s, t = n34.gen_rgg(case[1], case[2], case[3])
    g = n34.graph_from_edges(s, t)
    o = oracle.decompose(g)
    for fl in (
        n34.OPT_SCALAR_SCANS,
        n34.OPT_PIPELINED_DEBIT,
        n34.OPT_PIPELINED_DEBIT | n34.OPT_NO_SMALL_ROUNDS,
        n34.OPT_DEBIT_CURSOR,
        n34.OPT_DEBIT_CURSOR | n34.OPT_NO_SMALL_ROUNDS,
        n34.OPT_DEBIT_CURSOR | n34.OPT_LEAN_MEMORY,
        n34.OPT_LEAN_MEMORY,
        n34.OPT_LEAN_MEMORY | n34.OPT_SCALAR_SCANS,
        n34.OPT_NO_SMALL_ROUNDS | n34.OPT_SCALAR_SCANS,
    ):
        d = n34.decompose(g, variant="ondemand", flags=fl, n_quds=0)
        assert np.array_equal(d.k, o.k), fl
