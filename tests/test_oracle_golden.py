"""The CPU oracle against the golden fixtures produced by the reference's own
host code (tests/golden/make_golden.py runs oracle/_ref/cpu_ref).

Bit-exact: counts, K_max, the k file (sha256), and K_avg to the 6 significant
digits the reference prints."""
import hashlib
import json
import os

import numpy as np
import pytest

import golden_inputs

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
CASES = {c["name"]: c for c in GOLDEN["cases"]}


def _sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_cpu(name, oracle, n34, tmp_path):
    case = CASES[name]
    if case["triangle_count"] > 3_000_000 and os.environ.get("N34_FAST_CPU_TESTS"):
        pytest.skip("large case skipped by N34_FAST_CPU_TESTS")
    path = golden_inputs.materialise(case, str(tmp_path))
    assert _sha(path) == case["input_sha256"], "generator output changed"
    g = oracle.read_graph(path)
    assert g.n == case["vertex_count"]
    assert 2 * g.m == case["edge_count"]
    r = oracle.decompose(g)
    assert r.T == case["triangle_count"]
    assert r.Q == case["four_clique_count"]
    assert (r.k_max if r.T else 0) == case["K_max"]
    assert float(f"{r.k_avg:.6g}") == pytest.approx(case["K_avg_6sig"], rel=0, abs=0)
    kb = oracle.kfile_bytes(r.tris, r.k)
    assert hashlib.sha256(kb).hexdigest() == case["kfile_sha256"]
    if "kfile" in case:
        assert kb.decode() == case["kfile"]


@pytest.mark.parametrize("name", sorted(CASES))
def test_library_reader_matches_oracle_reader(name, oracle, n34, tmp_path):
    """The product reader (parallel, libnucleus34) builds the same oriented CSR
    as the oracle's restatement of from_edges + make_oriented."""
    case = CASES[name]
    path = golden_inputs.materialise(case, str(tmp_path))
    a = n34.load_graph(path)
    b = oracle.read_graph(path)
    assert (a.n, a.m) == (b.n, b.m)
    assert np.array_equal(a.O, b.O)
    assert np.array_equal(a.D, b.D)
    assert np.array_equal(a.E, b.E)
