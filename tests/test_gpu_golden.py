"""The CUDA path against the golden fixtures themselves: the outputs of the
reference's own host code (tests/golden/make_golden.py runs
oracle/_ref/cpu_ref) on every golden input. Both variants, through the
C-ABI: counts, K_max, K_avg to the 6 significant digits the reference prints,
and the k file byte for byte (sha256)."""
import hashlib
import json
import os

import pytest

import golden_inputs

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
CASES = {c["name"]: c for c in GOLDEN["cases"]}


@pytest.mark.parametrize("variant", ["direct", "ondemand"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_cuda_path_matches_the_reference_outputs(n34, name, variant, tmp_path):
    case = CASES[name]
    path = golden_inputs.materialise(case, str(tmp_path))
    g = n34.load_graph(path)
    assert g.n == case["vertex_count"] and 2 * g.m == case["edge_count"]
    kfile = str(tmp_path / "k.txt")
    d = n34.decompose(g, variant=variant, n_quds=0, kfile=kfile)
    r = d.result
    assert r["triangle_count"] == case["triangle_count"]
    assert r["four_clique_count"] == case["four_clique_count"]
    if case["four_clique_count"]:
        assert r["k_max"] == case["K_max"]
        assert float(f"{r['k_avg']:.6g}") == case["K_avg_6sig"]
    data = open(kfile, "rb").read()
    assert hashlib.sha256(data).hexdigest() == case["kfile_sha256"]
    if "kfile" in case:
        assert data.decode() == case["kfile"]
