"""The drop-in programs bin/cuNucleus34 and bin/cuNucleus34_ondemand: argv,
exit codes, the JSON record and the k file, as the reference mains behave
(nucleus/cuNucleus34.cu:144-839, nucleus/cuNucleus34_ondemand.cu:308-784):
usage on stderr and EXIT_FAILURE without a dataset; exit 0 with "errorstep"
and "error" (the exception text) in the record on a handled error."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "gpu-nucleus34_b200", "bin")
PROGRAMS = ["cuNucleus34", "cuNucleus34_ondemand"]

# K4 on {1,2,3,4} plus the unused vertex 0; the first non-comment line is the
# header that an edge-list reader consumes (graph.hpp:307-359)
K4_TEXT = "% comment\n1 2\n1 2\n2 3\n1 3\n3 4\n1 4\n2 4\n"


# dataset keys of a complete record, in the reference's order
# (cuNucleus34.cu:229-795, cuNucleus34_ondemand.cu field calls)
KEYS = {
    "cuNucleus34": ["file", "vertex_count", "edge_count", "data_loading_time_sec", "data_memory_bytes",
                    "triangle_time_sec", "triangle_count", "triangles", "triangle_graph_time_sec",
                    "four_clique_time_sec", "four_clique_count", "four-cliques", "four_clique_graph_time_sec",
                    "peeling_mode", "peeling_preprocess_time_sec", "peeling_time_sec", "peeling_iterations",
                    "K_max", "total_time_sec", "K_count", "K", "K_avg"],
    "cuNucleus34_ondemand": ["file", "vertex_count", "edge_count", "data_loading_time_sec", "triangle_time_sec",
                             "triangle_count", "incidence_time_sec", "incidence_entries", "four_clique_time_sec",
                             "four_clique_count", "unpeeled_count", "peeling_mode", "peeling_time_sec",
                             "peeling_iterations", "K_max", "total_time_sec", "K_count", "K", "K_avg"],
}


def run(prog, *args):
    r = subprocess.run([os.path.join(BIN, prog), *map(str, args)], capture_output=True, text=True, timeout=300)
    return r.returncode, r.stdout, r.stderr


def record(stdout):
    return json.loads(stdout)


@pytest.mark.parametrize("prog", PROGRAMS)
def test_usage_without_a_dataset(prog):
    rc, out, err = run(prog)
    assert rc == 1 and out == ""
    assert err.startswith(f"Usage: {prog} <dataset file (.mtx or .grh)>")
    assert ("[parts" in err) == (prog == "cuNucleus34")
    assert err.rstrip().endswith("[results output file (optional)]")


@pytest.mark.parametrize("prog", PROGRAMS)
@pytest.mark.parametrize("name,text,error", [
    ("absent.edges", None, "Dataset {path} is not accessible!"),
    ("graph.foo", "1 2\n2 3\n", "Unknown dataset format: .foo"),
    ("graph.mtx", "%%MatrixMarket matrix coordinate pattern general\nnot a header\n1 2\n",
     "Wrong header for mtx format!"),
])
def test_handled_errors_go_into_the_record(prog, tmp_path, name, text, error):
    path = tmp_path / name
    if text is not None:
        path.write_text(text)
    rc, out, err = run(prog, path)
    assert rc == 0
    rec = record(out)
    assert rec["environment"]["app"].startswith("b200-nucleus34-")
    ds = rec["dataset"]
    assert ds["file"] == name
    assert ds["errorstep"] == "0.2 Data loading and graph construction"
    assert ds["error"] == error.format(path=path)
    assert f"Error: {ds['error']}" in err


@pytest.mark.parametrize("prog", PROGRAMS)
def test_record_holds_the_reader_counts(prog, tmp_path):
    path = tmp_path / "k4.edges"
    path.write_text(K4_TEXT)
    rc, out, err = run(prog, path)
    assert rc == 0
    ds = record(out)["dataset"]
    assert ds["vertex_count"] == 5 and ds["edge_count"] == 12
    # the reference's memory milestone line after the load (cuNucleus34.cu:272-279)
    assert "[mem] graph vertices=5 oriented_edges=6 " in err and "| gpu_free=" in err
    if "error" in ds:  # no device here: the device step fails after the load
        assert ds["errorstep"].startswith("1.1 ")
    else:
        assert ds["triangle_count"] == 4 and ds["four_clique_count"] == 1


@pytest.mark.gpu
@pytest.mark.parametrize("prog", PROGRAMS)
def test_records_and_k_files_match_the_oracle(n34, oracle, prog, tmp_path):
    s, t = n34.gen_rmat(9, 8, 3)
    path = tmp_path / "rmat9.edges"
    n34.write_edges(s, t, str(path))
    g = n34.load_graph(str(path))
    want = oracle.decompose(g, quds_cap=0)
    kfile = tmp_path / "k.txt"
    args = [path, 1, kfile] if prog == "cuNucleus34" else [path, kfile]
    rc, out, err = run(prog, *args)
    assert rc == 0, err
    ds = record(out)["dataset"]
    assert "error" not in ds, ds.get("error")
    assert list(ds) == KEYS[prog]
    assert ds["vertex_count"] == g.n and ds["edge_count"] == 2 * g.m
    assert ds["triangle_count"] == want.T and ds["four_clique_count"] == want.Q
    assert ds["K_max"] == want.k_max and ds["K_count"] == want.T
    assert ds["K"] == [int(x) for x in want.k[:5]]
    # printed with the stream's default six significant digits, as the reference does
    assert abs(ds["K_avg"] - want.k_avg) <= 1e-5 * max(1.0, abs(want.k_avg))
    rows = kfile.read_text().splitlines()
    assert rows == [f"({a},{b},{c})\t{k}" for (a, b, c), k in zip(want.tris.tolist(), want.k.tolist())]
    if prog == "cuNucleus34":
        assert len(ds["triangles"]) == min(5, want.T)
        assert ds["triangles"][0] == "({},{},{})".format(*want.tris[0].tolist())
