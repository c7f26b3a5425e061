"""Generates the golden fixtures that pin the CPU oracle (test infrastructure).

Runs the REFERENCE's own host implementation (oracle/_ref/cpu_ref, built from
the reference sources by `make -C oracle ref`) on seeded synthetic graphs and
on small hand-written files that exercise the reader's quirks, and records
its outputs in tests/golden/golden.json: counts, K_max, K_avg and the sha256
of the per-triangle k file "(a,b,c)\\t<k>" in canonical order. Inputs are
regenerated by the tests from the recorded parameters (their sha256 is
recorded too), so no graph file is committed.

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "gpu-nucleus34_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import nucleus34  # noqa: E402
import golden_inputs  # noqa: E402

CPU_REF = os.path.join(ROOT, "oracle", "_ref", "cpu_ref")


def sha(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for b in iter(lambda: f.read(1 << 20), b""):
            h.update(b)
    return h.hexdigest()


def main():
    if not os.path.exists(CPU_REF):
        sys.exit("build the reference first: make -C oracle ref")
    out = {"generator": "tests/golden/make_golden.py", "reference": "oracle/_ref/cpu_ref", "cases": []}
    with tempfile.TemporaryDirectory() as td:
        for case in golden_inputs.CASES:
            path = golden_inputs.materialise(case, td)
            kfile = os.path.join(td, case["name"] + ".k")
            r = subprocess.run([CPU_REF, path, kfile], check=True, capture_output=True, text=True)
            rec = json.loads(r.stdout.strip().splitlines()[-1])
            entry = dict(case)
            entry.update({
                "input_sha256": sha(path),
                "vertex_count": rec["vertex_count"],
                "edge_count": rec["edge_count"],
                "triangle_count": rec["triangle_count"],
                "four_clique_count": rec["four_clique_count"],
                "K_max": rec["K_max"],
                "K_avg_6sig": rec["K_avg"],
                "kfile_sha256": sha(kfile),
            })
            if rec["triangle_count"] <= 64:
                entry["kfile"] = open(kfile).read()
            out["cases"].append(entry)
            print(case["name"], rec["triangle_count"], rec["four_clique_count"], rec["K_max"], flush=True)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
