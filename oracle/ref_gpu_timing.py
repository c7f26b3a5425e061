#!/usr/bin/env python3
"""Times the reference's own GPU programs (built for sm_100a by
`make -C oracle ref`) on the seeded R-MAT workloads -- test infrastructure for
the comparison tables, not product code.

The reference's single-shot triangle phase stores length-2 path offsets in
32-bit EDGE_T (nucleus/utils.cuh:407-411, 543-547), which wraps once the path
count reaches 2^32 (R-MAT scale 20: 4.42e9). Its own planner switches to the
segmented pass, whose segments stay below that, when
path_count * 16 B > 0.8 * free memory (nucleus/cuNucleus34_ondemand.cu:428-434).
With --free-gb G a sidecar process holds device memory so that about G GB stay
free, and the reference takes its segmented path by its own rule.

    python oracle/ref_gpu_timing.py --scale 18 --program ondemand
    python oracle/ref_gpu_timing.py --scale 20 --program ondemand --free-gb 80
    python oracle/ref_gpu_timing.py --graph rgg --n 4000000 --degree 48 --seed 3

With --compare the same graph also goes through libnucleus34's one-shot call
and the record's counts, K_max, K_avg and first k values are compared.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "gpu-nucleus34_b200"))

SIDECAR = r"""
import sys, time, torch
free, total = torch.cuda.mem_get_info()
keep = int(float(sys.argv[1]) * 1e9)
hold = max(0, free - keep)
x = torch.empty(hold, dtype=torch.uint8, device="cuda") if hold else None
print("holding", hold, flush=True)
time.sleep(3600)
"""


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--graph", choices=["rmat", "rgg"], default="rmat")
    ap.add_argument("--scale", type=int, default=12)
    ap.add_argument("--n", type=int, default=4000000)
    ap.add_argument("--degree", type=float, default=48.0)
    ap.add_argument("--compare", action="store_true")
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--program", choices=["ondemand", "direct"], default="ondemand")
    ap.add_argument("--free-gb", type=float, default=0.0)
    ap.add_argument("--timeout", type=float, default=900)
    a = ap.parse_args()
    import nucleus34 as n34
    exe = os.path.join(HERE, "_ref", "cuNucleus34_ondemand" if a.program == "ondemand" else "cuNucleus34")
    if not os.path.exists(exe):
        sys.exit(f"{exe} missing (make -C oracle ref)")
    if a.graph == "rmat":
        out = {"graph": "rmat", "scale": a.scale, "edge_factor": a.edge_factor, "seed": a.seed}
    else:
        out = {"graph": "rgg", "n": a.n, "degree": a.degree, "seed": a.seed}
    out["program"] = os.path.basename(exe)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "graph.edges")
        if a.graph == "rmat":
            s, d = n34.gen_rmat(a.scale, a.edge_factor, a.seed)
        else:
            s, d = n34.gen_rgg(a.n, a.degree, a.seed)
        n34.write_edges(s, d, path)
        side = None
        try:
            if a.free_gb > 0:
                side = subprocess.Popen([sys.executable, "-c", SIDECAR, str(a.free_gb)], stdout=subprocess.PIPE,
                                        text=True)
                line = side.stdout.readline().strip()
                out["sidecar"] = line
            t0 = time.time()
            r = subprocess.run([exe, path], capture_output=True, text=True, timeout=a.timeout)
            out["wall_s"] = time.time() - t0
            out["returncode"] = r.returncode
            try:
                out["record"] = json.loads(r.stdout)["dataset"]
            except Exception:
                out["stdout_tail"] = r.stdout[-2000:]
            out["stderr_tail"] = r.stderr[-1500:]
        except subprocess.TimeoutExpired:
            out["timeout_s"] = a.timeout
        finally:
            if side is not None:
                side.terminate()
                side.wait(timeout=30)
        if a.compare and "record" in out:
            g = n34.load_graph(path)
            dec = n34.decompose(g, variant=a.program, n_quds=0)
            rec, res = out["record"], dec.result
            kref = [int(x) for x in rec.get("K", [])]
            ours = {"triangle_count": int(res["triangle_count"]), "four_clique_count": int(res["four_clique_count"]),
                    "K_max": int(res["k_max"]), "K_avg": float(res["k_avg"]), "t_total": float(res["t_total"]),
                    "K": [int(x) for x in dec.k[:len(kref)]]}
            out["ours"] = ours
            out["equal"] = {
                "triangle_count": int(rec.get("triangle_count", -1)) == ours["triangle_count"],
                "four_clique_count": int(rec.get("four_clique_count", -1)) == ours["four_clique_count"],
                "K_max": int(rec.get("K_max", -1)) == ours["K_max"],
                # the record prints K_avg with 6 significant digits
                "K_avg": float(f"{ours['K_avg']:.6g}") == float(rec.get("K_avg", -1)),
                "K_first": kref == ours["K"],
            }
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
