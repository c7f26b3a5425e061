#!/usr/bin/env python3
"""Runs the reference's own GPU programs (built for sm_100a -O3 from the
reference sources by `make -C oracle ref`) on a seeded graph and compares
them with libnucleus34 on the same GPU -- test infrastructure for the
comparison records, not product code.

Per run it prints one JSON line with:
  reference   the program's record (counts, K_max, K_avg, K[0..], phase times,
              total_time_sec) and its wall time;
  ours        the library on the same graph: device-timed t_total of a warm
              context (median of --ours-runs), counts and K fields;
  kfile       with --kfile: sha256 of both k files. The on-demand program
              writes canonical rows "(a,b,c)\\t<k>" (cuNucleus34_ondemand.cu:
              724-733), so the files must be byte-identical. The direct
              program writes its rows before its sort and its k after it
              (cuNucleus34.cu:412-428, 751-772), so it is compared as two
              multisets: the triangle rows, and the k values;
  equal       every comparison;
  clocks      nvidia-smi samples (SM MHz, throttle reasons) during each side;
  ratio       reference total_time_sec / our median t_total.

Both k files stream through FIFOs into sha256 (R-MAT scale 20 has 4.2e8
rows, ~13 GB of text), so nothing large touches the disk.

The reference's single-shot triangle phase stores length-2 path offsets in
32-bit EDGE_T (nucleus/utils.cuh:407-411, 543-547), which wraps once the path
count reaches 2^32 (R-MAT scale 20: 4.42e9). Its own planner switches to the
segmented pass, whose segments stay below that, when path_count * 16 B > 0.8 *
free memory (nucleus/cuNucleus34_ondemand.cu:428-434). With --free-gb G a
sidecar process holds device memory so that about G GB stay free, and the
reference takes its segmented path by its own rule. Scale 20 must be run with
--free-gb (80 works); the script refuses otherwise.

    python oracle/ref_gpu_timing.py --scale 12 --seed 1 --program ondemand --kfile
    python oracle/ref_gpu_timing.py --scale 18 --program ondemand --kfile
    python oracle/ref_gpu_timing.py --scale 20 --program ondemand --kfile --free-gb 80
    python oracle/ref_gpu_timing.py --graph rgg --n 4000000 --degree 48 --seed 3 --kdiff

With --kdiff (on-demand) the reference's k file is not hashed but reduced to
its k column by oracle/_build/kfile_column and compared with ours row by row:
the differing rows, their triangles and their highest edge ids are reported.
"""
import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
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
torch.cuda.synchronize()
print("holding", hold, "free_after", torch.cuda.mem_get_info()[0], flush=True)
time.sleep(3600)
"""

CLOCK_QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
               "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
               "clocks_event_reasons.sw_power_cap")


class Clocks:
    """nvidia-smi samples every 200 ms while a side runs."""

    def __init__(self):
        self.rows, self.proc = [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--id=0", f"--query-gpu={CLOCK_QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=lambda: self.rows.extend(
                [x.strip() for x in ln.split(",")] for ln in self.proc.stdout), daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        sm, mx, reasons = [], [], set()
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
                for nm, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                                 r[3:7]):
                    if v.lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


class FifoHash:
    """Reads a FIFO in a thread: sha256 of the whole stream, or (multiset
    mode) the rows kept in memory for a sorted comparison."""

    def __init__(self, path, keep_rows=False):
        self.path, self.keep_rows = path, keep_rows
        os.mkfifo(path)
        self.h, self.rows, self.bytes = hashlib.sha256(), [], 0
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        with open(self.path, "rb") as f:
            parts = []
            while True:
                chunk = f.read(1 << 22)
                if not chunk:
                    break
                self.bytes += len(chunk)
                self.h.update(chunk)
                if self.keep_rows:
                    parts.append(chunk)
            if self.keep_rows:
                self.rows = b"".join(parts).decode().splitlines()

    def finish(self, timeout=1800):
        # a writer that never opened the FIFO leaves the reader blocked in open():
        # open the write end once ourselves so that it sees end-of-file
        if self.t.is_alive():
            try:
                fd = os.open(self.path, os.O_WRONLY | os.O_NONBLOCK)
                os.close(fd)
            except OSError:
                pass
        self.t.join(timeout)
        return self.h.hexdigest()


def multiset_digest(rows):
    """(sha256 of the sorted triangle parts, sha256 of the sorted k values)."""
    tris, ks = [], []
    for r in rows:
        a, _, b = r.partition("\t")
        tris.append(a)
        ks.append(int(b))
    ks.sort()
    tris.sort()
    return (hashlib.sha256("\n".join(tris).encode()).hexdigest(),
            hashlib.sha256(",".join(map(str, ks)).encode()).hexdigest())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--graph", choices=["rmat", "rgg"], default="rmat")
    ap.add_argument("--scale", type=int, default=12)
    ap.add_argument("--n", type=int, default=4000000)
    ap.add_argument("--degree", type=float, default=48.0)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--program", choices=["ondemand", "direct"], default="ondemand")
    ap.add_argument("--kfile", action="store_true", help="compare the k files (sha256 or multisets)")
    ap.add_argument("--kdiff", action="store_true",
                    help="on-demand: also compare the k files row by row (the reference's k column through "
                         "oracle/_build/kfile_column) and report the differing rows and their edges")
    ap.add_argument("--ours-runs", type=int, default=3)
    ap.add_argument("--free-gb", type=float, default=0.0)
    ap.add_argument("--timeout", type=float, default=1200)
    a = ap.parse_args()
    import nucleus34 as n34
    exe = os.path.join(HERE, "_ref", "cuNucleus34_ondemand" if a.program == "ondemand" else "cuNucleus34")
    if not os.path.exists(exe):
        sys.exit(f"{exe} missing (make -C oracle ref)")
    if a.graph == "rmat" and a.scale >= 20 and a.free_gb <= 0:
        sys.exit("scale >= 20 needs --free-gb: the reference's single-shot path wraps its 32-bit path offsets")
    env = dict(os.environ)
    env.setdefault("CUDA_VISIBLE_DEVICES", "0")  # the reference enables peer access to every visible GPU
    if a.graph == "rmat":
        out = {"graph": f"R-MAT scale {a.scale} ef {a.edge_factor} seed {a.seed}"}
        s, d = n34.gen_rmat(a.scale, a.edge_factor, a.seed)
    else:
        out = {"graph": f"RGG n {a.n} degree {a.degree} seed {a.seed}"}
        s, d = n34.gen_rgg(a.n, a.degree, a.seed)
    out["program"] = os.path.basename(exe)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "graph.edges")
        n34.write_edges(s, d, path)
        del s, d
        g = n34.load_graph(path)  # the reader's semantics, first-line drop included
        out["vertices"], out["oriented_edges"] = int(g.n), int(g.m)
        # ---- reference ----
        side = None
        kcol_proc = None
        if a.kdiff:
            # the reference's k file goes through kfile_column (its k column to a file), not the hasher
            fifo = os.path.join(td, "ref.k")
            os.mkfifo(fifo)
            tool = os.path.join(HERE, "_build", "kfile_column")
            kcol_proc = subprocess.Popen([tool, fifo, os.path.join(td, "ref.k8")], stdout=subprocess.PIPE, text=True)
            ref_fifo = None
        else:
            ref_fifo = FifoHash(os.path.join(td, "ref.k"), keep_rows=a.program == "direct") if a.kfile else None
        try:
            if a.free_gb > 0:
                side = subprocess.Popen([sys.executable, "-c", SIDECAR, str(a.free_gb)], stdout=subprocess.PIPE,
                                        text=True, env=env)
                out["sidecar"] = side.stdout.readline().strip()
                out["mode"] = f"segmented listing forced: about {a.free_gb:g} GB left free by a sidecar"
            else:
                out["mode"] = "the reference's own choice with the whole GPU free"
            # cuNucleus34 <dataset> [parts] [out]; cuNucleus34_ondemand <dataset> [out]
            kpath = ref_fifo.path if ref_fifo else (os.path.join(td, "ref.k") if kcol_proc else None)
            cmd = [exe, path] + (["1"] if a.program == "direct" else []) + ([kpath] if kpath else [])
            with Clocks() as ck:
                t0 = time.time()
                r = subprocess.run(cmd, capture_output=True, text=True, timeout=a.timeout, env=env)
                out["reference_wall_s"] = time.time() - t0
            out["clocks_reference"] = ck.summary()
            out["returncode"] = r.returncode
            try:
                out["reference"] = json.loads(r.stdout)["dataset"]
            except Exception:
                out["stdout_tail"] = r.stdout[-2000:]
            out["stderr_tail"] = r.stderr[-1200:]
        except subprocess.TimeoutExpired:
            out["timeout_s"] = a.timeout
        finally:
            if side is not None:
                side.terminate()
                side.wait(timeout=60)
        ref_sha = ref_fifo.finish() if ref_fifo else None
        ref_k8 = None
        if kcol_proc is not None:
            if kcol_proc.poll() is None:  # the reference never opened its k file: unblock the reader
                try:
                    os.close(os.open(os.path.join(td, "ref.k"), os.O_WRONLY | os.O_NONBLOCK))
                except OSError:
                    pass
            kcol_proc.wait(timeout=600)
            import numpy as np
            ref_k8 = np.fromfile(os.path.join(td, "ref.k8"), dtype=np.uint8)
        # ---- ours ----
        with n34.Context() as ctx:
            ctx.upload(g)
            ctx.run(a.program)  # warm-up
            runs = []
            with Clocks() as ck:
                for _ in range(max(1, a.ours_runs)):
                    res = ctx.run(a.program)
                    runs.append(res)
            out["clocks_ours"] = ck.summary()
            if ref_k8 is not None:
                K, TR = ctx.copy_k(int(res["triangle_count"]), with_tris=True)
            else:
                K = ctx.copy_k(int(res["triangle_count"]))
        tt = [x["t_total"] for x in runs]
        res = runs[-1]
        ours = {"t_total_median": statistics.median(tt), "t_total_runs": tt,
                "phases_s": {k: res[k] for k in ("t_triangles", "t_incidence", "t_support", "t_cliques", "t_peel")},
                "triangle_count": int(res["triangle_count"]), "four_clique_count": int(res["four_clique_count"]),
                "K_max": int(res["k_max"]), "K_avg": float(res["k_avg"]), "peak_device_bytes":
                int(res["peak_device_bytes"])}
        out["ours"] = ours
        if ref_k8 is not None:
            import numpy as np
            ours_k = K.astype(np.int64)
            n_cmp = min(len(ref_k8), len(ours_k))
            diff = np.flatnonzero(ref_k8[:n_cmp].astype(np.int64) != ours_k[:n_cmp])
            dd = {"rows_reference": int(len(ref_k8)), "rows_ours": int(len(ours_k)), "rows_differing": int(len(diff))}
            if len(diff):
                top_edge = TR[diff].max(axis=1).astype(np.int64)
                m = int(g.m)
                dd["first"] = [{"row": int(i), "triangle": [int(x) for x in TR[i]], "k_reference": int(ref_k8[i]),
                                "k_ours": int(ours_k[i])} for i in diff[:12]]
                dd["oriented_edges"] = m
                dd["highest_edge_of_differing_rows"] = {"min": int(top_edge.min()), "max": int(top_edge.max()),
                                                        "within_last_1024_edges": int((top_edge >= m - 1024).sum())}
                dd["k_reference_minus_ours"] = {str(v): int(c) for v, c in zip(*np.unique(
                    ref_k8[diff].astype(np.int64) - ours_k[diff], return_counts=True))}
            out["kdiff"] = dd
        if a.kfile and ref_k8 is None:
            our_fifo = FifoHash(os.path.join(td, "ours.k"), keep_rows=a.program == "direct")
            try:
                n34.decompose(g, variant=a.program, n_quds=0, kfile=our_fifo.path)
            finally:
                our_sha = our_fifo.finish()
            if a.program == "ondemand":
                out["kfile"] = {"reference_sha256": ref_sha, "ours_sha256": our_sha,
                                "reference_bytes": ref_fifo.bytes, "ours_bytes": our_fifo.bytes}
            else:
                rt, rk = multiset_digest(ref_fifo.rows)
                ot, ok = multiset_digest(our_fifo.rows)
                out["kfile"] = {"reference_rows_sorted_sha256": rt, "ours_rows_sorted_sha256": ot,
                                "reference_k_sorted_sha256": rk, "ours_k_sorted_sha256": ok,
                                "rows": len(ref_fifo.rows)}
        rec = out.get("reference")
        if rec:
            kref = [int(x) for x in rec.get("K", [])]
            eq = {
                "triangle_count": int(rec.get("triangle_count", -1)) == ours["triangle_count"],
                "four_clique_count": int(rec.get("four_clique_count", -1)) == ours["four_clique_count"],
                "K_max": int(rec.get("K_max", -1)) == ours["K_max"],
                # the record prints K_avg with 6 significant digits
                "K_avg": float(f"{ours['K_avg']:.6g}") == float(rec.get("K_avg", -1)),
                "K_first": kref == [int(x) for x in K[: len(kref)]],
            }
            if "kfile" in out:
                kf = out["kfile"]
                if a.program == "ondemand":
                    eq["kfile_sha256"] = kf["reference_sha256"] == kf["ours_sha256"]
                else:
                    eq["kfile_rows_multiset"] = kf["reference_rows_sorted_sha256"] == kf["ours_rows_sorted_sha256"]
                    eq["kfile_k_multiset"] = kf["reference_k_sorted_sha256"] == kf["ours_k_sorted_sha256"]
            if "kdiff" in out:
                eq["kfile_rows"] = out["kdiff"]["rows_differing"] == 0 and \
                    out["kdiff"]["rows_reference"] == out["kdiff"]["rows_ours"]
            out["equal"] = eq
            out["all_equal"] = all(eq.values())
            if rec.get("total_time_sec"):
                out["ratio_total"] = float(rec["total_time_sec"]) / ours["t_total_median"]
    print(json.dumps(out), flush=True)
    return 0 if out.get("all_equal") else 1


if __name__ == "__main__":
    sys.exit(main())
