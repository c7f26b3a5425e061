#!/usr/bin/env python3
"""Benchmark of the (3,4)-nucleus decomposition hot path.

One step = one full decomposition (triangle listing, edge->triangle
incidence, four-clique support, device-resident peel) of the workload graph,
through libnucleus34's C-ABI.

  value  triangles peeled per second with the oriented CSR already resident in
         HBM (nucleus34_ctx_run; device time from CUDA events on the library
         stream), whole job over all ranks.
  e2e    the same metric through the one-shot drop-in call
         (nucleus34_decompose_ondemand / nucleus34_decompose) with the CSR in
         pinned host memory: H2D of the CSR and D2H of every triangle's k are
         inside the timed region.

Default workload: R-MAT scale 20, edge factor 16, (a,b,c,d) =
(.57,.19,.19,.05), seed 2 (~15.7M undirected edges), on-demand variant: its
four-clique count (~1.7e10) cannot be materialised as the direct variant's
clique list on one GPU, so the on-demand variant carries the at-scale number.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

With --impl reference the reference's own CPU implementation of the path
(oracle/_ref/cpu_ref, built from the reference sources; else the oracle port)
is timed on the host cores on a bounded sample of the workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-nucleus34_b200"))

METRIC = "triangles peeled/sec"
UNIT = "triangles/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--scale", type=int, default=20)
    p.add_argument("--edge-factor", type=int, default=16)
    p.add_argument("--seed", type=int, default=2)
    p.add_argument("--variant", default="ondemand", choices=["ondemand", "direct"])
    p.add_argument("--cpu-sample-scale", type=int, default=14)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--workload", default="decompose", choices=["decompose", "batch", "serve", "variants", "csr"],
                   help="decompose: the headline single-graph metric; batch: the batched form "
                        "(graphs/s of nucleus34_batch_decompose vs one decomposition per graph)")
    p.add_argument("--capture-run", action="store_true",
                   help="exactly one decomposition of the workload graph (for ncu captures); prints its record")
    p.add_argument("--peel-profile", action="store_true",
                   help="with --capture-run: per-step profiling mode (plain launches, per-round trace on stderr)")
    p.add_argument("--host-loop", action="store_true",
                   help="with --capture-run: the peel's host-driven replay graphs instead of the device loop")
    p.add_argument("--batch-graphs", type=int, default=4096)
    p.add_argument("--serve-requests", type=int, default=400)
    p.add_argument("--serve-max-edges", type=float, default=1e6)
    p.add_argument("--serve-master-seed", type=int, default=5)
    p.add_argument("--serve-load", default="0.5,1,2,4",
                   help="arrival rates as multiples of the serial plain capacity")
    p.add_argument("--serve-route", default="memory", choices=["memory", "ondemand"],
                   help="variant per request: by memory estimate (direct when it fits budget/direct_div) or on-demand")
    p.add_argument("--serve-direct-div", type=int, default=0)
    p.add_argument("--serve-budget-gb", type=float, default=0.0, help="server memory budget (0: the device's)")
    p.add_argument("--serve-workers", type=int, default=3)
    p.add_argument("--serve-concurrent-runs", type=int, default=0,
                   help="decompositions running at once per device slot (0: no limit)")
    p.add_argument("--batch-master-seed", type=int, default=4)
    return p.parse_args()


# ------------------------------------------------------------------ clocks --

class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.rows = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------- workloads --

def make_graph(n34, scale, ef, seed):
    s, d = n34.gen_rmat(scale, ef, seed)
    return n34.graph_from_edges(s, d)


def workload_name(a):
    return (f"R-MAT scale {a.scale} ef {a.edge_factor} (a,b,c,d)=(.57,.19,.19,.05) seed {a.seed}, "
            f"{a.variant} variant")


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return PEAKS_FALLBACK, "fallback"


_GOLD = 0x9E3779B97F4A7C15
_MIX1 = 0xBF58476D1CE4E5B9
_MIX2 = 0x94D049BB133111EB


def _mix64(z):
    """splitmix64 finaliser on a uint64 array (wrapping arithmetic)."""
    import numpy as np
    z = z + np.uint64(_GOLD)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(_MIX1)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(_MIX2)
    return z ^ (z >> np.uint64(31))


def rmat_edges_numpy(scale: int, ef: int, seed: int, a=0.57, b=0.19, c=0.19):
    """The library's seeded R-MAT generator restated in numpy, so that the
    reference arm's process maps no library of this project: edge i draws
    `scale` quadrant choices from a counter-based splitmix64 stream keyed by
    (seed, i); the list is then made undirected (u < v), loop-free, sorted
    and unique. Equal, edge for edge, to nucleus34.gen_rmat (checked by
    tests/test_bench_contract.py)."""
    import numpy as np
    m = int(ef) << int(scale)
    idx = np.arange(m, dtype=np.uint64)
    st = _mix64(np.uint64(seed) ^ _mix64(idx ^ np.uint64(0xD1B54A32D192ED03)))
    u = np.zeros(m, np.uint64)
    v = np.zeros(m, np.uint64)
    ab, abc = a + b, a + b + c
    for _ in range(scale):
        z = _mix64(st)
        st = st + np.uint64(_GOLD)
        r = (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
        bv = ((r >= a) & (r < ab)) | (r >= abc)
        bu = r >= ab
        u = (u << np.uint64(1)) | bu.astype(np.uint64)
        v = (v << np.uint64(1)) | bv.astype(np.uint64)
    keep = u != v
    lo, hi = np.minimum(u[keep], v[keep]), np.maximum(u[keep], v[keep])
    key = np.unique((lo << np.uint64(32)) | hi)
    return (key >> np.uint64(32)).astype(np.uint32), (key & np.uint64(0xffffffff)).astype(np.uint32)


def write_edges_text(src, dst, path: str) -> None:
    """`.edges` text as the library's writer makes it: the first edge twice
    (the reference reader consumes the first line as a header), then one
    "u v" line per edge."""
    import numpy as np
    if len(src) == 0:
        open(path, "w").close()
        return
    s = np.concatenate([src[:1], src]).astype(np.uint64)
    d = np.concatenate([dst[:1], dst]).astype(np.uint64)
    with open(path, "w") as f:
        step = 1 << 20
        for i in range(0, len(s), step):
            f.write("\n".join(f"{x} {y}" for x, y in zip(s[i:i + step].tolist(), d[i:i + step].tolist())))
            f.write("\n")


def cpu_reference_run(a, steps: int, warmup: int = 0):
    """Times the reference's CPU path (or the oracle port) on the bounded
    sample: `warmup` untimed runs, then `steps` timed ones (median). The
    sample file is generated in numpy here: this process loads no library of
    this project."""
    ref = os.path.join(ROOT, "oracle", "_ref", "cpu_ref")
    kind = "reference"
    if not os.path.exists(ref):
        ref = os.path.join(ROOT, "oracle", "_build", "nucleus34_oracle")
        kind = "port"
        if not os.path.exists(ref):
            subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "sample.edges")
        s, d = rmat_edges_numpy(a.cpu_sample_scale, a.edge_factor, a.seed)
        write_edges_text(s, d, path)
        for _ in range(warmup):
            subprocess.run([ref, path], check=True, capture_output=True, text=True)
        vals, recs = [], []
        for _ in range(steps):
            out = subprocess.run([ref, path], check=True, capture_output=True, text=True).stdout
            rec = json.loads(out.strip().splitlines()[-1])
            recs.append(rec)
            vals.append(rec["triangle_count"] / rec["t_decomp"])
    rec = recs[-1]
    return {
        "value": statistics.median(vals), "unit": UNIT, "cores": int(rec.get("threads", os.cpu_count())),
        "kind": kind,
        "sample": (f"R-MAT scale {a.cpu_sample_scale} ef {a.edge_factor} seed {a.seed} "
                   f"({rec['triangle_count']} triangles, {rec['four_clique_count']} four-cliques): the same "
                   f"generator and decomposition as the workload, bounded to ~seconds of CPU time; "
                   f"t_decomp = listing + cliques + peel, load excluded; median of {steps}. The reference's "
                   f"CPU path cannot hold the scale-{a.scale} workload: it materialises every four-clique "
                   f"(~64 B each; scale 18 already exceeds 62 GB of host memory)"),
        "t_decomp_s": statistics.median([r["t_decomp"] for r in recs]),
    }


# ------------------------------------------------------------------ main --

def batch_specs(count, master):
    """The batched workload: half R-MAT (scale U{8..14}, edge factor U{8..24},
    a/b/c/d .57/.19/.19/.05), half Watts-Strogatz (n log-uniform in
    [500, 20000], k=10, beta=0.1); graph i's parameters and seed come from
    splitmix64 of (master, i)."""
    import math
    import numpy as np
    import nucleus34 as n34
    out = []
    for i in range(count):
        s = n34.splitmix64((master << 32) ^ i)
        r = np.random.default_rng(s)
        if i % 2 == 0:
            out.append(("rmat", int(r.integers(8, 15)), int(r.integers(8, 25)), s & 0xffffffff))
        else:
            n = int(round(math.exp(r.uniform(math.log(500), math.log(20000)))))
            out.append(("ws", n, 10, s & 0xffffffff))
    return out


def replica_setup():
    """(rank, world, local device, dist module or None) for replicas under
    torchrun: one process per GPU, NCCL only for the barrier and the
    max-over-ranks timing (the graphs are independent: no data collective)."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world <= 1:
        return 0, 1, local, None
    import torch.distributed as tdist
    from datetime import timedelta
    tdist.init_process_group("nccl", timeout=timedelta(seconds=600))
    return rank, world, local, tdist


def my_share(n34, graphs, rank, world):
    """Indices of the graphs this rank decomposes (nucleus34_split_plan by
    estimated cost; every rank derives the same plan)."""
    if world <= 1:
        return list(range(len(graphs)))
    part_of, _ = n34.split_plan([n34.graph_cost(g) for g in graphs], world)
    return [i for i in range(len(graphs)) if part_of[i] == rank]


def run_batch(a):
    """Batched form: one nucleus34_batch_decompose pass over all graphs against
    one nucleus34_ctx_upload + nucleus34_ctx_run per graph on the same GPU;
    every graph's k compared bit for bit. Under torchrun each rank takes its
    share of the graphs (replicas); times are the slowest rank's."""
    import numpy as np
    import torch
    import nucleus34 as n34
    rank, world, dev, tdist = replica_setup()
    t0 = time.perf_counter()
    graphs = []
    for kind, x, y, seed in batch_specs(a.batch_graphs, a.batch_master_seed):
        src, dst = n34.gen_rmat(x, y, seed) if kind == "rmat" else n34.gen_ws(x, y, 0.1, seed)
        graphs.append(n34.graph_from_edges(src, dst))
    n_all = len(graphs)
    share = my_share(n34, graphs, rank, world)
    graphs = [graphs[i] for i in share]
    log(f"[bench] rank {rank}: {len(graphs)} of {n_all} graphs in {time.perf_counter() - t0:.1f} s, "
        f"{sum(g.m for g in graphs)} oriented edges")
    # plain: one decomposition per graph (context reused, graph uploaded each time)
    plain_k, plain_dev = [], 0.0
    with n34.Context(device=dev) as ctx:
        ctx.upload(graphs[0])
        ctx.run("ondemand")  # warm-up
        torch.cuda.synchronize()
        if tdist:
            tdist.barrier()
        w0 = time.perf_counter()
        for g in graphs:
            ctx.upload(g)
            r = ctx.run("ondemand")
            plain_dev += r["t_total"]
            plain_k.append(ctx.copy_k(int(r["triangle_count"])))
        plain_wall = time.perf_counter() - w0
    # batched: warm-up pass, then the timed pass
    with n34.batch_decompose(graphs[: min(64, len(graphs))], device=dev):
        pass
    torch.cuda.synchronize()
    if tdist:
        tdist.barrier()
    w0 = time.perf_counter()
    b = n34.batch_decompose(graphs, device=dev)
    batch_wall = time.perf_counter() - w0
    res = b.result
    mism = 0
    for i in range(len(graphs)):
        if not np.array_equal(b.copy_k(i), plain_k[i]):
            mism += 1
    b.close()
    if tdist:
        batch_wall = max_over_ranks(batch_wall, f"cuda:{dev}")
        plain_wall = max_over_ranks(plain_wall, f"cuda:{dev}")
        plain_dev = max_over_ranks(plain_dev, f"cuda:{dev}")
        mism = int(max_over_ranks(float(mism), f"cuda:{dev}"))
        tdist.barrier()
        tdist.destroy_process_group()
        if rank != 0:
            return 0
    n = n_all
    line = {
        "metric": "graphs/s (batched form)", "value": n / batch_wall, "unit": "graphs/s", "n_gpus": world,
        "scaling": "strong", "parallelism": f"replicas x{world}: graphs split by nucleus34_split_plan, no collective",
        "higher_is_better": True, "dtype": "int32", "data": "synthetic (seeded R-MAT + Watts-Strogatz)",
        "config": {"workload": f"{n} graphs: half R-MAT scale 8..14 ef 8..24, half Watts-Strogatz n 500..20000 "
                               f"k=10 beta=0.1, master seed {a.batch_master_seed}",
                   "triangles": int(res["triangle_count"]), "four_cliques": int(res["four_clique_count"])},
        "batched": {"wall_s": batch_wall, "device_s": res["t_total"], "upload_s": res["t_upload"],
                    "peel_rounds": int(res["peeling_iterations"]), "gpu_launches": int(res["gpu_launches"]),
                    "peak_device_bytes": int(res["peak_device_bytes"])},
        "plain": {"wall_s": plain_wall, "device_s": plain_dev, "graphs_per_s": n / plain_wall},
        "speedup_wall": plain_wall / batch_wall,
        "speedup_device": plain_dev / res["t_total"] if res["t_total"] else None,
        "k_mismatched_graphs": mism,
    }
    print(json.dumps(line), flush=True)
    return 0 if mism == 0 else 1


def serve_specs(count, master, max_edges):
    """Serving workload: half R-MAT (a/b/c/d .57/.19/.19/.05), half 2D random
    geometric graphs with expected degree U[16, 64]; undirected edge counts
    log-uniform over [1e3, max_edges]; request i's parameters and seed come
    from splitmix64 of (master, i)."""
    import math
    import numpy as np
    import nucleus34 as n34
    out = []
    for i in range(count):
        s = n34.splitmix64((master << 32) ^ (i + 0x9e3779b9))
        r = np.random.default_rng(s)
        m = math.exp(r.uniform(math.log(1e3), math.log(max_edges)))
        if i % 2 == 0:
            scale = max(4, int(math.ceil(math.log2(m / 16.0))))
            ef = max(1, int(round(m / (1 << scale))))
            out.append(("rmat", scale, ef, s & 0xffffffff))
        else:
            deg = float(r.uniform(16, 64))
            n = max(64, int(round(2 * m / deg)))
            out.append(("rgg", n, deg, s & 0xffffffff))
    return out


def run_serve(a):
    """Serving: Poisson arrivals into nucleus34_server (continuous batching,
    variant chosen per request by its memory estimate) against serial plain
    execution (one on-demand decomposition per request, FIFO, same arrival
    times: latencies from the measured service times). Under torchrun each
    rank serves its share of the requests (nucleus34_split_plan) on its own
    GPU with the same arrival times; latencies are gathered on rank 0."""
    import numpy as np
    import torch
    import nucleus34 as n34
    rank, world, dev, tdist = replica_setup()
    t0 = time.perf_counter()
    graphs = []
    for kind, x, y, seed in serve_specs(a.serve_requests, a.serve_master_seed, a.serve_max_edges):
        src, dst = n34.gen_rmat(x, y, seed) if kind == "rmat" else n34.gen_rgg(x, y, seed)
        graphs.append(n34.graph_from_edges(src, dst))
    n_all = len(graphs)
    share = my_share(n34, graphs, rank, world)
    log(f"[bench] rank {rank}: {len(share)} of {n_all} requests in {time.perf_counter() - t0:.1f} s, "
        f"{sum(graphs[i].m for i in share)} oriented edges")
    route = n34.ROUTE_MEMORY if a.serve_route == "memory" else n34.ROUTE_ONDEMAND
    budget = int(a.serve_budget_gb * 1e9)
    # serial plain service times (and the reference results) of this rank's share
    service, alone_k = {}, {}
    with n34.Context(device=dev) as ctx:
        ctx.upload(graphs[share[0]])
        ctx.run("ondemand")
        for i in share:
            w = time.perf_counter()
            ctx.upload(graphs[i])
            r = ctx.run("ondemand")
            k = ctx.copy_k(int(r["triangle_count"]))
            service[i] = time.perf_counter() - w
            alone_k[i] = k
    tot_service = sum(service.values())
    if tdist:
        tot_service = max_over_ranks(tot_service, f"cuda:{dev}")
    cap = n_all / tot_service  # plain capacity of the job (each rank serially), requests/s
    rng = np.random.default_rng(a.serve_master_seed)
    gaps = rng.exponential(1.0, n_all)
    sweeps = []
    mism = 0
    for load in [float(x) for x in a.serve_load.split(",")]:
        rate = load * cap
        arr = np.cumsum(gaps / rate)
        # serial plain: FIFO single server per rank
        done, lat_plain = 0.0, []
        for i in share:
            start = max(arr[i], done)
            done = start + service[i]
            lat_plain.append(done - arr[i])
        plain_end = done - arr[0]
        # the server, fed in real time
        if tdist:
            tdist.barrier()
        with n34.Server(device=dev, mem_budget_bytes=budget, workers=a.serve_workers, route=route,
                        direct_div=a.serve_direct_div, concurrent_runs=a.serve_concurrent_runs) as srv:
            ids = {}
            w0 = time.perf_counter()
            for i in share:
                wait = arr[i] - arr[0] - (time.perf_counter() - w0)
                if wait > 0:
                    time.sleep(wait)
                ids[i] = srv.submit(graphs[i])
            infos = {i: srv.wait(rid) for i, rid in ids.items()}
            end = time.perf_counter() - w0
            for i, rid in ids.items():
                if not np.array_equal(srv.copy_k(rid, infos[i]["triangle_count"]), alone_k[i]):
                    mism += 1
            st = srv.stats()
        slat = [infos[i]["latency_seconds"] for i in share]
        ndirect = sum(1 for i in share if infos[i]["direct"])
        worst = sorted(share, key=lambda i: -infos[i]["latency_seconds"])[:8]
        log(f"[bench] rank {rank} load {load}: slowest requests (latency, queue, triangles, pass, arrival, direct): " +
            "; ".join(f"{infos[i]['latency_seconds']:.3f} {infos[i]['queue_seconds']:.3f} "
                      f"{infos[i]['triangle_count']} {infos[i]['pass']} {arr[i] - arr[0]:.2f} {int(infos[i]['direct'])}"
                      for i in worst))
        mine = {"slat": slat, "plat": lat_plain, "end": end, "plain_end": plain_end, "passes": int(st["passes"]),
                "direct": ndirect}
        parts = [mine]
        if tdist:
            parts = [None] * world
            tdist.all_gather_object(parts, mine)
        slat_all = [x for p in parts for x in p["slat"]]
        plat_all = [x for p in parts for x in p["plat"]]
        end_all = max(p["end"] for p in parts)
        plain = {"p50_s": float(np.percentile(plat_all, 50)), "p99_s": float(np.percentile(plat_all, 99)),
                 "graphs_per_s": n_all / max(p["plain_end"] for p in parts)}
        served = {"p50_s": float(np.percentile(slat_all, 50)), "p99_s": float(np.percentile(slat_all, 99)),
                  "graphs_per_s": n_all / end_all, "passes": sum(p["passes"] for p in parts),
                  "direct_requests": sum(p["direct"] for p in parts)}
        sweeps.append({"load": load, "rate_per_s": rate, "server": served, "serial_plain": plain})
        log(f"[bench] load {load}: server p50 {served['p50_s']:.3f} p99 {served['p99_s']:.3f} "
            f"{served['graphs_per_s']:.1f}/s ({served['passes']} passes, {served['direct_requests']} direct); "
            f"plain p50 {plain['p50_s']:.3f} p99 {plain['p99_s']:.3f} {plain['graphs_per_s']:.1f}/s")
    if tdist:
        mism = int(max_over_ranks(float(mism), f"cuda:{dev}"))
        tdist.barrier()
        tdist.destroy_process_group()
        if rank != 0:
            return 0
    top = sweeps[-1]
    line = {
        "metric": "graphs/s and p50/p99 latency (serving)", "value": top["server"]["graphs_per_s"],
        "unit": "graphs/s", "n_gpus": world, "higher_is_better": True, "dtype": "int32", "scaling": "strong",
        "data": "synthetic (seeded R-MAT + 2D random geometric graphs)",
        "config": {"workload": f"{n_all} requests, Poisson arrivals, half R-MAT half RGG (degree 16..64), undirected "
                               f"edges log-uniform 1e3..{a.serve_max_edges:.0e}, master seed {a.serve_master_seed}",
                   "serial_plain_capacity_per_s": cap, "route": a.serve_route, "workers": a.serve_workers,
                   "concurrent_runs": a.serve_concurrent_runs,
                   "budget_bytes": budget or "device", "parallelism": f"replicas x{world}"},
        "sweep": sweeps, "k_mismatched_requests": mism,
    }
    print(json.dumps(line), flush=True)
    return 0 if mism == 0 else 1


def run_variants(a):
    """Direct against on-demand by graph size: device time (median of 3 warm
    runs on one context) and measured peak bytes of both variants on seeded
    graphs of serving sizes, one JSON line per graph (the data behind the
    serving loop's routing rule)."""
    import numpy as np
    import nucleus34 as n34
    cases = [("rmat", s, ef, 7) for s in (8, 10, 12, 14, 16) for ef in (8, 16, 24)] + \
            [("rgg", n, d, 3) for n in (2000, 20000, 200000) for d in (16.0, 32.0, 64.0)] + \
            [("ws", n, 10, 5) for n in (1000, 10000, 100000)]
    for kind, x, y, seed in cases:
        if kind == "rmat":
            s, d = n34.gen_rmat(x, y, seed)
        elif kind == "rgg":
            s, d = n34.gen_rgg(x, y, seed)
        else:
            s, d = n34.gen_ws(x, y, 0.1, seed)
        g = n34.graph_from_edges(s, d)
        D = g.D.astype(np.int64)
        row = {"graph": f"{kind} {x} {y}", "n": g.n, "m": g.m, "wedges": int((D * (D - 1) // 2).sum()),
               "triples": int((D * (D - 1) * (D - 2) // 6).sum())}
        with n34.Context() as ctx:
            ctx.upload(g)
            for v in ("ondemand", "direct"):
                ctx.run(v)
                ts = []
                for _ in range(3):
                    r = ctx.run(v)
                    ts.append(r["t_total"])
                row[v] = {"t_ms": 1e3 * float(np.median(ts)), "peak": int(r["peak_device_bytes"]),
                          "T": int(r["triangle_count"]), "Q": int(r["four_clique_count"])}
        print(json.dumps(row), flush=True)
    return 0


def run_csr(a):
    """The oriented CSR of an edge list built on the host
    (nucleus34_graph_from_edges) and on the device
    (nucleus34_ctx_upload_edges: pairs to the device, symmetrise, sort,
    unique, orient there), RGG 4M points degree 48 seed 3 and R-MAT scale 20:
    wall time of each (median of 3 after one warm-up), and the two CSRs
    compared entry for entry."""
    import numpy as np
    import nucleus34 as n34
    rows = []
    for name, gen in (("RGG 4M degree 48 seed 3", lambda: n34.gen_rgg(4000000, 48.0, 3)),
                      ("R-MAT scale 20 ef 16 seed 2", lambda: n34.gen_rmat(20, 16, 2))):
        s, d = gen()
        host, dev = [], []
        g = None
        for _ in range(4):
            t0 = time.perf_counter()
            g = n34.graph_from_edges(s, d)
            host.append(time.perf_counter() - t0)
        with n34.Context() as ctx:
            for _ in range(4):
                t0 = time.perf_counter()
                n, m = ctx.upload_edges(s, d)
                dev.append(time.perf_counter() - t0)
            got = ctx.copy_csr()
        same = (n, m) == (g.n, g.m) and np.array_equal(got.O, g.O[: g.n + 1]) and np.array_equal(got.E, g.E)
        rows.append({"graph": name, "pairs": int(len(s)), "n": int(g.n), "m": int(g.m),
                     "host_build_s": statistics.median(host[1:]), "device_build_s": statistics.median(dev[1:]),
                     "host_threads": os.cpu_count(), "same_csr": bool(same)})
        log(f"[bench] {name}: host {rows[-1]['host_build_s']:.3f} s, device {rows[-1]['device_build_s']:.3f} s, "
            f"same {same}")
    print(json.dumps({"metric": "oriented CSR build time", "unit": "s", "rows": rows}), flush=True)
    return 0 if all(r["same_csr"] for r in rows) else 1


def capture_run(a):
    """One decomposition and nothing else, so that ncu launch indices are
    those of that decomposition alone."""
    import nucleus34 as n34
    g = make_graph(n34, a.scale, a.edge_factor, a.seed)
    flags = (n34.OPT_PROFILE_PEEL if a.peel_profile else 0) | (n34.OPT_HOST_LOOP if a.host_loop else 0)
    with n34.Context(flags=flags) as ctx:
        ctx.upload(g)
        r = ctx.run(a.variant)
    print(json.dumps({"workload": workload_name(a), **r}), flush=True)
    return 0


def spread(xs):
    """min / median / max of the timed steps, and (max - min) / median."""
    med = statistics.median(xs)
    return {"min": min(xs), "median": med, "max": max(xs), "spread": (max(xs) - min(xs)) / med if med else None}


def max_over_ranks(x: float, device: str) -> float:
    """The slowest rank's time (all_reduce MAX over the process group): the
    job is done when its last replica is."""
    import torch
    import torch.distributed as tdist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def job_value(world: int, triangles: int, steps: int, seconds: float) -> float:
    """Whole-job throughput of N replicas: every rank peels the workload's
    triangles once per step, all within the slowest rank's time."""
    return world * triangles * steps / seconds


def main():
    a = parse()
    if a.capture_run:
        return capture_run(a)
    if a.workload == "batch":
        return run_batch(a)
    if a.workload == "serve":
        return run_serve(a)
    if a.workload == "variants":
        return run_variants(a)
    if a.workload == "csr":
        return run_csr(a)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(a.gpus)))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if a.impl == "reference":
        if rank != 0:
            return 0
        steps = max(1, a.steps)
        warmup = max(0, a.warmup)
        cb = cpu_reference_run(a, steps, warmup)
        line = {
            "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": a.gpus,
            "steps": steps, "warmup": warmup, "ms_per_step": cb["t_decomp_s"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": workload_name(a), "sample": cb["sample"],
                       "same_config": False,
                       "why_sample": "the reference CPU path materialises every four-clique (~64 B each): the "
                                     f"scale-{a.scale} graph's ~1.7e10 cliques do not fit host memory"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return 0

    import numpy as np
    import torch
    import nucleus34 as n34

    dist = world > 1
    if dist:
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=600))
    device = local if dist else 0
    torch.cuda.set_device(device)

    g = make_graph(n34, a.scale, a.edge_factor, a.seed)
    log(f"[bench] rank {rank}: graph n={g.n} m={g.m}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{device}")

    def barrier():
        if dist:
            tdist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident steps (value) ----
    ctx = n34.Context(device=device)
    ctx.upload(g)
    for _ in range(a.warmup):
        r = ctx.run(a.variant)
    barrier()
    clocks = ClockSampler(device)
    clocks.start()
    times, results = [], []
    wall0 = time.perf_counter()
    for _ in range(a.steps):
        flush.zero_()               # L2 flush between steps (256 MiB write)
        torch.cuda.synchronize()
        r = ctx.run(a.variant)      # synchronous; device time from library events
        times.append(r["t_total"])
        results.append(r)
    barrier()
    wall = time.perf_counter() - wall0
    clk = clocks.stop()
    T = results[-1]["triangle_count"]
    dev_time = sum(times)
    if dist:
        dev_time = max_over_ranks(dev_time, f"cuda:{device}")
    ms_per_step = dev_time / a.steps * 1e3
    value = job_value(world, T, a.steps, dev_time)
    launches = sum(r["gpu_launches"] for r in results)
    ctx.close()

    # ---- one untimed run with per-kernel CUDA events in the peel: device time
    # of the re-enumeration (debit) kernels for the roofline ----
    with n34.Context(device=device, flags=n34.OPT_PROFILE_PEEL) as pctx:
        pctx.upload(g)
        prof = pctx.run(a.variant)

    # ---- end-to-end through the one-shot C-ABI call (e2e) ----
    e2e = None
    if not a.no_e2e:
        import ctypes as C
        L = n34.lib()
        O = torch.empty(g.n, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
        D = torch.empty(g.n, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
        E = torch.empty(max(g.m, 1), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
        O[:] = g.O[:-1]
        D[:] = g.D
        E[: g.m] = g.E
        kbuf = torch.empty(max(T, 1), dtype=torch.int32, pin_memory=True).numpy()
        u32p = C.POINTER(C.c_uint32)
        csr = n34.Csr(g.n, g.m, O.ctypes.data_as(u32p), D.ctypes.data_as(u32p), E.ctypes.data_as(u32p))
        opts = n34.make_opts(device)
        fn = L.nucleus34_decompose_ondemand if a.variant == "ondemand" else L.nucleus34_decompose
        e2e_times = []
        for it in range(max(1, a.steps)):
            flush.zero_()
            torch.cuda.synchronize()
            barrier()
            t0 = time.perf_counter()
            res = n34.Result()
            h = C.c_void_p()
            rc = fn(C.byref(csr), C.byref(opts), C.byref(res), C.byref(h))
            if rc:
                raise n34.Nucleus34Error(rc, "decompose", n34.last_error())
            rc = L.nucleus34_copy_k(h, kbuf.ctypes.data_as(C.POINTER(C.c_int32)), None)
            t1 = time.perf_counter()
            L.nucleus34_free(h)
            if rc:
                raise n34.Nucleus34Error(rc, "copy_k", n34.last_error())
            e2e_times.append(t1 - t0)
        et = sum(e2e_times)
        if dist:
            et = max_over_ranks(et, f"cuda:{device}")
        e2e = {"value": job_value(world, T, len(e2e_times), et), "unit": UNIT,
               "h2d_bytes_per_step": int(4 * (2 * g.n + g.m)), "d2h_bytes_per_step": int(4 * T),
               "ms_per_step": et / len(e2e_times) * 1e3,
               "api": "nucleus34_decompose_ondemand + nucleus34_copy_k" if a.variant == "ondemand"
               else "nucleus34_decompose + nucleus34_copy_k"}

    if dist:
        tdist.barrier()
        tdist.destroy_process_group()
    if rank != 0:
        return 0

    peaks, peak_kind = measured_peaks()
    r = results[-1]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic (seeded R-MAT; no datasets on this system)",
        "config": {"workload": workload_name(a), "vertices": int(g.n), "oriented_edges": int(g.m),
                   "triangles": int(T), "four_cliques": int(r["four_clique_count"]),
                   "parallelism": f"replicas x{world} (one graph per GPU, no collective)",
                   "l2": "inputs > L2 and a 256 MiB L2-flush write between steps"},
        "phases_ms": {k: r[k] * 1e3 for k in ("t_triangles", "t_incidence", "t_support", "t_cliques", "t_peel")},
        "steps_ms": {k: spread([x[k] * 1e3 for x in results])
                     for k in ("t_total", "t_triangles", "t_incidence", "t_support", "t_peel")},
        "peel_rounds": int(r["peeling_iterations"]), "k_max": int(r["k_max"]),
        "peak_device_bytes": int(r["peak_device_bytes"]),
        "gpu_launches": int(launches),
        "wall_s": wall,
        "clocks": clk,
    }
    if e2e:
        line["e2e"] = e2e
    line["roofline"], line["roofline_support"] = roofline(r, prof, peaks, peak_kind)
    if not a.no_cpu_baseline:
        try:
            cb = cpu_reference_run(a, 1)
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as ex:  # reported, never fatal
            line["cpu_baseline"] = {"error": str(ex)}
    print(json.dumps(line), flush=True)
    return 0


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per algorithmic
# byte of k_support, from its single-launch ncu capture on a smaller case of
# the same workload (R-MAT scale 17), applied to this run's algorithmic bytes:
# its traffic grows with the lists it reads. The debit runs as thousands of
# launches of different sizes, and an ncu capture covers one to three of them,
# so no per-launch figure of its traffic matches the whole-peel `achieved`:
# its `traffic` is null, and its single-round captures are summarised beside
# the kernel's profile.
NCU_TRAFFIC_PER_ALG_BYTE = {"k_support": 0.028}


def roofline(r, prof, peaks, kind):
    """HBM roofline of the two intersection phases.

    Algorithmic bytes of one full enumeration (every triangle's lists
    intersected once) use the zipper bound 4*sum_e T(e)^2 + 36*T + 48*Q: each
    triangle reads its three edges' incidence lists (4 B per entry), its own
    record and list bounds (36 B), and each of the 4Q clique occurrences reads
    3 partner ids (48 B per clique). The support count performs one
    enumeration in one launch (k_support); the peel performs it once more,
    spread over its rounds (k_debit_flags_warp + k_debit_flags_thread, two
    launches per round), timed by CUDA events around those kernels in a
    separate profiling run of the same workload. Both kernels intersect only
    the two shortest lists of a triangle, so they move fewer bytes than this
    bound and a fraction above 1 is possible."""
    T, Q, S2 = r["triangle_count"], r["four_clique_count"], r["sum_te_sq"]
    alg = 4 * S2 + 36 * T + 48 * Q
    peak = peaks.get("hbm_gbs")
    pk = f"{kind} ({'hbm_gbs' if kind == 'measured' else 'fallback 6.65 TB/s'})"
    out = []
    for name, key, t, launches, what in (
            ("k_debit_flags_warp+k_debit_flags_thread", "debit", prof.get("t_peel_debit", 0.0),
             2 * int(prof.get("peeling_iterations", 0)), "peel re-enumeration, all rounds (profiling run)"),
            ("k_support", "k_support", r["t_support"], 1, "support count (one launch, timed run)")):
        ach = alg / t / 1e9 if t > 0 else None
        ratio = NCU_TRAFFIC_PER_ALG_BYTE.get(key)
        out.append({"kernel": name, "what": what, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                    "frac": (ach / peak) if (ach and peak) else None,
                    "traffic": (ratio * alg) if ratio else None, "algorithmic_bytes": alg,
                    "device_seconds": t, "launches": launches, "peak_kind": pk,
                    "definition": "4*sum_e T(e)^2 + 36T + 48Q bytes per full enumeration (zipper bound)"})
    # the dominant kernel is the one with the larger device time
    if out[1]["device_seconds"] > out[0]["device_seconds"]:
        out.reverse()
    return out[0], out[1]


if __name__ == "__main__":
    sys.exit(main())
