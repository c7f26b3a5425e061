"""ctypes binding of libnucleus34 (the C-ABI declared in include/nucleus34.h).

This is the Python face of the library for the tests, the bench and
scripting: every call goes through the same extern "C" entry points a C/C++
caller uses. The library must be built first (``make -C gpu-nucleus34_b200``);
there is no pure-Python or CPU fallback for the decomposition -- a missing
library raises.

Reference mapping: ``decompose(..., variant="direct")`` is the device
pipeline of nucleus/cuNucleus34.cu:283-721, ``variant="ondemand"`` that of
nucleus/cuNucleus34_ondemand.cu:407-690; ``load_graph`` is graph_t::from_edges
/ deserialize + make_oriented (nucleus/graph/graph.hpp:176-218, 285-411,
491-536).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT_DIR = os.path.dirname(PKG_DIR)
LIB_PATH = os.path.join(ROOT_DIR, "lib", "libnucleus34.so")
BIN_DIR = os.path.join(ROOT_DIR, "bin")

OK = 0
E_INVALID = -1
E_OOM_BUDGET = -2
E_RANGE32 = -3
E_CUDA = -4
E_TIMEOUT = -5
E_IO = -6
E_FORMAT = -7
E_NODEVICE = -8
E_STATE = -9

DIRECT = 0
ONDEMAND = 1
_VARIANTS = {"direct": DIRECT, "ondemand": ONDEMAND, DIRECT: DIRECT, ONDEMAND: ONDEMAND}

# Every symbol include/nucleus34.h declares (checked by the CPU test suite).
EXPORTED = (
    "nucleus34_decompose", "nucleus34_decompose_ondemand", "nucleus34_copy_k",
    "nucleus34_copy_quds", "nucleus34_write_kfile", "nucleus34_free", "nucleus34_release_cached_memory",
    "nucleus34_batch_decompose", "nucleus34_batch_summary", "nucleus34_batch_copy_k", "nucleus34_batch_free",
    "nucleus34_server_create", "nucleus34_server_submit", "nucleus34_server_wait", "nucleus34_server_copy_k",
    "nucleus34_server_copy_quds", "nucleus34_server_release", "nucleus34_server_stats", "nucleus34_server_destroy",
    "nucleus34_strerror", "nucleus34_last_error",
    "nucleus34_ctx_create", "nucleus34_ctx_upload", "nucleus34_ctx_run",
    "nucleus34_ctx_copy_k", "nucleus34_ctx_destroy", "nucleus34_ctx_verify",
    "nucleus34_tune_lookup", "nucleus34_tune_store", "nucleus34_ctx_set_tune", "nucleus34_ctx_last_tune",
    "nucleus34_ctx_autotune", "nucleus34_ctx_upload_edges", "nucleus34_ctx_copy_csr",
    "nucleus34_graph_load", "nucleus34_graph_from_edges", "nucleus34_graph_save_grh",
    "nucleus34_graph_release", "nucleus34_graph_csr",
    "nucleus34_gen_rmat", "nucleus34_gen_rgg", "nucleus34_gen_ws",
    "nucleus34_edges_write", "nucleus34_edges_release", "nucleus34_splitmix64",
    "nucleus34_graph_cost", "nucleus34_split_plan", "nucleus34_server_estimate",
)


class Nucleus34Error(RuntimeError):
    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        msg = f"{where}: {strerror(code)} ({code})"
        if detail:
            msg += f": {detail}"
        super().__init__(msg)


class Csr(C.Structure):
    _fields_ = [("n", C.c_uint64), ("m", C.c_uint64), ("O", C.POINTER(C.c_uint32)),
                ("D", C.POINTER(C.c_uint32)), ("E", C.POINTER(C.c_uint32))]


class Opts(C.Structure):
    _fields_ = [("mem_budget_bytes", C.c_uint64), ("device", C.c_int),
                ("parts", C.c_uint32), ("tune_table", C.c_char_p), ("flags", C.c_uint32)]


TUNE_NEVER = 0xFFFFFFFF
_TUNE_FIELDS = ("lane_max", "compact_div", "sort_shift", "rounds_per_replay")


class Tune(C.Structure):
    """nucleus34_tune: scheduling settings of the on-demand variant (0 = default)."""
    _fields_ = [(f, C.c_uint32) for f in _TUNE_FIELDS]

    def as_dict(self) -> dict:
        return {f: ("never" if getattr(self, f) == TUNE_NEVER else int(getattr(self, f))) for f in _TUNE_FIELDS}

    @classmethod
    def from_dict(cls, d: dict) -> "Tune":
        unknown = set(d) - set(_TUNE_FIELDS)
        if unknown:
            raise ValueError(f"unknown tune settings: {sorted(unknown)}")
        return cls(*[TUNE_NEVER if d.get(f, 0) == "never" else int(d.get(f, 0)) for f in _TUNE_FIELDS])


class Result(C.Structure):
    _fields_ = [("triangle_count", C.c_uint64), ("four_clique_count", C.c_uint64),
                ("peeling_iterations", C.c_uint64), ("unpeeled_count", C.c_uint64),
                ("k_max", C.c_uint32), ("k_avg", C.c_double),
                ("t_triangles", C.c_double), ("t_incidence", C.c_double),
                ("t_support", C.c_double), ("t_cliques", C.c_double),
                ("t_peel", C.c_double), ("t_total", C.c_double),
                ("incidence_entries", C.c_uint64), ("gpu_launches", C.c_uint64),
                ("peak_device_bytes", C.c_uint64), ("variant", C.c_int),
                ("sum_te_sq", C.c_uint64), ("t_peel_debit", C.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class BatchResult(C.Structure):
    _fields_ = [("graphs", C.c_uint64), ("triangle_count", C.c_uint64), ("four_clique_count", C.c_uint64),
                ("peeling_iterations", C.c_uint64), ("t_upload", C.c_double), ("t_triangles", C.c_double),
                ("t_incidence", C.c_double), ("t_support", C.c_double), ("t_peel", C.c_double),
                ("t_total", C.c_double), ("gpu_launches", C.c_uint64), ("peak_device_bytes", C.c_uint64),
                ("chunks", C.c_uint64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class GraphSummary(C.Structure):
    _fields_ = [("triangle_count", C.c_uint64), ("four_clique_count", C.c_uint64), ("k_max", C.c_uint32),
                ("k_avg", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerOpts(C.Structure):
    _fields_ = [("workers", C.c_uint32), ("max_batch_graphs", C.c_uint64), ("route", C.c_uint32),
                ("direct_div", C.c_uint32), ("device_count", C.c_uint32), ("devices", C.POINTER(C.c_int)),
                ("concurrent_runs", C.c_uint32)]


class RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("summary", GraphSummary), ("queue_seconds", C.c_double),
                ("latency_seconds", C.c_double), ("pass_", C.c_uint64), ("direct", C.c_int)]

    def as_dict(self) -> dict:
        return {"status": self.status, **self.summary.as_dict(), "queue_seconds": self.queue_seconds,
                "latency_seconds": self.latency_seconds, "pass": self.pass_, "direct": bool(self.direct)}


class RequestEstimate(C.Structure):
    _fields_ = [("ondemand_bytes", C.c_uint64), ("direct_bytes", C.c_uint64), ("triangle_bound", C.c_uint64),
                ("clique_bound", C.c_uint64), ("direct", C.c_int)]


class ServerCounters(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("passes", "served", "pending", "busy_workers", "workers",
                                          "in_flight_bytes", "budget_bytes", "direct_served", "devices")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Graph(C.Structure):
    _fields_ = [("n", C.c_uint64), ("m", C.c_uint64), ("O", C.POINTER(C.c_uint32)),
                ("D", C.POINTER(C.c_uint32)), ("E", C.POINTER(C.c_uint32))]


class Edges(C.Structure):
    _fields_ = [("count", C.c_uint64), ("src", C.POINTER(C.c_uint32)),
                ("dst", C.POINTER(C.c_uint32))]


_LIB: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """Loads libnucleus34.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(
            f"{LIB_PATH} is missing: build it with `make -C {ROOT_DIR}` "
            "(there is no fallback implementation)")
    L = C.CDLL(LIB_PATH)
    u32p, u64 = C.POINTER(C.c_uint32), C.c_uint64
    L.nucleus34_strerror.restype = C.c_char_p
    L.nucleus34_strerror.argtypes = [C.c_int]
    L.nucleus34_last_error.restype = C.c_char_p
    L.nucleus34_last_error.argtypes = []
    for fn in ("nucleus34_decompose", "nucleus34_decompose_ondemand"):
        getattr(L, fn).argtypes = [C.POINTER(Csr), C.POINTER(Opts), C.POINTER(Result), C.POINTER(C.c_void_p)]
        getattr(L, fn).restype = C.c_int
    L.nucleus34_copy_k.argtypes = [C.c_void_p, C.POINTER(C.c_int32), u32p]
    L.nucleus34_copy_k.restype = C.c_int
    L.nucleus34_copy_quds.argtypes = [C.c_void_p, u64, u64, u32p]
    L.nucleus34_copy_quds.restype = C.c_int
    L.nucleus34_write_kfile.argtypes = [C.c_void_p, C.c_char_p]
    L.nucleus34_write_kfile.restype = C.c_int
    L.nucleus34_free.argtypes = [C.c_void_p]
    L.nucleus34_free.restype = None
    L.nucleus34_release_cached_memory.argtypes = [C.c_int]
    L.nucleus34_release_cached_memory.restype = C.c_int
    L.nucleus34_batch_decompose.argtypes = [C.POINTER(Csr), C.c_uint64, C.POINTER(Opts), C.POINTER(BatchResult),
                                            C.POINTER(C.c_void_p)]
    L.nucleus34_batch_decompose.restype = C.c_int
    L.nucleus34_batch_summary.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(GraphSummary)]
    L.nucleus34_batch_summary.restype = C.c_int
    L.nucleus34_batch_copy_k.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(C.c_int32), u32p]
    L.nucleus34_batch_copy_k.restype = C.c_int
    L.nucleus34_batch_free.argtypes = [C.c_void_p]
    L.nucleus34_batch_free.restype = None
    L.nucleus34_graph_cost.argtypes = [C.POINTER(Csr), C.POINTER(C.c_uint64)]
    L.nucleus34_graph_cost.restype = C.c_int
    L.nucleus34_split_plan.argtypes = [C.POINTER(C.c_uint64), C.c_uint64, C.c_uint32, C.POINTER(C.c_uint32),
                                       C.POINTER(C.c_uint64)]
    L.nucleus34_split_plan.restype = C.c_int
    L.nucleus34_server_estimate.argtypes = [C.POINTER(Csr), C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                                            C.POINTER(RequestEstimate)]
    L.nucleus34_server_estimate.restype = C.c_int
    L.nucleus34_server_create.argtypes = [C.POINTER(Opts), C.POINTER(ServerOpts), C.POINTER(C.c_void_p)]
    L.nucleus34_server_create.restype = C.c_int
    L.nucleus34_server_submit.argtypes = [C.c_void_p, C.POINTER(Csr), C.c_uint32, C.POINTER(C.c_uint64)]
    L.nucleus34_server_submit.restype = C.c_int
    L.nucleus34_server_wait.argtypes = [C.c_void_p, C.c_uint64, C.c_int64, C.POINTER(RequestInfo)]
    L.nucleus34_server_wait.restype = C.c_int
    L.nucleus34_server_copy_k.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(C.c_int32), u32p]
    L.nucleus34_server_copy_k.restype = C.c_int
    L.nucleus34_server_copy_quds.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, u32p]
    L.nucleus34_server_copy_quds.restype = C.c_int
    L.nucleus34_server_release.argtypes = [C.c_void_p, C.c_uint64]
    L.nucleus34_server_release.restype = C.c_int
    L.nucleus34_server_stats.argtypes = [C.c_void_p, C.POINTER(ServerCounters)]
    L.nucleus34_server_stats.restype = C.c_int
    L.nucleus34_server_destroy.argtypes = [C.c_void_p]
    L.nucleus34_server_destroy.restype = None
    L.nucleus34_ctx_create.argtypes = [C.POINTER(Opts), C.POINTER(C.c_void_p)]
    L.nucleus34_ctx_create.restype = C.c_int
    L.nucleus34_ctx_upload.argtypes = [C.c_void_p, C.POINTER(Csr)]
    L.nucleus34_ctx_upload.restype = C.c_int
    L.nucleus34_ctx_run.argtypes = [C.c_void_p, C.c_int, C.POINTER(Result)]
    L.nucleus34_ctx_run.restype = C.c_int
    L.nucleus34_ctx_copy_k.argtypes = [C.c_void_p, C.POINTER(C.c_int32), u32p]
    L.nucleus34_ctx_copy_k.restype = C.c_int
    L.nucleus34_ctx_verify.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.nucleus34_ctx_verify.restype = C.c_int
    L.nucleus34_ctx_destroy.argtypes = [C.c_void_p]
    L.nucleus34_ctx_upload_edges.argtypes = [C.c_void_p, u32p, u32p, u64, C.POINTER(C.c_uint64),
                                             C.POINTER(C.c_uint64)]
    L.nucleus34_ctx_upload_edges.restype = C.c_int
    L.nucleus34_ctx_copy_csr.argtypes = [C.c_void_p, u32p, u32p, u32p]
    L.nucleus34_ctx_copy_csr.restype = C.c_int
    L.nucleus34_tune_lookup.argtypes = [C.c_char_p, u64, u64, u64, C.c_uint32, C.POINTER(Tune), C.POINTER(C.c_int)]
    L.nucleus34_tune_lookup.restype = C.c_int
    L.nucleus34_tune_store.argtypes = [C.c_char_p, u64, u64, u64, C.c_uint32, C.POINTER(Tune), C.c_double,
                                       C.c_double]
    L.nucleus34_tune_store.restype = C.c_int
    L.nucleus34_ctx_set_tune.argtypes = [C.c_void_p, C.POINTER(Tune)]
    L.nucleus34_ctx_set_tune.restype = C.c_int
    L.nucleus34_ctx_last_tune.argtypes = [C.c_void_p, C.POINTER(Tune)]
    L.nucleus34_ctx_last_tune.restype = C.c_int
    L.nucleus34_ctx_autotune.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(Tune), C.POINTER(C.c_double),
                                         C.POINTER(C.c_double)]
    L.nucleus34_ctx_autotune.restype = C.c_int
    L.nucleus34_ctx_destroy.restype = None
    L.nucleus34_graph_load.argtypes = [C.c_char_p, C.POINTER(Graph)]
    L.nucleus34_graph_load.restype = C.c_int
    L.nucleus34_graph_from_edges.argtypes = [u32p, u32p, u64, C.POINTER(Graph)]
    L.nucleus34_graph_from_edges.restype = C.c_int
    L.nucleus34_graph_save_grh.argtypes = [C.POINTER(Graph), C.c_char_p]
    L.nucleus34_graph_save_grh.restype = C.c_int
    L.nucleus34_graph_release.argtypes = [C.POINTER(Graph)]
    L.nucleus34_graph_release.restype = None
    L.nucleus34_gen_rmat.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, u64, C.POINTER(Edges)]
    L.nucleus34_gen_rmat.restype = C.c_int
    L.nucleus34_gen_rgg.argtypes = [u64, C.c_double, u64, C.POINTER(Edges)]
    L.nucleus34_gen_rgg.restype = C.c_int
    L.nucleus34_gen_ws.argtypes = [u64, C.c_uint32, C.c_double, u64, C.POINTER(Edges)]
    L.nucleus34_gen_ws.restype = C.c_int
    L.nucleus34_edges_write.argtypes = [C.POINTER(Edges), C.c_char_p]
    L.nucleus34_edges_write.restype = C.c_int
    L.nucleus34_edges_release.argtypes = [C.POINTER(Edges)]
    L.nucleus34_edges_release.restype = None
    L.nucleus34_splitmix64.argtypes = [u64]
    L.nucleus34_splitmix64.restype = u64
    _LIB = L
    return L


def strerror(code: int) -> str:
    return lib().nucleus34_strerror(code).decode()


def last_error() -> str:
    return lib().nucleus34_last_error().decode()


def _check(rc: int, where: str) -> None:
    if rc != OK:
        raise Nucleus34Error(rc, where, last_error())


def _u32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def splitmix64(x: int) -> int:
    return int(lib().nucleus34_splitmix64(C.c_uint64(x & 0xFFFFFFFFFFFFFFFF)))


# ---------------------------------------------------------------- graphs ----

def graph_cost(g: "HostGraph") -> int:
    """Estimated cost of decomposing g: oriented edges plus out-wedges."""
    c = C.c_uint64()
    csr = g.csr()
    _check(lib().nucleus34_graph_cost(C.byref(csr), C.byref(c)), "graph_cost")
    return int(c.value)


def split_plan(costs, parts: int):
    """Share of each graph when `len(costs)` graphs are split over `parts`
    replicas (nucleus34_split_plan: greedy longest-processing-time,
    deterministic). Returns (part_of, load) as numpy arrays."""
    c = np.ascontiguousarray(np.asarray(costs, dtype=np.uint64))
    part_of = np.zeros(len(c), np.uint32)
    load = np.zeros(max(parts, 1), np.uint64)
    _check(lib().nucleus34_split_plan(c.ctypes.data_as(C.POINTER(C.c_uint64)), len(c), parts,
                                      _u32p(part_of) if len(c) else None,
                                      load.ctypes.data_as(C.POINTER(C.c_uint64))), "split_plan")
    return part_of, load[:parts]


def server_estimate(g: "HostGraph", budget: int, route: int = 0, direct_div: int = 0,
                    cliques: bool = False, triangles: bool = False) -> dict:
    """The serving loop's admission estimates and variant for g, without a
    server or a device (nucleus34_server_estimate): budget is the smallest
    slot budget, route a ROUTE_* constant, direct_div 0 for the default."""
    e = RequestEstimate()
    csr = g.csr()
    flags = (REQ_CLIQUES if cliques else 0) | (REQ_TRIANGLES if triangles else 0)
    _check(lib().nucleus34_server_estimate(C.byref(csr), budget, route, direct_div, flags, C.byref(e)),
           "server_estimate")
    return {"ondemand_bytes": int(e.ondemand_bytes), "direct_bytes": int(e.direct_bytes),
            "triangle_bound": int(e.triangle_bound), "clique_bound": int(e.clique_bound),
            "direct": bool(e.direct)}


@dataclass
class HostGraph:
    """Oriented CSR as numpy arrays (O has n+1 entries)."""
    n: int
    m: int
    O: np.ndarray
    D: np.ndarray
    E: np.ndarray

    def csr(self) -> Csr:
        return Csr(self.n, self.m, _u32p(self.O), _u32p(self.D), _u32p(self.E))


def _take_graph(g: Graph) -> HostGraph:
    L = lib()
    n, m = int(g.n), int(g.m)
    O = np.ctypeslib.as_array(g.O, shape=(n + 1,)).copy()
    D = np.ctypeslib.as_array(g.D, shape=(n,)).copy() if n else np.zeros(0, np.uint32)
    E = np.ctypeslib.as_array(g.E, shape=(m,)).copy() if m else np.zeros(0, np.uint32)
    L.nucleus34_graph_release(C.byref(g))
    return HostGraph(n, m, O, D, E)


def load_graph(path: str) -> HostGraph:
    g = Graph()
    _check(lib().nucleus34_graph_load(os.fsencode(path), C.byref(g)), f"load_graph({path})")
    return _take_graph(g)


def graph_from_edges(src: np.ndarray, dst: np.ndarray) -> HostGraph:
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    g = Graph()
    _check(lib().nucleus34_graph_from_edges(_u32p(src), _u32p(dst), len(src), C.byref(g)),
           "graph_from_edges")
    return _take_graph(g)


def save_grh(g: HostGraph, path: str) -> None:
    gg = Graph(g.n, g.m, _u32p(g.O), _u32p(g.D), _u32p(g.E))
    _check(lib().nucleus34_graph_save_grh(C.byref(gg), os.fsencode(path)), "save_grh")


# ------------------------------------------------------------ generators ----

def _take_edges(e: Edges):
    c = int(e.count)
    src = np.ctypeslib.as_array(e.src, shape=(c,)).copy() if c else np.zeros(0, np.uint32)
    dst = np.ctypeslib.as_array(e.dst, shape=(c,)).copy() if c else np.zeros(0, np.uint32)
    lib().nucleus34_edges_release(C.byref(e))
    return src, dst


def gen_rmat(scale: int, edge_factor: int, seed: int, a=0.57, b=0.19, c=0.19):
    e = Edges()
    _check(lib().nucleus34_gen_rmat(scale, edge_factor, a, b, c, seed, C.byref(e)), "gen_rmat")
    return _take_edges(e)


def gen_rgg(n: int, degree: float, seed: int):
    e = Edges()
    _check(lib().nucleus34_gen_rgg(n, degree, seed, C.byref(e)), "gen_rgg")
    return _take_edges(e)


def gen_ws(n: int, k: int, beta: float, seed: int):
    e = Edges()
    _check(lib().nucleus34_gen_ws(n, k, beta, seed, C.byref(e)), "gen_ws")
    return _take_edges(e)


def write_edges(src: np.ndarray, dst: np.ndarray, path: str) -> None:
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    e = Edges(len(src), _u32p(src), _u32p(dst))
    _check(lib().nucleus34_edges_write(C.byref(e), os.fsencode(path)), "write_edges")


# --------------------------------------------------------- decomposition ----

@dataclass
class Decomposition:
    result: dict
    k: np.ndarray
    tris: np.ndarray
    quds: Optional[np.ndarray] = None
    extra: dict = field(default_factory=dict)


OPT_STAMP_PEEL = 0x1
OPT_PROFILE_PEEL = 0x2
OPT_LEAN_MEMORY = 0x4
OPT_VERIFIABLE = 0x8
OPT_HOST_RESULTS = 0x10
OPT_HOST_LOOP = 0x20
OPT_NO_SMALL_ROUNDS = 0x40
OPT_FRONTIER_BY_C = 0x80
OPT_CHUNKED_DEBIT = 0x100
OPT_SCALAR_SCANS = 0x200
OPT_PIPELINED_DEBIT = 0x400
OPT_DEBIT_CURSOR = 0x800


# The tune table the autotuner wrote on a B200 for this build's measured graph
# classes; used when no other table is given ("" selects the built-in
# defaults).
SHIPPED_TUNE_TABLE = os.path.join(ROOT_DIR, "tune", "b200.tune")


def make_opts(device: int = 0, mem_budget_bytes: int = 0, parts: int = 1, flags: int = 0,
              tune_table: Optional[str] = None) -> Opts:
    if tune_table is None and os.path.exists(SHIPPED_TUNE_TABLE):
        tune_table = SHIPPED_TUNE_TABLE
    return Opts(mem_budget_bytes, device, parts, os.fsencode(tune_table) if tune_table else None, flags)


def tune_lookup(path: str, triangles: int, n: int, m: int, max_out: int) -> tuple:
    """(settings dict, matched) that the tune table at path gives a graph of
    `triangles` triangles whose oriented CSR has n vertices, m edges and
    maximum out-degree max_out (nucleus34_tune_lookup; host only)."""
    t, matched = Tune(), C.c_int()
    _check(lib().nucleus34_tune_lookup(os.fsencode(path), triangles, n, m, max_out, C.byref(t),
                                       C.byref(matched)), "tune_lookup")
    return t.as_dict(), bool(matched.value)


def tune_store(path: str, triangles: int, n: int, m: int, max_out: int, settings: dict,
               sec: float = 0.0, default_sec: float = 0.0) -> None:
    """Writes settings as the line of that graph's class into the table at
    path (nucleus34_tune_store; host only)."""
    t = Tune.from_dict(settings)
    _check(lib().nucleus34_tune_store(os.fsencode(path), triangles, n, m, max_out, C.byref(t), sec, default_sec),
           "tune_store")


def decompose(g: HostGraph, variant="direct", device: int = 0, mem_budget_bytes: int = 0,
              n_quds: int = 5, kfile: Optional[str] = None, flags: int = 0,
              tune_table: Optional[str] = None) -> Decomposition:
    """One-shot decomposition through nucleus34_decompose[_ondemand]."""
    L = lib()
    v = _VARIANTS[variant]
    opts = make_opts(device, mem_budget_bytes, flags=flags, tune_table=tune_table)
    res = Result()
    h = C.c_void_p()
    csr = g.csr()
    fn = L.nucleus34_decompose if v == DIRECT else L.nucleus34_decompose_ondemand
    _check(fn(C.byref(csr), C.byref(opts), C.byref(res), C.byref(h)), "decompose")
    try:
        T = int(res.triangle_count)
        k = np.zeros(T, np.int32)
        tris = np.zeros(3 * T, np.uint32)
        _check(L.nucleus34_copy_k(h, k.ctypes.data_as(C.POINTER(C.c_int32)), _u32p(tris)), "copy_k")
        quds = None
        if v == DIRECT and n_quds:
            q = min(int(n_quds), int(res.four_clique_count))
            quds = np.zeros(4 * q, np.uint32)
            if q:
                _check(L.nucleus34_copy_quds(h, 0, q, _u32p(quds)), "copy_quds")
            quds = quds.reshape(-1, 4)
        if kfile:
            _check(L.nucleus34_write_kfile(h, os.fsencode(kfile)), "write_kfile")
        return Decomposition(res.as_dict(), k, tris.reshape(-1, 3), quds)
    finally:
        L.nucleus34_free(h)


class Batch:
    """Results of nucleus34_batch_decompose: one shared device pass over many graphs."""

    def __init__(self, handle: C.c_void_p, result: dict, count: int):
        self._L = lib()
        self._h = handle
        self.result = result
        self.count = count

    def summary(self, i: int) -> dict:
        s = GraphSummary()
        _check(self._L.nucleus34_batch_summary(self._h, i, C.byref(s)), "batch_summary")
        return s.as_dict()

    def copy_k(self, i: int, with_tris: bool = False):
        T = self.summary(i)["triangle_count"]
        k = np.zeros(T, np.int32)
        tris = np.zeros(3 * T, np.uint32) if with_tris else None
        _check(self._L.nucleus34_batch_copy_k(self._h, i, k.ctypes.data_as(C.POINTER(C.c_int32)),
                                              _u32p(tris) if tris is not None else None), "batch_copy_k")
        return (k, tris.reshape(-1, 3)) if with_tris else k

    def close(self) -> None:
        if self._h:
            self._L.nucleus34_batch_free(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_decompose(graphs, device: int = 0, mem_budget_bytes: int = 0, flags: int = 0) -> Batch:
    """Decomposes a list of HostGraph in one device pass (nucleus34_batch_decompose)."""
    L = lib()
    arr = (Csr * len(graphs))(*[g.csr() for g in graphs])
    opts = make_opts(device, mem_budget_bytes, flags=flags)
    res = BatchResult()
    h = C.c_void_p()
    _check(L.nucleus34_batch_decompose(arr, len(graphs), C.byref(opts), C.byref(res), C.byref(h)), "batch_decompose")
    return Batch(h, res.as_dict(), len(graphs))


REQ_CLIQUES = 0x1
REQ_TRIANGLES = 0x2
ROUTE_MEMORY = 0
ROUTE_ONDEMAND = 1


class DeviceBatch:
    """Graphs split over several devices (replicas, no collective): each
    device decomposes its share as one nucleus34_batch_decompose, all shares
    at once on host threads (the C calls release the GIL). Results are read
    by global graph index, like a Batch."""

    def __init__(self, parts, where, result):
        self._parts, self._where, self.result = parts, where, result

    def summary(self, i: int) -> dict:
        p, j = self._where[i]
        return self._parts[p].summary(j)

    def copy_k(self, i: int, with_tris: bool = False):
        p, j = self._where[i]
        return self._parts[p].copy_k(j, with_tris)

    def close(self) -> None:
        for b in self._parts:
            if b is not None:
                b.close()
        self._parts = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def batch_decompose_devices(graphs, devices, mem_budget_bytes: int = 0, flags: int = 0) -> DeviceBatch:
    """The batched form over several devices: nucleus34_split_plan assigns
    each graph to one device by estimated cost, every device runs its share
    as a batch, and results stay addressed by the caller's graph index. A
    device may appear more than once (several shares on one GPU)."""
    import threading
    devices = list(devices)
    part_of, load = split_plan([graph_cost(g) for g in graphs], len(devices))
    shares = [[i for i in range(len(graphs)) if part_of[i] == p] for p in range(len(devices))]
    parts = [None] * len(devices)
    errors = [None] * len(devices)

    def run(p):
        try:
            if shares[p]:
                parts[p] = batch_decompose([graphs[i] for i in shares[p]], device=devices[p],
                                           mem_budget_bytes=mem_budget_bytes, flags=flags)
        except BaseException as e:  # reported below, after every share has ended
            errors[p] = e

    threads = [threading.Thread(target=run, args=(p,)) for p in range(len(devices))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for e in errors:
        if e is not None:
            for b in parts:
                if b is not None:
                    b.close()
            raise e
    where = {}
    for p, idx in enumerate(shares):
        for j, i in enumerate(idx):
            where[i] = (p, j)
    res = {"devices": devices, "share_graphs": [len(x) for x in shares], "share_cost": [int(x) for x in load],
           "shares": [b.result if b is not None else None for b in parts]}
    return DeviceBatch(parts, where, res)


class Server:
    """nucleus34_server_*: continuous batching of decomposition requests."""

    def __init__(self, device: int = 0, mem_budget_bytes: int = 0, workers: int = 3, max_batch_graphs: int = 256,
                 flags: int = 0, route: int = ROUTE_MEMORY, direct_div: int = 0, devices=None,
                 concurrent_runs: int = 0):
        """workers: concurrent passes per device slot; devices: slot ordinals
        (one may repeat), mem_budget_bytes applies to each slot; route and
        direct_div: the variant chosen per request by its memory estimate;
        concurrent_runs: decompositions running at once per slot (0: no
        limit)."""
        self._L = lib()
        opts = make_opts(device, mem_budget_bytes, flags=flags)
        self._devs = (C.c_int * len(devices))(*devices) if devices else None
        so = ServerOpts(workers, max_batch_graphs, route, direct_div, len(devices) if devices else 0,
                        C.cast(self._devs, C.POINTER(C.c_int)) if devices else None, concurrent_runs)
        self._h = C.c_void_p()
        _check(self._L.nucleus34_server_create(C.byref(opts), C.byref(so), C.byref(self._h)), "server_create")

    def submit(self, g: HostGraph, cliques: bool = False, triangles: bool = False) -> int:
        rid = C.c_uint64()
        csr = g.csr()
        flags = (REQ_CLIQUES if cliques else 0) | (REQ_TRIANGLES if triangles else 0)
        _check(self._L.nucleus34_server_submit(self._h, C.byref(csr), flags, C.byref(rid)), "server_submit")
        return int(rid.value)

    def wait(self, rid: int, timeout_ms: int = -1) -> dict:
        info = RequestInfo()
        _check(self._L.nucleus34_server_wait(self._h, rid, timeout_ms, C.byref(info)), "server_wait")
        return info.as_dict()

    def copy_k(self, rid: int, T: int, with_tris: bool = False):
        k = np.zeros(T, np.int32)
        tris = np.zeros(3 * T, np.uint32) if with_tris else None
        _check(self._L.nucleus34_server_copy_k(self._h, rid, k.ctypes.data_as(C.POINTER(C.c_int32)),
                                               _u32p(tris) if tris is not None else None), "server_copy_k")
        return (k, tris.reshape(-1, 3)) if with_tris else k

    def copy_quds(self, rid: int, first: int, count: int) -> np.ndarray:
        q = np.zeros(4 * count, np.uint32)
        _check(self._L.nucleus34_server_copy_quds(self._h, rid, first, count, _u32p(q)), "server_copy_quds")
        return q.reshape(-1, 4)

    def release(self, rid: int) -> None:
        _check(self._L.nucleus34_server_release(self._h, rid), "server_release")

    def stats(self) -> dict:
        c = ServerCounters()
        _check(self._L.nucleus34_server_stats(self._h, C.byref(c)), "server_stats")
        return c.as_dict()

    def close(self) -> None:
        if self._h:
            self._L.nucleus34_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """Device-resident context: upload once, run many times."""

    def __init__(self, device: int = 0, mem_budget_bytes: int = 0, flags: int = 0,
                 tune_table: Optional[str] = None):
        self._L = lib()
        self._opts = make_opts(device, mem_budget_bytes, flags=flags, tune_table=tune_table)
        self._h = C.c_void_p()
        self._nm = (0, 0)  # (n, m) of the resident graph
        _check(self._L.nucleus34_ctx_create(C.byref(self._opts), C.byref(self._h)), "ctx_create")

    def upload(self, g: HostGraph) -> None:
        csr = g.csr()
        _check(self._L.nucleus34_ctx_upload(self._h, C.byref(csr)), "ctx_upload")
        self._nm = (int(g.n), int(g.m))

    def upload_edges(self, src: np.ndarray, dst: np.ndarray) -> tuple:
        """nucleus34_ctx_upload_edges: the oriented CSR of an edge list built on
        the device (graph_from_edges semantics); returns (n, m)."""
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        if len(src) != len(dst):
            raise ValueError("src and dst differ in length")
        n, m = C.c_uint64(), C.c_uint64()
        _check(self._L.nucleus34_ctx_upload_edges(self._h, _u32p(src), _u32p(dst), len(src), C.byref(n),
                                                  C.byref(m)), "ctx_upload_edges")
        self._nm = (int(n.value), int(m.value))
        return self._nm

    def copy_csr(self) -> "HostGraph":
        """The resident oriented CSR (nucleus34_ctx_copy_csr) as a HostGraph."""
        n, m = self._nm
        O = np.zeros(n + 1, np.uint32)
        D = np.zeros(n, np.uint32)
        E = np.zeros(m, np.uint32)
        _check(self._L.nucleus34_ctx_copy_csr(self._h, _u32p(O), _u32p(D), _u32p(E)), "ctx_copy_csr")
        return HostGraph(n, m, O, D, E)

    def run(self, variant="ondemand") -> dict:
        res = Result()
        _check(self._L.nucleus34_ctx_run(self._h, _VARIANTS[variant], C.byref(res)), "ctx_run")
        self._last = res.as_dict()
        return self._last

    def copy_k(self, T: int, with_tris: bool = False):
        k = np.zeros(T, np.int32)
        tris = np.zeros(3 * T, np.uint32) if with_tris else None
        _check(self._L.nucleus34_ctx_copy_k(
            self._h, k.ctypes.data_as(C.POINTER(C.c_int32)),
            _u32p(tris) if tris is not None else None), "ctx_copy_k")
        return (k, tris.reshape(-1, 3)) if with_tris else k

    def set_tune(self, settings: Optional[dict]) -> None:
        """Pins the on-demand settings of later runs (None: back to the table / defaults)."""
        t = Tune.from_dict(settings) if settings is not None else None
        _check(self._L.nucleus34_ctx_set_tune(self._h, C.byref(t) if t is not None else None), "ctx_set_tune")

    def last_tune(self) -> dict:
        t = Tune()
        _check(self._L.nucleus34_ctx_last_tune(self._h, C.byref(t)), "ctx_last_tune")
        return t.as_dict()

    def autotune(self, table: Optional[str] = None) -> dict:
        """nucleus34_ctx_autotune on the uploaded graph: the best settings and
        the device times (s) of the default and the tuned decomposition."""
        t, best, default = Tune(), C.c_double(), C.c_double()
        _check(self._L.nucleus34_ctx_autotune(self._h, os.fsencode(table) if table else None, C.byref(t),
                                              C.byref(best), C.byref(default)), "ctx_autotune")
        return {"tune": t.as_dict(), "tuned_sec": best.value, "default_sec": default.value}

    def verify(self) -> tuple:
        """(violations, checked) of nucleus34_ctx_verify for the last run."""
        v, n = C.c_uint64(), C.c_uint64()
        _check(self._L.nucleus34_ctx_verify(self._h, C.byref(v), C.byref(n)), "ctx_verify")
        return int(v.value), int(n.value)

    def close(self) -> None:
        if self._h:
            self._L.nucleus34_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
