"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, and only as the checker / the timed CPU baseline. The product
path (libnucleus34) never loads the oracle.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
CLI_PATH = os.path.join(HERE, "_build", "nucleus34_oracle")
REF_DIR = os.path.join(HERE, "_ref")
REF_CPU = os.path.join(REF_DIR, "cpu_ref")
REF_DIRECT = os.path.join(REF_DIR, "cuNucleus34")
REF_ONDEMAND = os.path.join(REF_DIR, "cuNucleus34_ondemand")


class OGraph(C.Structure):
    _fields_ = [("n", C.c_uint64), ("m", C.c_uint64), ("O", C.POINTER(C.c_uint32)),
                ("D", C.POINTER(C.c_uint32)), ("E", C.POINTER(C.c_uint32))]


class OResult(C.Structure):
    _fields_ = [("T", C.c_uint64), ("Q", C.c_uint64), ("k_max", C.c_int32), ("k_avg", C.c_double),
                ("tris", C.POINTER(C.c_uint32)), ("support", C.POINTER(C.c_int32)),
                ("k", C.POINTER(C.c_int32)), ("quds", C.POINTER(C.c_uint32)),
                ("quds_len", C.c_uint64)]


_LIB = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        u32p = C.POINTER(C.c_uint32)
        L.oracle_read_graph.argtypes = [C.c_char_p, C.POINTER(OGraph)]
        L.oracle_graph_from_pairs.argtypes = [u32p, u32p, C.c_uint64, C.POINTER(OGraph)]
        L.oracle_graph_from_oriented.argtypes = [C.c_uint64, C.c_uint64, u32p, u32p, C.POINTER(OGraph)]
        L.oracle_graph_free.argtypes = [C.POINTER(OGraph)]
        L.oracle_graph_free.restype = None
        L.oracle_decompose.argtypes = [C.POINTER(OGraph), C.c_uint64, C.POINTER(OResult)]
        L.oracle_result_free.argtypes = [C.POINTER(OResult)]
        L.oracle_result_free.restype = None
        L.oracle_count_triangles.argtypes = [C.POINTER(OGraph)]
        L.oracle_count_triangles.restype = C.c_uint64
        L.oracle_count_k4.argtypes = [C.POINTER(OGraph)]
        L.oracle_count_k4.restype = C.c_uint64
        L.oracle_peel_rounds.argtypes = [C.POINTER(OGraph), u32p, C.c_uint64, C.POINTER(C.c_int32), u32p]
        L.oracle_peel_rounds.restype = C.c_int
        L.oracle_certify.argtypes = [C.POINTER(OGraph), u32p, C.c_uint64, C.POINTER(C.c_int32), u32p]
        L.oracle_certify.restype = C.c_int64
        _LIB = L
    return _LIB


@dataclass
class OracleGraph:
    n: int
    m: int
    O: np.ndarray
    D: np.ndarray
    E: np.ndarray


@dataclass
class OracleResult:
    T: int
    Q: int
    k_max: int
    k_avg: float
    tris: np.ndarray
    support: np.ndarray
    k: np.ndarray
    quds: np.ndarray


def _take_graph(g: OGraph) -> OracleGraph:
    n, m = int(g.n), int(g.m)
    O = np.ctypeslib.as_array(g.O, shape=(n + 1,)).copy()
    D = np.ctypeslib.as_array(g.D, shape=(n,)).copy() if n else np.zeros(0, np.uint32)
    E = np.ctypeslib.as_array(g.E, shape=(m,)).copy() if m else np.zeros(0, np.uint32)
    lib().oracle_graph_free(C.byref(g))
    return OracleGraph(n, m, O, D, E)


def read_graph(path: str) -> OracleGraph:
    g = OGraph()
    rc = lib().oracle_read_graph(os.fsencode(path), C.byref(g))
    if rc:
        raise RuntimeError(f"oracle_read_graph({path}) = {rc}")
    return _take_graph(g)


def graph_from_pairs(src, dst) -> OracleGraph:
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    g = OGraph()
    rc = lib().oracle_graph_from_pairs(src.ctypes.data_as(C.POINTER(C.c_uint32)),
                                       dst.ctypes.data_as(C.POINTER(C.c_uint32)), len(src), C.byref(g))
    if rc:
        raise RuntimeError(f"oracle_graph_from_pairs = {rc}")
    return _take_graph(g)


def decompose(g, quds_cap: int = 5) -> OracleResult:
    """g: anything with n, m, D, E (oriented CSR)."""
    D = np.ascontiguousarray(g.D, np.uint32)
    E = np.ascontiguousarray(g.E, np.uint32)
    og = OGraph()
    L = lib()
    rc = L.oracle_graph_from_oriented(int(g.n), int(g.m), D.ctypes.data_as(C.POINTER(C.c_uint32)),
                                      E.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(og))
    if rc:
        raise RuntimeError(f"oracle_graph_from_oriented = {rc}")
    r = OResult()
    try:
        rc = L.oracle_decompose(C.byref(og), quds_cap, C.byref(r))
        if rc:
            raise RuntimeError(f"oracle_decompose = {rc}")
        T = int(r.T)
        tris = np.ctypeslib.as_array(r.tris, shape=(3 * T,)).copy().reshape(-1, 3) if T else np.zeros((0, 3), np.uint32)
        sup = np.ctypeslib.as_array(r.support, shape=(T,)).copy() if T else np.zeros(0, np.int32)
        k = np.ctypeslib.as_array(r.k, shape=(T,)).copy() if T else np.zeros(0, np.int32)
        ql = int(r.quds_len)
        quds = np.ctypeslib.as_array(r.quds, shape=(4 * ql,)).copy().reshape(-1, 4) if ql else np.zeros((0, 4), np.uint32)
        return OracleResult(T, int(r.Q), int(r.k_max), float(r.k_avg), tris, sup, k, quds)
    finally:
        L.oracle_result_free(C.byref(r))
        L.oracle_graph_free(C.byref(og))


def kfile_bytes(tris: np.ndarray, k: np.ndarray) -> bytes:
    """Rows "(a,b,c)\\t<k>\\n" as the programs write them."""
    lines = [f"({a},{b},{c})\t{kk}\n" for (a, b, c), kk in zip(tris.tolist(), k.tolist())]
    return "".join(lines).encode()


def count_k4(g) -> int:
    """Four-cliques of the oriented CSR g, counted by oriented neighbourhoods
    (independent of the incidence-based support count)."""
    D = np.ascontiguousarray(g.D, np.uint32)
    E = np.ascontiguousarray(g.E if g.m else np.zeros(1, np.uint32), np.uint32)
    og = OGraph()
    L = lib()
    rc = L.oracle_graph_from_oriented(int(g.n), int(g.m), D.ctypes.data_as(C.POINTER(C.c_uint32)),
                                      E.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(og))
    if rc:
        raise RuntimeError(f"oracle_graph_from_oriented = {rc}")
    try:
        return int(L.oracle_count_k4(C.byref(og)))
    finally:
        L.oracle_graph_free(C.byref(og))


def _oriented(g):
    D = np.ascontiguousarray(g.D, np.uint32)
    E = np.ascontiguousarray(g.E if g.m else np.zeros(1, np.uint32), np.uint32)
    og = OGraph()
    rc = lib().oracle_graph_from_oriented(int(g.n), int(g.m), D.ctypes.data_as(C.POINTER(C.c_uint32)),
                                          E.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(og))
    if rc:
        raise RuntimeError(f"oracle_graph_from_oriented = {rc}")
    return og


def peel_rounds(g, tris: np.ndarray):
    """Level-synchronous peel (the device peel's rules) on the canonical
    triangle list: (k, death round) per triangle."""
    T = len(tris)
    t3 = np.ascontiguousarray(tris, np.uint32).reshape(-1)
    k = np.zeros(max(T, 1), np.int32)
    r = np.zeros(max(T, 1), np.uint32)
    og = _oriented(g)
    try:
        rc = lib().oracle_peel_rounds(C.byref(og), t3.ctypes.data_as(C.POINTER(C.c_uint32)), T,
                                      k.ctypes.data_as(C.POINTER(C.c_int32)), r.ctypes.data_as(C.POINTER(C.c_uint32)))
        if rc:
            raise RuntimeError(f"oracle_peel_rounds = {rc}")
    finally:
        lib().oracle_graph_free(C.byref(og))
    return k[:T], r[:T]


def certify(g, tris: np.ndarray, k: np.ndarray, rounds: np.ndarray) -> int:
    """Number of triangles (and rounds) failing the certificate conditions."""
    T = len(tris)
    t3 = np.ascontiguousarray(tris, np.uint32).reshape(-1)
    kk = np.ascontiguousarray(k, np.int32)
    rr = np.ascontiguousarray(rounds, np.uint32)
    og = _oriented(g)
    try:
        v = lib().oracle_certify(C.byref(og), t3.ctypes.data_as(C.POINTER(C.c_uint32)), T,
                                 kk.ctypes.data_as(C.POINTER(C.c_int32)), rr.ctypes.data_as(C.POINTER(C.c_uint32)))
    finally:
        lib().oracle_graph_free(C.byref(og))
    if v < 0:
        raise RuntimeError(f"oracle_certify = {v}")
    return int(v)
