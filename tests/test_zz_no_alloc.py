"""Triangle listing without device allocation (nucleus34_list_triangles_noalloc).

This entry point is for callers that cannot allocate device memory while they
run: a service that reserves all of HBM up front and hands slices out itself,
a process whose framework allocator owns the device, or a latency-critical
loop where an allocation's cost or failure is not acceptable. They pass their
own device buffers (here: torch tensors) for the oriented CSR and the output,
and the library keeps its temporaries in a fixed static device array.

Checked against the existing entry point (nucleus34_decompose_ondemand +
nucleus34_copy_k, which lists triangles with library-allocated scratch), on
two calls in a row, bit for bit: the listing is integer work, so the tolerance
is exact equality. The file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_VERTICES = 1 << 20


def _entry(n34):
    f = n34.lib().nucleus34_list_triangles_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p, C.c_uint64,
                  C.POINTER(C.c_uint64), C.c_int, C.c_void_p]
    f.restype = C.c_int
    return f


def _device_csr(g):
    import torch
    dO = torch.from_numpy(g.O.astype(np.uint32).view(np.int32)).to("cuda:0")
    dE = torch.from_numpy((g.E if g.m else np.zeros(1, np.uint32)).astype(np.uint32).view(np.int32)).to("cuda:0")
    return dO, dE


@pytest.mark.parametrize("case", [("rmat", 12, 16, 1), ("rgg", 20000, 24.0, 3), ("rmat", 16, 16, 2)])
def test_noalloc_listing_matches_existing_entry_point(n34, case):
    import torch
    if case[0] == "rmat":
        s, d = n34.gen_rmat(case[1], case[2], case[3])
    else:
        s, d = n34.gen_rgg(case[1], case[2], case[3])
    g = n34.graph_from_edges(s, d)
    assert g.n <= MAX_VERTICES
    ref = n34.decompose(g, variant="ondemand", n_quds=0)  # existing entry point
    T = int(ref.result["triangle_count"])
    f = _entry(n34)
    dO, dE = _device_csr(g)
    out = torch.empty(3 * T + 3, dtype=torch.int32, device="cuda:0")
    for _call in range(2):
        out.fill_(-1)  # the scratch keeps the last call's contents; the output must not depend on it
        torch.cuda.synchronize()
        cnt = C.c_uint64(0)
        rc = f(dO.data_ptr(), dE.data_ptr(), g.n, g.m, out.data_ptr(), T + 1, C.byref(cnt), 0, None)
        assert rc == 0, n34.last_error()
        assert cnt.value == T
        got = out[: 3 * T].cpu().numpy().view(np.uint32).reshape(-1, 3)
        assert np.array_equal(got, ref.tris)
        assert np.all(out[3 * T:].cpu().numpy() == -1)  # nothing written past the triangles


def test_noalloc_count_only_and_capacity(n34):
    import torch
    s, d = n34.gen_rmat(10, 8, 7)
    g = n34.graph_from_edges(s, d)
    f = _entry(n34)
    dO, dE = _device_csr(g)
    cnt = C.c_uint64(0)
    assert f(dO.data_ptr(), dE.data_ptr(), g.n, g.m, None, 0, C.byref(cnt), 0, None) == 0
    T = cnt.value
    assert T == n34.decompose(g, variant="ondemand", n_quds=0).result["triangle_count"]
    small = torch.full((3 * max(T // 2, 1),), -1, dtype=torch.int32, device="cuda:0")
    rc = f(dO.data_ptr(), dE.data_ptr(), g.n, g.m, small.data_ptr(), T // 2, C.byref(cnt), 0, None)
    assert rc == n34.E_INVALID and cnt.value == T
    assert np.all(small.cpu().numpy() == -1)


def test_noalloc_rejects_graphs_beyond_its_scratch(n34):
    f = _entry(n34)
    cnt = C.c_uint64(7)
    rc = f(None, None, MAX_VERTICES + 1, 0, None, 0, C.byref(cnt), 0, None)
    assert rc == n34.E_INVALID
    assert "at most" in n34.last_error()
    assert cnt.value == 0


def test_noalloc_rejects_malformed_csr_and_writes_nothing(n34):
    """A CSR that breaks the input contract (O[n] != m, an unsorted list, an
    edge stored in both directions, a self-loop) is refused before anything
    is written, and the caller's current device is unchanged."""
    import torch
    s, d = n34.gen_rmat(9, 8, 3)
    g = n34.graph_from_edges(s, d)
    O = g.O[: g.n + 1].astype(np.uint32)
    E = g.E.astype(np.uint32)
    u = int(np.argmax(np.diff(O.astype(np.int64))))  # a vertex with at least two out-edges
    assert O[u + 1] - O[u] >= 2
    unsorted = E.copy()
    unsorted[O[u]], unsorted[O[u] + 1] = unsorted[O[u] + 1], unsorted[O[u]]
    loop = E.copy()
    loop[O[u]] = u
    # symmetric: every edge in both directions (a triangle would be listed several times)
    src = np.repeat(np.arange(g.n, dtype=np.uint32), np.diff(O.astype(np.int64)))
    both_s = np.concatenate([src, E])
    both_d = np.concatenate([E, src])
    order = np.lexsort((both_d, both_s))
    both_s, both_d = both_s[order], both_d[order]
    symO = np.zeros(g.n + 1, np.uint32)
    np.add.at(symO, both_s.astype(np.int64) + 1, 1)
    symO = np.cumsum(symO).astype(np.uint32)
    bad_m = O.copy()
    bad_m[-1] -= 1
    cases = {"O[n] != m": (bad_m, E, g.m), "unsorted list": (O, unsorted, g.m), "self-loop": (O, loop, g.m),
             "both directions": (symO, both_d, len(both_d))}
    f = _entry(n34)
    torch.cuda.set_device(0)
    for name, (o, e, m) in cases.items():
        dO = torch.from_numpy(o.view(np.int32).copy()).to("cuda:0")
        dE = torch.from_numpy(e.view(np.int32).copy()).to("cuda:0")
        out = torch.full((3 * 4096,), -1, dtype=torch.int32, device="cuda:0")
        cnt = C.c_uint64(123)
        rc = f(dO.data_ptr(), dE.data_ptr(), g.n, m, out.data_ptr(), 4096, C.byref(cnt), 0, None)
        assert rc == n34.E_INVALID, name
        assert "each undirected edge once" in n34.last_error(), name
        assert cnt.value == 0, name
        assert np.all(out.cpu().numpy() == -1), name
        assert torch.cuda.current_device() == 0
