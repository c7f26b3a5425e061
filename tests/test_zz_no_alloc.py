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
