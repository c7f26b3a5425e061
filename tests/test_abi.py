"""The C-ABI library loads and exports every entry point include/nucleus34.h
declares (no compute call: these run without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "nucleus34.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nucleus34_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_drop_in_entry_points():
    names = declared_functions()
    for fn in ("nucleus34_decompose", "nucleus34_decompose_ondemand", "nucleus34_copy_k",
               "nucleus34_free", "nucleus34_strerror"):
        assert fn in names


def test_library_exports_every_declared_symbol(n34):
    lib = ctypes.CDLL(n34.LIB_PATH)
    missing = [f for f in declared_functions() if not hasattr(lib, f)]
    assert not missing, missing
    assert set(n34.EXPORTED) <= set(declared_functions())


def test_strerror_and_no_device_error(n34):
    assert n34.strerror(0) == "success"
    assert "budget" in n34.strerror(n34.E_OOM_BUDGET)


def test_null_arguments_are_rejected(n34):
    L = n34.lib()
    assert L.nucleus34_decompose(None, None, None, None) == n34.E_INVALID
    assert L.nucleus34_copy_k(None, None, None) == n34.E_INVALID
    L.nucleus34_free(None)


def test_every_handle_entry_point_rejects_null_arguments(n34):
    """No entry point dereferences a null handle or output: each returns
    E_INVALID (the destroy/free calls accept null and do nothing)."""
    L = n34.lib()
    E = n34.E_INVALID
    calls = {
        "copy_quds": lambda: L.nucleus34_copy_quds(None, 0, 1, None),
        "write_kfile": lambda: L.nucleus34_write_kfile(None, b"/tmp/unused"),
        "ctx_create": lambda: L.nucleus34_ctx_create(None, None),
        "ctx_upload": lambda: L.nucleus34_ctx_upload(None, None),
        "ctx_run": lambda: L.nucleus34_ctx_run(None, n34.ONDEMAND, None),
        "ctx_copy_k": lambda: L.nucleus34_ctx_copy_k(None, None, None),
        "ctx_verify": lambda: L.nucleus34_ctx_verify(None, None, None),
        "ctx_set_tune": lambda: L.nucleus34_ctx_set_tune(None, None),
        "ctx_last_tune": lambda: L.nucleus34_ctx_last_tune(None, None),
        "ctx_autotune": lambda: L.nucleus34_ctx_autotune(None, None, None, None, None),
        "ctx_upload_edges": lambda: L.nucleus34_ctx_upload_edges(None, None, None, 0, None, None),
        "ctx_copy_csr": lambda: L.nucleus34_ctx_copy_csr(None, None, None, None),
        "tune_lookup": lambda: L.nucleus34_tune_lookup(b"/tmp/unused", 0, 0, 0, 0, None, None),
        "tune_store": lambda: L.nucleus34_tune_store(b"/tmp/unused", 0, 0, 0, 0, None, 0.0, 0.0),
        "batch_decompose": lambda: L.nucleus34_batch_decompose(None, 1, None, None, None),
        "batch_summary": lambda: L.nucleus34_batch_summary(None, 0, None),
        "batch_copy_k": lambda: L.nucleus34_batch_copy_k(None, 0, None, None),
        "server_create": lambda: L.nucleus34_server_create(None, None, None),
        "server_submit": lambda: L.nucleus34_server_submit(None, None, 0, None),
        "server_wait": lambda: L.nucleus34_server_wait(None, 1, 0, None),
        "server_copy_k": lambda: L.nucleus34_server_copy_k(None, 1, None, None),
        "server_copy_quds": lambda: L.nucleus34_server_copy_quds(None, 1, 0, 1, None),
        "server_release": lambda: L.nucleus34_server_release(None, 1),
        "server_stats": lambda: L.nucleus34_server_stats(None, None),
        "graph_load": lambda: L.nucleus34_graph_load(None, None),
        "graph_from_edges": lambda: L.nucleus34_graph_from_edges(None, None, 1, None),
        "graph_save_grh": lambda: L.nucleus34_graph_save_grh(None, b"/tmp/unused.grh"),
        "edges_write": lambda: L.nucleus34_edges_write(None, b"/tmp/unused.edges"),
    }
    bad = {name: rc for name, rc in ((n, f()) for n, f in calls.items()) if rc != E}
    assert not bad, bad
    for fn in ("nucleus34_ctx_destroy", "nucleus34_batch_free", "nucleus34_server_destroy",
               "nucleus34_graph_release", "nucleus34_edges_release"):
        getattr(L, fn)(None)


def test_missing_device_is_reported_not_worked_around(n34):
    """Without a CUDA device the decomposition fails with E_NODEVICE: there
    is no CPU fallback behind the C-ABI (skipped where a device exists)."""
    import ctypes as C
    L = n34.lib()
    h = C.c_void_p()
    if L.nucleus34_ctx_create(None, C.byref(h)) != n34.E_NODEVICE:
        if h:
            L.nucleus34_ctx_destroy(h)
        pytest.skip("a CUDA device is present")
    assert "no CUDA device" in n34.last_error()
    s, d = n34.gen_rmat(6, 8, 1)
    g = n34.graph_from_edges(s, d)
    for variant in ("direct", "ondemand"):
        with pytest.raises(n34.Nucleus34Error) as e:
            n34.decompose(g, variant=variant)
        assert e.value.code == n34.E_NODEVICE
