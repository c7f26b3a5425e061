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
