"""Shared test setup: import paths, build-on-demand of the in-tree libraries,
the `gpu` marker and small graph fixtures."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gpu-nucleus34_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_built():
    lib = os.path.join(PKG, "lib", "libnucleus34.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", PKG, "-j8"], check=True)
    olib = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
    if not os.path.exists(olib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)


_ensure_built()


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def n34():
    import nucleus34
    nucleus34.lib()
    return nucleus34


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.lib()
    return o
