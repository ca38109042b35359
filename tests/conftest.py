"""Shared fixtures.  `-m gpu` tests need a CUDA device; everything else runs on CPU.

The checkers (oracle/liboracle.so, our CPU restatement, and oracle/_ref/libref.so,
the reference's own C compiled unchanged) are test infrastructure: they are
loaded here only to compare against the engine.
"""
from __future__ import annotations

import importlib
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def _ensure_built():
    lib = os.path.join(ROOT, "3d_fdtd_b200", "lib", "libfdtd_b200.so")
    if not os.path.exists(lib):
        subprocess.run([sys.executable, os.path.join(ROOT, "3d_fdtd_b200", "build.py")], check=True)
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)


_ensure_built()


@pytest.fixture(scope="session")
def fd():
    return importlib.import_module("3d_fdtd_b200")


@pytest.fixture(scope="session")
def orc():
    from bindings import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from bindings import REF_SO, Reference
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref/libref.so not built (needs the reference sources: make -C oracle ref)")
    return Reference()


@pytest.fixture(scope="session")
def gpu(fd):
    if fd.lib.fdtd_device_count() <= 0:
        fd.lib.fdtd_clear_error()
        pytest.skip("no CUDA device")
    return True


@pytest.fixture(autouse=True)
def _clear_errors(fd):
    fd.lib.fdtd_clear_error()
    yield
