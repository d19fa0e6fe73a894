"""Shared test setup.

Markers: `gpu` tests need a B200 and the built library; the rest run on CPU.
The plain-C oracle (oracle/_ref/libndgoracle.so) is built here if missing;
the reference checker (oracle/_ref/libndgref.so) exists only where the
reference sources were available when oracle/Makefile ran, so tests that use
it skip without it.
"""
from __future__ import annotations

import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a) and ndg_cuda_b200/libndg_b200.so")


def _ensure_oracle():
    lib = os.path.join(ROOT, "oracle", "_ref", "libndgoracle.so")
    src = os.path.join(ROOT, "oracle", "ndg_oracle.c")
    if not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "restatement"], check=True)


_ensure_oracle()


@pytest.fixture(scope="session")
def ref_available():
    from oracle import pyoracle
    if not pyoracle.ref_available():
        pytest.skip("reference checker oracle/_ref/libndgref.so not built here")
    return True
