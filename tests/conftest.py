"""Shared fixtures for the test suite.

Markers:
  gpu   -- needs a CUDA device (runs the CUDA library); everything else runs
           on the CPU (oracle vs reference, golden fixtures, C-ABI exports,
           loaders, host-side plan logic, multi-process gloo tests).
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA device")


def _has_gpu() -> bool:
    try:
        import dynasor_plus_b200 as d
        return d.device_count() > 0
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def bindings():
    from oracle import bindings as B
    if not B.oracle_available():
        pytest.skip("oracle/liboracle.so not built (run __graft_entry__.build())")
    return B


@pytest.fixture(scope="session")
def refb(bindings):
    if not bindings.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference tree at build time)")
    return bindings


def load_golden(name):
    path = os.path.join(GOLDEN, name)
    with np.load(path, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def rel_fro(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
