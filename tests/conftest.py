"""Shared test setup.

Markers: ``gpu`` tests need an sm_100 device and call the CUDA library through
its C ABI; everything else runs on the CPU (oracle vs golden vectors, host
logic, the library's exported surface).
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (os.path.join(ROOT, "hyper-vlasov_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) device")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def golden():
    cache = {}

    def load(name):
        if name not in cache:
            with np.load(os.path.join(GOLDEN, name)) as f:
                cache[name] = {k: f[k] for k in f.files}
        return cache[name]

    return load


@pytest.fixture(scope="session")
def hv():
    import hv_b200

    hv_b200.load()
    return hv_b200


def world_of(g):
    return (tuple(int(v) for v in g["n"]), tuple(float(v) for v in g["d_max"]))


def max_rel(a, b):
    """max|a - b| / max|b| (0 when both are zero)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.max(np.abs(b)) if b.size else 0.0
    num = np.max(np.abs(a - b)) if b.size else 0.0
    return 0.0 if num == 0.0 else num / (den if den > 0 else 1.0)
