"""Shared pytest setup.

Markers: `gpu` — needs a B200 (sm_100) device; everything else runs on the CPU.
Paths: the repository root (bench.py, __graft_entry__.py), the package directory
(``import ipg``) and ``oracle/`` (``import oracle``, the CPU checker; only tests use it).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "interatomicpotentials.jl_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 (B200) device")


@pytest.fixture(scope="session")
def golden():
    """Fixtures generated by tests/golden/make_golden.py from the reference's test files."""
    return np.load(os.path.join(GOLDEN, "reference_fixtures.npz"), allow_pickle=False)


@pytest.fixture(scope="session")
def ctx():
    import ipg
    return ipg.default_context()


def rel_err(a, b):
    """max|a - b| / max|b| (the tolerance measure for arrays)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b)) if b.size else 0.0
    num = np.max(np.abs(a - b)) if a.size else 0.0
    return num / den if den > 0 else num


# FP64 parity bound with the reference algorithm (relative, per array).
TOL = 1e-10
