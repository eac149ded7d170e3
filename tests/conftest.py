"""Test configuration: the ``gpu`` marker and shared fixtures.

``-m "not gpu"`` runs on any machine (oracle against the golden fixtures,
host logic, library loading); ``-m gpu`` runs the CUDA engine against the
oracle on a B200.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)

ELECTRON_REST = 510998.95069


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(os.path.join(GOLDEN, name))
    return load


@pytest.fixture
def rin():
    return np.array(np.zeros((6, 1)), order="F")


def scale_rel_diff(a, b):
    """max |a-b| per coordinate, divided by that coordinate's max |b|
    (rows where both are finite)."""
    a = np.asarray(a).reshape(6, -1)
    b = np.asarray(b).reshape(6, -1)
    ok = np.all(np.isfinite(a), axis=0) & np.all(np.isfinite(b), axis=0)
    if not ok.any():
        return 0.0
    d = np.abs(a[:, ok] - b[:, ok]).max(axis=1)
    s = np.abs(b[:, ok]).max(axis=1)
    s[s == 0] = 1.0
    return float((d / s).max())
