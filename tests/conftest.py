"""Shared test setup: the ``gpu`` marker, import paths and small helpers.

``-m "not gpu"`` runs on a machine without a GPU: the oracle against the golden
fixtures and against the reference (when it was compiled here), host-side
logic, and the C-ABI export table.  ``-m gpu`` runs the CUDA path against the
oracle through the C ABI.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "smdlt-ca-chrg-flow_b200")
for p in (os.path.join(ROOT, "oracle"), PKG, ROOT, os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")


def rel_err(a, b):
    """Norm-wise relative error ||a - b|| / ||b|| (0 when both vanish)."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    nb = np.linalg.norm(b)
    na = np.linalg.norm(a - b)
    return 0.0 if nb == 0 and na == 0 else na / max(nb, 1e-300)


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))
    return load
