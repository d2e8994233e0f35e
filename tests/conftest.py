"""Shared test set-up: markers, import paths and the parity norms."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def rel_maxnorm(a, b):
    """max|a - b| / max|b|: the parity norm (1e-5 bar for FP32 vs the reference)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


@pytest.fixture(scope="session")
def gpu_ok():
    """Skip-free guard: GPU tests fail loudly if the library or device is missing."""
    import freelb_b200  # noqa: F401  (raises ImportError if the .so is missing)
    from freelb_b200 import _capi
    _capi.load()
    return True
