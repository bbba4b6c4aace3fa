import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def golden():
    return np.load(os.path.join(ROOT, "tests", "golden", "ldl_cases.npz"))


def backward_error(system, x, b):
    """||b - K x||_inf / (||K||_inf ||x||_inf + ||b||_inf), column-wise max."""
    r = b - system.matvec(x)
    kn = system.inf_norm()
    x2 = x.reshape(system.n, -1)
    b2 = b.reshape(system.n, -1)
    r2 = r.reshape(system.n, -1)
    num = np.abs(r2).max(axis=0)
    den = kn * np.abs(x2).max(axis=0) + np.abs(b2).max(axis=0)
    return float(np.max(num / den))
