import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden(name):
    return os.path.join(GOLDEN, name)


def rmse_close(v0, v1, tol):
    """rmse_comparison of the reference tests (testing/tests_general.hpp:70-88):
    ||v0 - v1||_2 / max(1, ||v0||_inf, ||v1||_inf) < tol * sqrt(N)."""
    v0 = np.asarray(v0, dtype=np.float64)
    v1 = np.asarray(v1, dtype=np.float64)
    diff = np.linalg.norm(v0 - v1)
    scale = max(1.0, np.abs(v0).max(initial=0), np.abs(v1).max(initial=0))
    return diff / scale < tol * np.sqrt(max(len(v0), 1))


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.fixture(scope="session")
def cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch.device("cuda:0")
