import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the product kernels")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(os.path.join(GOLDEN, name), allow_pickle=False)
    return load


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    oracle.set_threads(os.cpu_count() or 1)
    return oracle


@pytest.fixture(scope="session")
def plib():
    from nufht_b200 import _lib
    return _lib.lib()


@pytest.fixture(scope="session")
def cuda():
    if not gpu_available():
        pytest.fail("GPU test run without a CUDA device")
    import torch
    torch.cuda.init()
    return torch.device("cuda", 0)


def grids(kind, m, n, seed):
    sys.path.insert(0, GOLDEN)
    from make_golden import grids as g
    return g(kind, m, n, seed)


def col_err(a, b, c):
    """max_i |a[i,t] - b[i,t]| / ||c[:,t]||_1, per column t."""
    a = np.asarray(a).reshape(a.shape[0], -1)
    b = np.asarray(b).reshape(b.shape[0], -1)
    c = np.asarray(c).reshape(c.shape[0], -1)
    return np.abs(a - b).max(axis=0) / np.abs(c).sum(axis=0)
