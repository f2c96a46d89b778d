import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def golden():
    return np.load(os.path.join(GOLDEN, "ref_kernels.npz"))


@pytest.fixture(scope="session")
def native():
    """The product library, built for sm_100a (fails loudly if it cannot be built)."""
    from colvillea_b200 import build, _native
    build.build()
    return _native


def ulp_diff(a, b):
    """Distance in units in the last place between float32 arrays (NaN==NaN is 0)."""
    a = np.ascontiguousarray(a, np.float32).ravel()
    b = np.ascontiguousarray(b, np.float32).ravel()
    ai = a.view(np.int32).astype(np.int64)
    bi = b.view(np.int32).astype(np.int64)
    ai = np.where(ai < 0, -(2 ** 31) - ai, ai)
    bi = np.where(bi < 0, -(2 ** 31) - bi, bi)
    d = np.abs(ai - bi)
    d[np.isnan(a) & np.isnan(b)] = 0
    return d
