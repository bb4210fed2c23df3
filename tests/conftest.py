import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "multigrid-fvm_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200)")


def interior(a):
    return a[1:-1, 1:-1]


def assert_bitexact(a, b, what=""):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, f"{what}: shape {a.shape} vs {b.shape}"
    if not np.array_equal(a, b):
        bad = np.argwhere(a != b)
        k = tuple(bad[0])
        raise AssertionError(f"{what}: {len(bad)} entries differ, first at {k}: {a[k]!r} vs {b[k]!r}, "
                             f"max |diff| {np.nanmax(np.abs(a - b)):.3e}")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


@pytest.fixture(scope="session")
def oracle_built():
    import oracle
    if not os.path.exists(oracle.ORACLE_SO):
        oracle.build()
    return oracle
