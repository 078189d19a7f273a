import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a)")


def load_goldens():
    z = np.load(os.path.join(GOLDEN, "gse_goldens.npz"))
    cases = {}
    for k in z.files:
        name, field = k.split("/")
        cases.setdefault(name, {})[field] = z[k]
    return cases


@pytest.fixture(scope="session")
def goldens():
    return load_goldens()


def load_grid_goldens():
    """Cases of tests/golden/grid_ops_goldens.npz (make_grid_ops_goldens.py)."""
    z = np.load(os.path.join(GOLDEN, "grid_ops_goldens.npz"))
    cases = {}
    for k in z.files:
        name, field = k.split("/")
        cases.setdefault(name, {})[field] = z[k]
    return cases


@pytest.fixture(scope="session")
def grid_goldens():
    return load_grid_goldens()


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build(with_reference=os.path.isdir("/root/reference"))
    return oracle
