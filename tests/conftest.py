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


def load_ref48k():
    """The reference's own real-system case test48K (make_ref48k.py): the
    48,191-charge input as float64 [n, 4] and the reference's outputs."""
    import lzma
    with lzma.open(os.path.join(GOLDEN, "xyzq_48k.txt.xz"), "rt") as f:
        x = np.array([float(t) for t in f.read().split()], dtype=np.float64).reshape(-1, 4)
    z = np.load(os.path.join(GOLDEN, "ref48k.npz"))
    return x, {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def ref48k():
    return load_ref48k()


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build(with_reference=oracle.reference_dir() is not None)
    return oracle


REF_CONFIGS = ("water_262143_L140_M144", "water_48000_L78.4_M80")


def load_ref_config(name):
    """A benchmark-configuration box (make_ref_configs.py): the input
    regenerated from its seed as float32 [n, 4] (checked against the stored
    sha256 of its float64 widening) and the compiled reference's outputs."""
    import hashlib
    from gse_b200 import workloads as W
    system = {"water_262143_L140_M144": W.config_water_262k,
              "water_48000_L78.4_M80": W.config_water_48k}[name]()
    z = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    z = {k: z[k] for k in z.files}
    x64 = system.xyzq.astype(np.float64)
    if hashlib.sha256(x64.tobytes()).digest() != z["xyzq_sha"].tobytes():
        raise AssertionError(f"{name}: the seeded generator no longer gives the golden's input")
    return system, z
