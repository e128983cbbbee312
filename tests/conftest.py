import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_lib():
    """The in-house C restatement (built with gcc on demand)."""
    from oracle import oracle
    if not os.path.exists(oracle.ORACLE_LIB):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    return oracle.CLib(oracle.ORACLE_LIB)


@pytest.fixture(scope="session")
def oracle_omp_lib():
    """The same restatement built with OpenMP (identical results, all host
    cores): the checker for the full-size configurations."""
    from oracle import oracle
    if not os.path.exists(oracle.ORACLE_OMP_LIB):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    return oracle.CLib(oracle.ORACLE_OMP_LIB)


@pytest.fixture(scope="session")
def tensors():
    return np.load(os.path.join(GOLDEN, "tensors.npz"))


@pytest.fixture(scope="session")
def trajectories():
    return np.load(os.path.join(GOLDEN, "trajectories.npz"))


@pytest.fixture(scope="session")
def forces_golden():
    return np.load(os.path.join(GOLDEN, "forces.npz"))


def rel_err(a, b):
    """max |a - b| / max |b| (the matrix-level relative error used throughout)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    na, nb = ~np.isfinite(a), ~np.isfinite(b)
    if not np.array_equal(na, nb):
        return float("inf")  # non-finite entries (e.g. overlapping lubricated pairs) must coincide
    a, b = a[~na], b[~nb]
    if b.size == 0:
        return 0.0
    scale = np.max(np.abs(b))
    if scale == 0:
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a - b)) / scale)
