import os
import sys

import numpy as np
import pytest

# tests exercise error paths: make libqbgpu report failures (qb_last_error,
# RuntimeError in the binding) instead of aborting the process
os.environ.setdefault("QB_ABORT_ON_ERROR", "0")

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "inhom-quantum-boltzmann-fourier-c_b200")
GOLDEN = os.path.join(REPO, "tests", "golden")
for p in (PKG, os.path.join(REPO, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: minutes of CPU oracle work; run with QB_RUN_SLOW=1")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("QB_RUN_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow oracle case; set QB_RUN_SLOW=1")
    for it in items:
        if "slow" in it.keywords:
            it.add_marker(skip)


# ---- golden fixtures (raw little-endian float64, N = 32) ----------------------
def golden_c(name, shape=(32, 32)):
    return np.fromfile(os.path.join(GOLDEN, name)).view(np.complex128).reshape(shape)


def golden_r(name, shape):
    return np.fromfile(os.path.join(GOLDEN, name)).reshape(shape)


def avg_abs_err(a, b):
    """upstream test/I1_test.c:82-87: mean over grid points of |dRe| + |dIm|"""
    return float((np.abs(a.real - b.real) + np.abs(a.imag - b.imag)).mean())


def rel_l1(a, b):
    """upstream test/Cc_test.c:177-189: sum |a - b| / sum |b|"""
    return float(np.abs(a - b).sum() / np.abs(b).sum())


@pytest.fixture(scope="session")
def golden_W():
    """test/data/W0..3.dat: real velocity-space Pauli components, N = 32"""
    return np.stack([golden_r(f"W{i}.dat", (32, 32)) for i in range(4)])
