import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libsw2gpu.so")


@pytest.fixture(scope="session")
def channel_ref():
    return dict(np.load(os.path.join(GOLDEN, "channel_ref.npz")))


@pytest.fixture(scope="session")
def basin_ref():
    return dict(np.load(os.path.join(GOLDEN, "basin_ref.npz")))


@pytest.fixture(scope="session")
def mass_ref():
    return dict(np.load(os.path.join(GOLDEN, "mass_ref.npz")))


@pytest.fixture(scope="session")
def transport_ref():
    return dict(np.load(os.path.join(GOLDEN, "transport_ref.npz")))


def relerr(a, b):
    """max |a - b| / max |b| (the per-field error used throughout the tests)."""
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
