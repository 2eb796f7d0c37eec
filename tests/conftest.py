import ctypes
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def _gpu_count():
    try:
        cuda = ctypes.CDLL("libcuda.so.1")
    except OSError:
        return 0
    if cuda.cuInit(0) != 0:
        return 0
    n = ctypes.c_int()
    if cuda.cuDeviceGetCount(ctypes.byref(n)) != 0:
        return 0
    return n.value


HAVE_GPU = _gpu_count() > 0


def pytest_collection_modifyitems(config, items):
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device visible")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def golden_catalogs():
    return dict(np.load(os.path.join(GOLDEN, "catalogs.npz")))


@pytest.fixture(scope="session")
def golden_tables():
    return dict(np.load(os.path.join(GOLDEN, "tables.npz")))


def uniform_catalog(n, lo, hi, seed, weights="unit"):
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    posw = np.empty((n, 4))
    posw[:, :3] = lo + (hi - lo) * rng.random((n, 3))
    if weights == "unit":
        posw[:, 3] = 1.0
    else:
        posw[:, 3] = rng.uniform(0.5, 1.5, n)
    return posw


def clustered_catalog(n, lo, hi, seed, ncenters=50, sigma=None):
    """Gaussian clumps inside [lo, hi) plus a uniform background."""
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    if sigma is None:
        sigma = 0.02 * float(np.min(hi - lo))
    centers = lo + (hi - lo) * rng.random((ncenters, 3))
    pick = rng.integers(0, ncenters, n // 2)
    pts = centers[pick] + rng.normal(0, sigma, (n // 2, 3))
    pts = np.clip(pts, lo, hi - 1e-9 * (hi - lo))
    uni = lo + (hi - lo) * rng.random((n - n // 2, 3))
    posw = np.empty((n, 4))
    posw[:, :3] = np.concatenate([pts, uni])
    posw[:, 3] = rng.uniform(0.5, 1.5, n)
    return posw
