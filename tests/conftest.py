import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "umap-rs_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path")


def _gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def ub():
    lib = os.path.join(PKG, "umap_b200", "libumap_b200.so")
    if not os.path.exists(lib):
        sys.path.insert(0, PKG)
        import build as B
        B.build()
    import umap_b200
    return umap_b200


def ring_fixture(seed=0, n=50, k=10, dim=2):
    """Shape of the reference's generate_test_data (umap-rs/src/tests.rs:14-38): ring kNN
    idx[i,j] = (i+j+1) % n, distances U[0,2) (unsorted, no self column), init U[0,10).
    Seeded here (the reference's is unseeded)."""
    g = np.random.Generator(np.random.PCG64(seed))
    idx = np.array([[(i + j + 1) % n for j in range(k)] for i in range(n)], np.uint32)
    dist = (g.random((n, k), dtype=np.float32) * 2.0).astype(np.float32)
    init = (g.random((n, dim), dtype=np.float32) * 10.0).astype(np.float32)
    return idx, dist, init


def pairs_fixture(n_pairs=300, dim=2, seed=0):
    """Disjoint pairs (2m, 2m+1): each row's kNN is [self (0), partner (d > 0)], so after
    the prune every vertex has one edge of weight 1 (epochs_per_sample 1) to its partner.
    With negative_sample_rate = 0 an epoch's result does not depend on the order of the
    edge updates (each snapshot row is read and moved by one edge only), so every
    implementation of the SGD rule must agree up to rounding."""
    g = np.random.Generator(np.random.PCG64(seed))
    n = 2 * n_pairs
    idx = np.empty((n, 2), np.uint32)
    idx[:, 0] = np.arange(n)
    idx[:, 1] = np.arange(n) ^ 1
    dist = np.zeros((n, 2), np.float32)
    dist[:, 1] = (g.random(n, dtype=np.float32) + 0.5).astype(np.float32)
    init = (g.random((n, dim), dtype=np.float32) * 10.0).astype(np.float32)
    return idx, dist, init


@pytest.fixture(scope="session")
def ring():
    return ring_fixture()


@pytest.fixture(scope="session")
def gauss10k():
    """10,000 points, D=32, 10 isotropic Gaussians, seed 0; exact kNN k=15 (self first)."""
    from umap_b200 import workloads as W
    cache = os.path.join(ROOT, "tests", "golden", "gauss10k_knn.npz")
    if os.path.exists(cache):
        z = np.load(cache)
        return z["idx"], z["dist"], W.uniform_init(10_000)
    X, _ = W.gaussians_10k()
    idx, dist = W.knn_exact_numpy(X, 15)
    return idx, dist, W.uniform_init(10_000)


def small_gauss(n, k, seed, d=8, clusters=4):
    from umap_b200 import workloads as W
    X, _ = W.gaussian_mixture(n, d, clusters, 5.0, seed=seed)
    idx, dist = W.knn_exact_numpy(X, k)
    return idx, dist, W.uniform_init(n, seed=seed)
