"""kNN producer (umap_knn_bruteforce*): the tensor-core candidate pass + exact rerank +
certificate must return exactly the reference example's brute force
(examples/src/bin/mnist_demo.rs:203-229) as restated by the oracle: identical indices and
bit-identical distances, ties in index order, self excluded, zero padding when n - 1 < k."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _data(n, d, seed, kind="gauss"):
    g = np.random.Generator(np.random.PCG64(seed))
    if kind == "gauss":
        return g.normal(0, 1, (n, d)).astype(np.float32)
    if kind == "clusters":    # 20 blobs: within-blob distances small against the spread
        centres = g.normal(0, 10, (20, d))
        lab = g.integers(0, 20, n)
        return (centres[lab] + g.normal(0, 0.5, (n, d))).astype(np.float32)
    if kind == "ties":        # small integers: many exactly equal distances and duplicate rows
        return g.integers(0, 3, (n, d)).astype(np.float32)
    if kind == "pixels":      # MNIST-like: values in [0, 1], mostly zeros
        x = g.random((n, d)).astype(np.float32)
        x[x < 0.8] = 0.0
        return x
    if kind == "offset":      # far from the origin: centring matters
        return (g.normal(0, 1, (n, d)) + 1000.0).astype(np.float32)
    raise ValueError(kind)


@pytest.mark.parametrize("n,d,k,kind", [
    (2, 3, 1, "gauss"), (3, 2, 5, "gauss"), (17, 7, 16, "gauss"), (257, 1, 15, "gauss"),
    (300, 64, 15, "gauss"), (1000, 100, 32, "gauss"), (2049, 16, 15, "clusters"), (1500, 8, 20, "ties"),
    (1200, 784, 15, "pixels"), (900, 33, 10, "offset"), (5000, 64, 15, "clusters"),
    (300, 1500, 15, "gauss"), (2000, 3, 1, "ties"), (700, 130, 31, "clusters"),
    # from 16,384 points the scan runs in pivot (locality) order
    (20000, 24, 15, "clusters"), (16400, 100, 32, "pixels"), (16384, 5, 15, "ties"),
])
def test_knn_matches_oracle(ub, oracle, n, d, k, kind):
    X = _data(n, d, seed=n + d, kind=kind)
    gi, gd, rec = ub.knn_bruteforce(X, k, return_stats=True)
    oi, od = oracle.knn_bruteforce(X, k)
    bad = np.nonzero((gi != oi).any(1) | (gd != od).any(1))[0]
    assert len(bad) == 0, (len(bad), rec, bad[:5], gi[bad[:2]], oi[bad[:2]], gd[bad[:2]], od[bad[:2]])
    if n - 1 < k:
        assert (gi[:, n - 1:] == 0).all() and (gd[:, n - 1:] == 0).all()
    print(f"n={n} d={d} k={k} {kind}: rows recomputed {rec}")


@pytest.mark.parametrize("n,d,k,kind", [(700, 16, 33, "gauss"), (1500, 40, 100, "clusters"),
                                         (400, 8, 128, "ties"), (60, 5, 100, "gauss")])
def test_knn_long_lists_exact_path(ub, oracle, n, d, k, kind):
    """k above the candidate pass's 32: every row on the exact CUDA-core path, still equal to
    the reference example's brute force (including zero padding when n - 1 < k)."""
    X = _data(n, d, seed=n + k, kind=kind)
    gi, gd, rec = ub.knn_bruteforce(X, k, return_stats=True)
    oi, od = oracle.knn_bruteforce(X, k)
    assert rec == n
    assert np.array_equal(gi, oi) and np.array_equal(gd, od)


def test_knn_device_matches_host_and_uses_fallback_only_when_needed(ub, oracle):
    import torch
    X = _data(4096, 48, seed=3, kind="gauss")
    hi, hd, rh = ub.knn_bruteforce(X, 15, return_stats=True)
    di, dd, rd = ub.knn_bruteforce(torch.from_numpy(X).cuda(), 15, return_stats=True)
    assert np.array_equal(hi, di.cpu().numpy().view(np.uint32)) and np.array_equal(hd, dd.cpu().numpy())
    assert rh == rd and rh < 4096 // 20


def test_knn_certificate_failures_are_recomputed(ub, oracle):
    """Tight blobs far apart: the FP16 error bound (relative to the spread of the whole set)
    exceeds the gaps inside a blob, so certificates fail and rows take the exact path."""
    g = np.random.Generator(np.random.PCG64(9))
    centres = g.normal(0, 1000, (8, 24))
    X = (centres[g.integers(0, 8, 3000)] + g.normal(0, 0.01, (3000, 24))).astype(np.float32)
    gi, gd, rec = ub.knn_bruteforce(X, 12, return_stats=True)
    oi, od = oracle.knn_bruteforce(X, 12)
    assert rec > 0
    assert np.array_equal(gi, oi) and np.array_equal(gd, od)


def test_knn_rejects_bad_input(ub):
    X = _data(100, 4, seed=1)
    X[3, 2] = np.nan
    with pytest.raises(ub.UmapError) as e:
        ub.knn_bruteforce(X, 5)
    assert e.value.code == ub.ERR_INVALID_ARGUMENT
    with pytest.raises(ub.UmapError):
        ub.knn_bruteforce(_data(100, 4, seed=1), ub.KNN_MAX_K + 1)
    with pytest.raises(ub.UmapError):
        ub.knn_bruteforce(_data(100, 4, seed=1), 0)
    i, d = ub.knn_bruteforce(np.zeros((0, 4), np.float32), 3)
    assert i.shape == (0, 3)


def test_knn_feeds_the_fit(ub, oracle):
    """The producer's output is the reference example's fit input: learn_manifold on it gives
    the same graph as on the oracle's kNN."""
    X = _data(3000, 32, seed=4, kind="clusters")
    gi, gd = ub.knn_bruteforce(X, 15)
    cfg = ub.UmapConfig()
    m = ub.Umap(cfg).learn_manifold(X, gi, gd)
    mo = oracle.learn_manifold(*oracle.knn_bruteforce(X, 15), oracle.OracleConfig())
    G = m.graph()
    ip, ix, _ = mo.graph()
    assert np.array_equal(G.indptr, ip) and np.array_equal(G.indices, ix)
