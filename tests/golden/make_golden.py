"""Writes tests/golden/golden.npz: inputs and oracle outputs of the fit path on small seeded
cases.  The reference (umap-rs) ships no numeric golden vectors (its tests pin shapes, epoch
bookkeeping and messages only) and cannot be built here, so these are produced by the CPU
restatement in oracle/ and pin it against accidental change; the GPU path is checked against
the same numbers by tests/test_golden.py.

Cases (inputs stored alongside the outputs):
  ring     the reference's generate_test_data shape (tests.rs:14-38), seeded: n=50, k=10
  gauss    600 points, D=8, 4 Gaussians, exact kNN k=15 (self first)
  disc     300 points, k=10, disconnection_distance 2.5 (edges removed, a vertex cut off)
  lcmix    300 points, k=10, local_connectivity 1.5, set_op_mix_ratio 0.6
Per case: sigmas, rhos, graph CSR, the optimiser's pruned edges (head, tail,
epochs_per_sample) for `total` epochs, the normalised initial embedding, and the exact fired
edge / negative-sample counts of every epoch.  Plus find_ab_params on five (spread, min_dist).

Usage: python tests/golden/make_golden.py   (needs the oracle library: make -C oracle)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "umap-rs_b200"))

AB_PAIRS = [(1.0, 0.1), (1.0, 0.0), (2.0, 0.5), (0.5, 0.25), (1.0, 0.99)]


def ring_inputs(seed=0, n=50, k=10, dim=2):
    g = np.random.Generator(np.random.PCG64(seed))
    idx = np.array([[(i + j + 1) % n for j in range(k)] for i in range(n)], np.uint32)
    dist = (g.random((n, k), dtype=np.float32) * 2.0).astype(np.float32)
    init = (g.random((n, dim), dtype=np.float32) * 10.0).astype(np.float32)
    return idx, dist, init


def gauss_inputs(n, k, seed, d=8, clusters=4):
    from umap_b200 import workloads as W
    X, _ = W.gaussian_mixture(n, d, clusters, 5.0, seed=seed)
    idx, dist = W.knn_exact_numpy(X, k)
    return idx.astype(np.uint32), dist.astype(np.float32), W.uniform_init(n, seed=seed)


def cases():
    """name -> (idx, dist, init, oracle config kwargs, total_epochs)"""
    out = {}
    out["ring"] = (*ring_inputs(), dict(n_neighbors=10, n_epochs=10), 10)
    out["gauss"] = (*gauss_inputs(600, 15, seed=7), dict(n_neighbors=15, n_epochs=200), 200)
    idx, dist, init = gauss_inputs(300, 10, seed=9)
    dist = dist.copy()
    dist[5, 1:] = np.inf  # vertex 5: every neighbour beyond the disconnection distance
    dist[idx == 5] = np.inf
    out["disc"] = (idx, dist, init, dict(n_neighbors=10, n_epochs=50, disconnection_distance=2.5), 50)
    out["lcmix"] = (*gauss_inputs(300, 10, seed=10),
                    dict(n_neighbors=10, n_epochs=30, local_connectivity=1.5, set_op_mix_ratio=0.6), 30)
    return out


def compute():
    import oracle as O
    O.build()
    O.set_threads(1)
    z = {}
    for i, (s, md) in enumerate(AB_PAIRS):
        a, b = O.find_ab_params(s, md)
        z[f"ab_{i}"] = np.array([s, md, a, b], np.float32)
    for name, (idx, dist, init, kw, total) in cases().items():
        cfg = O.OracleConfig(**kw)
        m = O.learn_manifold(idx, dist, cfg)
        info = m.info()
        sig, rho = m.sigmas_rhos()
        ip, ix, dt = m.graph()
        opt = O.Optimizer(m, init, total, cfg, seed=0)
        head, tail, eps = opt.edges()
        emb0 = opt.embedding()
        fires, negs = opt.step_epochs(total, counts=True)
        p = name + "/"
        z[p + "idx"], z[p + "dist"], z[p + "init"] = idx, dist, init
        z[p + "config"] = np.array([kw.get("n_neighbors", 15), total, kw.get("local_connectivity", 1.0),
                                    kw.get("set_op_mix_ratio", 1.0),
                                    kw.get("disconnection_distance", np.inf)], np.float64)
        z[p + "ab"] = np.array([info["a"], info["b"]], np.float32)
        z[p + "disconnection"] = np.array([info["edges_removed"], info["vertices_disconnected"]], np.uint64)
        z[p + "sigmas"], z[p + "rhos"] = sig, rho
        z[p + "indptr"], z[p + "indices"], z[p + "data"] = ip, ix, dt
        z[p + "head"], z[p + "tail"], z[p + "eps"] = head, tail, eps
        z[p + "emb0"] = emb0
        z[p + "fires"], z[p + "negs"] = fires, negs
    return z


def main():
    z = compute()
    path = os.path.join(HERE, "golden.npz")
    np.savez_compressed(path, **z)
    print(f"wrote {path}: {os.path.getsize(path)} bytes, {len(z)} arrays")


if __name__ == "__main__":
    main()
