"""Golden fixtures (tests/golden/golden.npz, written by tests/golden/make_golden.py from the
CPU oracle): the oracle must still reproduce them bit for bit (CPU), and the GPU path must
match them with the parity bar of the fit path: rho, CSR structure, pruned edge count and
edge lists bit-exact; sigma and weights within 1e-5 relative; the normalised initial
embedding bit-exact; per-epoch fired-edge / negative-sample totals from the schedule."""
import os

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.npz")
CASES = ["ring", "gauss", "disc", "lcmix"]
REL = 1e-5


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(GOLDEN))


def _rel_close(a, b, rel=REL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    with np.errstate(invalid="ignore"):
        return (a == b) | (np.abs(a - b) <= rel * np.maximum(np.abs(a), np.abs(b)))


def _oracle_config(oracle, z, name):
    k, total, lc, mix, disc = z[name + "/config"]
    return oracle.OracleConfig(n_neighbors=int(k), n_epochs=int(total), local_connectivity=float(lc),
                               set_op_mix_ratio=float(mix),
                               disconnection_distance=None if np.isinf(disc) else float(disc)), int(total)


def _ub_config(ub, z, name):
    k, total, lc, mix, disc = z[name + "/config"]
    c = ub.UmapConfig()
    c.graph.n_neighbors = int(k)
    c.graph.local_connectivity = float(lc)
    c.graph.set_op_mix_ratio = float(mix)
    c.graph.disconnection_distance = None if np.isinf(disc) else float(disc)
    c.optimization.n_epochs = int(total)
    return c, int(total)


def test_fixture_is_small_and_complete(golden):
    assert os.path.getsize(GOLDEN) < 512 * 1024
    for name in CASES:
        for key in ("idx", "dist", "init", "sigmas", "rhos", "indptr", "indices", "data", "head", "tail", "eps",
                    "emb0", "fires", "negs"):
            assert name + "/" + key in golden, (name, key)


def test_oracle_reproduces_golden(oracle, golden):
    oracle.set_threads(1)
    for i in range(5):
        s, md, a, b = golden[f"ab_{i}"]
        assert oracle.find_ab_params(float(s), float(md)) == (a, b)
    for name in CASES:
        p = name + "/"
        cfg, total = _oracle_config(oracle, golden, name)
        m = oracle.learn_manifold(golden[p + "idx"], golden[p + "dist"], cfg)
        s, r = m.sigmas_rhos()
        assert np.array_equal(s.view(np.uint32), golden[p + "sigmas"].view(np.uint32)), name
        assert np.array_equal(r.view(np.uint32), golden[p + "rhos"].view(np.uint32)), name
        ip, ix, dt = m.graph()
        assert np.array_equal(ip, golden[p + "indptr"]) and np.array_equal(ix, golden[p + "indices"]), name
        assert np.array_equal(dt.view(np.uint32), golden[p + "data"].view(np.uint32)), name
        opt = oracle.Optimizer(m, golden[p + "init"], total, cfg, seed=5)
        h, t, e = opt.edges()
        assert np.array_equal(h, golden[p + "head"]) and np.array_equal(t, golden[p + "tail"]), name
        assert np.array_equal(e.view(np.uint64), golden[p + "eps"].view(np.uint64)), name
        assert np.array_equal(opt.embedding(), golden[p + "emb0"]), name
        f, g = opt.step_epochs(total, counts=True)
        # the schedule is deterministic: counts do not depend on the seed
        assert np.array_equal(f, golden[p + "fires"]) and np.array_equal(g, golden[p + "negs"]), name


def test_abi_find_ab_params_matches_golden(ub, golden):
    for i in range(5):
        s, md, a, b = golden[f"ab_{i}"]
        assert ub.find_ab_params(float(s), float(md)) == (a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_matches_golden(ub, golden, name):
    p = name + "/"
    cfg, total = _ub_config(ub, golden, name)
    idx, dist, init = golden[p + "idx"], golden[p + "dist"], golden[p + "init"]
    m = ub.Umap(cfg).learn_manifold(idx.shape[0], idx, dist)
    assert m.curve_params() == tuple(golden[p + "ab"])
    assert m.disconnection_counts() == tuple(int(v) for v in golden[p + "disconnection"])
    s, r = m.sigmas_rhos()
    assert np.array_equal(r.view(np.uint32), golden[p + "rhos"].view(np.uint32)), "rho must be bit-exact"
    assert _rel_close(s, golden[p + "sigmas"]).all()
    G = m.graph()
    assert np.array_equal(G.indptr, golden[p + "indptr"]), "row pointers must be bit-exact"
    assert np.array_equal(G.indices, golden[p + "indices"]), "column indices must be bit-exact"
    assert _rel_close(G.data, golden[p + "data"]).all()
    opt = ub.Optimizer(m, init, total, cfg)
    h, t, e, _, _, _ = opt.export_edges()
    assert opt.n_edges() == len(golden[p + "head"]), "pruned edge count must be bit-exact"
    assert np.array_equal(h, golden[p + "head"]) and np.array_equal(t, golden[p + "tail"])
    assert _rel_close(e, golden[p + "eps"]).all()
    assert np.array_equal(opt.embedding(), golden[p + "emb0"])
    F, N = golden[p + "fires"], golden[p + "negs"]
    for a, b in [(0, 1), (0, total // 3), (total // 3, total), (0, total)]:
        f, g = opt.schedule_totals(a, b)
        fo, go = int(F[a:b].sum()), int(N[a:b].sum())
        assert abs(f - fo) <= 1e-4 * fo + 1, (a, b, f, fo)
        assert abs(g - go) <= 1e-4 * go + 5, (a, b, g, go)
    opt.step_epochs(total)
    emb = opt.embedding()
    rows_empty = np.diff(golden[p + "indptr"].astype(np.int64)) == 0
    assert np.isfinite(emb[~rows_empty]).all()
