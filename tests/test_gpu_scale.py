"""Size-independent properties of the fit path on a 3,000,000-point swiss roll (the
100M-point configuration's distribution; exact kNN on a uniform grid): the fuzzy union is
symmetric (set_op_mix_ratio 1), rows are sorted without self loops, weights lie in (0, 1],
a seeded sample of rows has bit-exact rho and sigma within 1e-5 of the oracle, the pruned
edge count equals the number of weights at or above max / total_epochs, the schedule totals
are additive over epoch ranges, and the fitted embedding is finite."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_swiss_roll_3m_properties(ub, oracle):
    import torch
    from umap_b200 import workloads as W
    n, total = 3_000_000, 200
    X = W.swiss_roll_torch(n, seed=2)
    idx, dist, _ = W.knn_grid_torch(X, 15)
    del X
    assert bool((idx[:, 0] == torch.arange(n, device=idx.device, dtype=torch.int32)).float().mean() > 0.999)
    cfg = ub.UmapConfig()
    cfg.optimization.n_epochs = total
    m = ub.Umap(cfg).learn_manifold(n, idx, dist)
    G = m.graph()
    ip = G.indptr.astype(np.int64)
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(ip))
    cols = G.indices.astype(np.int64)
    w = G.data
    assert (w > 0).all() and (w <= 1).all()
    assert not (rows == cols).any(), "no self loops"
    same_row = rows[1:] == rows[:-1]
    assert (cols[1:][same_row] > cols[:-1][same_row]).all(), "rows sorted, no duplicates"
    # symmetric: (r, c, w) and (c, r, w) both present
    key = rows * n + cols
    tkey = cols * n + rows
    order = np.argsort(tkey, kind="stable")
    assert np.array_equal(tkey[order], key), "structure symmetric"
    assert np.array_equal(w[order].view(np.uint32), w.view(np.uint32)), "weights symmetric"
    # sampled rows against the oracle's smooth-kNN
    s, r = m.sigmas_rhos()
    sample = np.sort(np.random.Generator(np.random.PCG64(1)).choice(n, 5000, replace=False))
    so, ro = oracle.smooth_knn_dist(dist[torch.from_numpy(sample).cuda()].cpu().numpy(), 15)
    assert np.array_equal(r[sample].view(np.uint32), ro.view(np.uint32))
    assert np.all(np.abs(s[sample].astype(np.float64) - so) <= 1e-5 * np.abs(so))
    thr = np.float32(np.float32(w.max()) / np.float32(total))
    kept = int((w >= thr).sum())
    g = torch.Generator(device="cuda").manual_seed(0)
    init = torch.rand((n, 2), generator=g, device="cuda") * 20.0 - 10.0
    opt = ub.Optimizer(m, init, total, cfg)
    assert opt.n_edges() == kept
    f_all, n_all = opt.schedule_totals(0, total)
    f1, n1 = opt.schedule_totals(0, 77)
    f2, n2 = opt.schedule_totals(77, total)
    assert (f1 + f2, n1 + n2) == (f_all, n_all)
    assert 0 < f_all and n_all > 4 * f_all
    opt.step_epochs(total)
    emb = opt.embedding()
    assert np.isfinite(emb).all()
