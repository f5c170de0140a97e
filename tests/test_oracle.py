"""CPU tests of the oracle (the C++ restatement of the reference's CPU path).

The reference pins no numeric value on this path (umap-rs/src/tests.rs holds smoke tests
only), so the oracle is checked here against (1) hand-derived known answers of each
reference function and (2) the reference's own smoke-test assertions, re-expressed.
"""
import math

import numpy as np
import pytest

from conftest import ring_fixture, small_gauss


def np_unrolled_mean(x):
    """ndarray 0.17 mean (sum via 8-way unrolled fold), written in numpy float32."""
    x = np.asarray(x, np.float32)
    f = np.float32
    p = [f(0)] * 8
    n = len(x)
    i = 0
    while n - i >= 8:
        for j in range(8):
            p[j] = f(p[j] + x[i + j])
        i += 8
    acc = f(0)
    for a, b in ((0, 4), (1, 5), (2, 6), (3, 7)):
        acc = f(acc + f(p[a] + p[b]))
    for t in range(min(n - i, 7)):
        acc = f(acc + x[i + t])
    return f(acc / f(n))


@pytest.mark.parametrize("n", [1, 7, 8, 9, 15, 16, 17, 31, 100, 1001])
def test_ndarray_mean_order(oracle, n):
    x = np.random.Generator(np.random.PCG64(n)).random(n, dtype=np.float32) * 3
    assert oracle.ndarray_mean(x) == np_unrolled_mean(x)


def test_find_ab_params_fits_curve(oracle):
    # find_ab_params.rs: 1 / (1 + a x^(2b)) fitted to the offset exponential on [0, 3*spread].
    for spread, min_dist in [(1.0, 0.1), (1.0, 0.0), (2.0, 0.5), (1.0, 0.99)]:
        a, b = oracle.find_ab_params(spread, min_dist)
        assert 0.001 <= a <= 10 and 0.001 <= b <= 10
        x = np.linspace(0, 3 * spread, 300)
        y = np.where(x < min_dist, 1.0, np.exp(-(x - min_dist) / spread))
        fit = 1.0 / (1.0 + a * x ** (2 * b))
        start = 1.0 / (1.0 + 1.5 * x ** (2 * 0.9))   # the GD's initial guess (a=1.5, b=0.9)
        assert np.mean((fit - y) ** 2) < np.mean((start - y) ** 2)
    a, b = oracle.find_ab_params(1.0, 0.1)
    assert a > 0 and b > 0  # tests.rs:77-78


def test_smooth_knn_equal_distances(oracle):
    # All neighbour distances equal d: rho = d, every term is 1 so psum = k-1 > log2(k) at
    # every step; mid halves 64 times, then the MIN_K_DIST_SCALE clamp gives 1e-3 * mean.
    k = 10
    d = np.zeros((1, k), np.float32)
    d[0, 1:] = 2.5
    s, r = oracle.smooth_knn_dist(d)
    assert r[0] == np.float32(2.5)
    assert s[0] == np.float32(np.float32(1e-3) * np_unrolled_mean(d[0]))


def test_smooth_knn_solves_target(oracle):
    g = np.random.Generator(np.random.PCG64(3))
    d = np.sort(g.random((200, 15), dtype=np.float32) * 4, axis=1)
    d[:, 0] = 0
    s, r = oracle.smooth_knn_dist(d)
    assert np.array_equal(r, d[:, 1])  # rho = first non-zero distance (local_connectivity 1)
    target = math.log2(15)
    for i in range(200):
        terms = np.where(d[i, 1:] - r[i] > 0, np.exp(-(d[i, 1:] - r[i]) / s[i]), 1.0)
        assert abs(terms.sum() - target) < 1e-4


def test_smooth_knn_local_connectivity_interpolation(oracle):
    d = np.array([[0, 1, 2, 4, 8, 9, 10, 11]], np.float32)
    _, r = oracle.smooth_knn_dist(d, local_connectivity=1.5)   # rho = d1 + 0.5 (d2 - d1)
    assert r[0] == np.float32(1.5)
    _, r = oracle.smooth_knn_dist(d, local_connectivity=0.5)   # index 0: 0.5 * first non-zero
    assert r[0] == np.float32(0.5)
    _, r = oracle.smooth_knn_dist(np.zeros((1, 8), np.float32))  # no non-zero -> 0
    assert r[0] == 0
    d2 = np.array([[0, 0, 0, 3, 0, 0, 0, 0]], np.float32)
    _, r = oracle.smooth_knn_dist(d2, local_connectivity=2.0)  # fewer non-zeros -> max
    assert r[0] == np.float32(3)


def test_zero_rho_uses_global_mean(oracle):
    d = np.ones((4, 6), np.float32)
    d[2] = 0.0
    s, r = oracle.smooth_knn_dist(d)
    assert r[2] == 0
    assert s[2] >= np.float32(1e-3) * np_unrolled_mean(d.ravel()) - 1e-12


def test_membership_and_union_known_answers(oracle):
    # 3 points; 0 -> 1 (dist 1 = rho, weight 1), 1 -> 2, 2 -> 0 with an extra self and
    # sentinel column that must be skipped.
    idx = np.array([[0, 1, 0xFFFFFFFF], [1, 2, 0], [2, 0, 1]], np.uint32)
    dist = np.array([[0, 1, 5], [0, 1, 3], [0, 2, 2.5]], np.float32)
    cfg = oracle.OracleConfig(n_neighbors=3, symmetrize=False)
    # n_samples must exceed n_neighbors: pad with an isolated 4th point
    idx4 = np.vstack([idx, [[3, 3, 3]]]).astype(np.uint32)
    dist4 = np.vstack([dist, [[0, 0, 0]]]).astype(np.float32)
    m = oracle.learn_manifold(idx4, dist4, cfg)
    ip, ix, dt = m.directed()
    sig, rho = m.sigmas_rhos()
    assert list(ip) == [0, 1, 3, 5, 5]
    assert list(ix[:1]) == [1]            # sentinel skipped, self skipped
    assert dt[0] == 1.0                   # d - rho <= 0
    # row 1: cols sorted (0, 2); weight for col 0 = exp(-(3 - 1)/sigma_1)
    assert list(ix[1:3]) == [0, 2]
    x = np.float32(np.float32(-(np.float32(3) - rho[1])) / sig[1])
    expect = np.float32(np.exp(np.float64(x)))   # correctly rounded; glibc expf is within 1 ulp
    assert abs(int(dt[1].view(np.int32)) - int(expect.view(np.int32))) <= 1
    # union with mix = 1: A + A^T - A o A^T
    cfg_u = oracle.OracleConfig(n_neighbors=3, symmetrize=True)
    mu = oracle.learn_manifold(idx4, dist4, cfg_u)
    Ad = np.zeros((4, 4), np.float32)
    for r_ in range(4):
        for q in range(ip[r_], ip[r_ + 1]):
            Ad[r_, ix[q]] = dt[q]
    uip, uix, udt = mu.graph()
    U = np.zeros((4, 4), np.float32)
    for r_ in range(4):
        for q in range(uip[r_], uip[r_ + 1]):
            U[r_, uix[q]] = udt[q]
    f = np.float32
    for i in range(4):
        for j in range(4):
            a, b = Ad[i, j], Ad[j, i]
            if a == 0 and b == 0:
                assert U[i, j] == 0
            elif a != 0:
                assert U[i, j] == f(f(f(1) * a + f(1) * b) + f(f(f(-1) * a) * b))
            else:
                assert U[i, j] == b
    assert np.array_equal(U, U.T)


def test_intersection_drops_one_sided(oracle):
    idx, dist, _ = ring_fixture()
    cfg = oracle.OracleConfig(n_neighbors=10, set_op_mix_ratio=0.0)
    m = oracle.learn_manifold(idx, dist, cfg)
    ip, ix, dt = m.graph()
    # ring kNN (i -> i+1..i+10) has no reciprocal pairs, so intersection is empty
    assert len(ix) == 0


def test_disconnection_distance(oracle):
    idx, dist, _ = ring_fixture()
    cfg = oracle.OracleConfig(n_neighbors=10, disconnection_distance=1.0, symmetrize=False)
    m = oracle.learn_manifold(idx, dist, cfg)
    info = m.info()
    assert info["edges_removed"] == int((dist >= 1.0).sum())
    ip, ix, _ = m.directed()
    assert ip[-1] <= int((dist < 1.0).sum())
    for r in range(len(idx)):            # no kept entry has a removed (>= 1.0) distance
        d_of = {int(c): float(d) for c, d in zip(idx[r], dist[r])}
        assert all(d_of[int(c)] < 1.0 for c in ix[ip[r]:ip[r + 1]])


def _repeat_neighbour(idx, dist, row, dup_col, src_col):
    """Row `row` lists neighbour idx[row, src_col] a second time, in column dup_col."""
    idx, dist = idx.copy(), dist.copy()
    idx[row, dup_col] = idx[row, src_col]
    return idx, dist


def test_repeated_neighbour_is_refused(oracle):
    """A kNN row that keeps one neighbour twice reaches sprs's CsMatI::new with a repeated
    column (fuzzy_simplicial_set.rs:291), whose structure check refuses it: the reference
    panics, the oracle returns that text with the smallest offending row."""
    idx, dist, _ = ring_fixture()
    bad_i, bad_d = _repeat_neighbour(idx, dist, 7, 4, 2)
    bad_i[30, 9] = bad_i[30, 0]
    with pytest.raises(oracle.OracleError, match=r"^knn_indices row 7 keeps the same neighbour more than once"):
        oracle.learn_manifold(bad_i, bad_d, oracle.OracleConfig(n_neighbors=10))
    with pytest.raises(oracle.OracleError, match=r"Unsorted\("):
        oracle.learn_manifold(bad_i, bad_d, oracle.OracleConfig(n_neighbors=10, symmetrize=False))


def test_repeated_neighbour_dropped_before_the_csr_is_accepted(oracle):
    """A repeat that never reaches the CSR is harmless: a disconnected copy (distance at or
    beyond disconnection_distance) or a repeated sentinel / self entry is skipped first."""
    idx, dist, _ = ring_fixture()
    i2, d2 = _repeat_neighbour(idx, dist, 7, 4, 2)
    d2[7, 4] = np.inf                                      # the repeat is disconnected
    m = oracle.learn_manifold(i2, d2, oracle.OracleConfig(n_neighbors=10))
    ip, ix, _ = m.directed()
    assert ip[8] - ip[7] == 9 and len(set(ix[ip[7]:ip[8]].tolist())) == 9
    i3 = idx.copy()
    i3[11, 3] = i3[11, 5] = 0xFFFFFFFF                     # two sentinels
    i3[12, 3] = i3[12, 6] = 12                             # self twice
    oracle.learn_manifold(i3, dist, oracle.OracleConfig(n_neighbors=10))


# ---- the reference's smoke tests (umap-rs/src/tests.rs), against the oracle
def test_ref_learn_manifold(oracle, ring):
    idx, dist, _ = ring
    m = oracle.learn_manifold(idx, dist, oracle.OracleConfig(n_neighbors=10))
    info = m.info()
    assert info["n_vertices"] == 50
    assert len(m.graph()[1]) > 0
    assert info["a"] > 0 and info["b"] > 0


def test_ref_high_level_fit(oracle, ring):
    idx, dist, init = ring
    emb, _, _ = oracle.fit(idx, dist, init, oracle.OracleConfig(n_neighbors=10, n_epochs=10))
    assert emb.shape == (50, 2)
    assert np.all(np.isfinite(emb) | np.isnan(emb))


def test_ref_optimizer_step_epochs_and_overstep(oracle, ring):
    idx, dist, init = ring
    cfg = oracle.OracleConfig(n_neighbors=10)
    m = oracle.learn_manifold(idx, dist, cfg)
    opt = oracle.Optimizer(m, init, 20, cfg)
    assert (opt.current_epoch(), opt.remaining_epochs()) == (0, 20)
    opt.step_epochs(5)
    assert (opt.current_epoch(), opt.remaining_epochs()) == (5, 15)
    opt.step_epochs(13)
    with pytest.raises(oracle.OracleError, match=r"^Cannot step 5 epochs: would exceed total_epochs 20 \(current: 18\)$"):
        opt.step_epochs(5)


def fixed_point_schedule(eps, total, neg):
    """The GPU's stateless schedule in exact integer arithmetic: Q = ceil(2^32/eps),
    m(n) = (n*Q) >> 32 firings by epoch n, y(x) = (x*neg*Q) >> 32; a firing at n with index m
    draws y(n) - y(p) negatives (p = epoch of firing m-1; y(n) - 1 for the first firing)."""
    Q = np.clip(np.ceil(4294967296.0 / eps), 1, 2 ** 32).astype(np.uint64)
    F, N = [], []
    for n in range(total):
        n64 = np.uint64(n)
        m = (n64 * Q) >> np.uint64(32)
        mp = ((np.uint64(n - 1) * Q) >> np.uint64(32)) if n > 0 else np.zeros_like(Q)
        fired = m > mp
        y = (n64 * np.uint64(neg) * Q) >> np.uint64(32)
        mm1 = np.maximum(m, np.uint64(1)) - np.uint64(1)
        p = ((mm1 << np.uint64(32)) + Q - np.uint64(1)) // Q
        yp = (p * np.uint64(neg) * Q) >> np.uint64(32)
        nn = np.where(m <= 1, y.astype(np.int64) - 1, y.astype(np.int64) - yp.astype(np.int64))
        F.append(int(fired.sum()))
        N.append(int(np.where(fired, np.maximum(nn, 0), 0).sum()))
    return np.array(F), np.array(N)


def test_schedule_closed_form_matches_state_arrays(oracle):
    """The GPU keeps one fixed-point value per edge and recomputes the schedule in closed
    form; it must reproduce the reference's f64 state evolution
    (optimize_layout_euclidean.rs:277-343) epoch by epoch."""
    idx, dist, init = small_gauss(600, 10, seed=5)
    cfg = oracle.OracleConfig(n_neighbors=10)
    m = oracle.learn_manifold(idx, dist, cfg)
    total = 60
    opt = oracle.Optimizer(m, init, total, cfg, seed=1)
    _, _, eps = opt.edges()
    F, N = opt.step_epochs(total, counts=True)
    gF, gN = fixed_point_schedule(eps, total, 5)
    assert np.abs(gF - F.astype(np.int64)).sum() <= 1e-5 * F.sum() + 1
    assert np.abs(gN - N.astype(np.int64)).sum() <= 1e-5 * N.sum() + 5


# ---------------------------------------------------------------- SGD update rules, known answers
def np_pairs_epochs(x0, a, b, gamma, lr, total, n_ep, generic):
    """One step_epochs(n_ep) call on the pairs graph (conftest.pairs_fixture) with
    negative_sample_rate = 0, in numpy float32: live buffer `x`, snapshot `c` cloned once
    (optimizer.rs:314), every edge (j -> j^1) fires at every epoch >= 1.  Euclidean rule:
    optimize_layout_euclidean.rs:284-306; generic rule with EuclideanMetric:
    optimize_layout_generic.rs:62-86 + distances.rs:22-37."""
    f = np.float32
    x = x0.astype(np.float32).copy()
    c = x.copy()
    n, dim = x.shape
    part = np.arange(n) ^ 1
    a, b = f(a), f(b)
    for e in range(n_ep):
        alpha = f(f(lr) * f(f(1) - f(f(e) / f(total))))
        if e == 0:
            continue                      # epoch_of_next_sample starts at 1
        y = c[part]
        diff = x - y
        ds = np.zeros(n, np.float32)
        for d in range(dim):
            ds = (ds + diff[:, d] * diff[:, d]).astype(np.float32)
        if generic:
            dist = np.sqrt(ds)
            den = (dist + f(1e-6)).astype(np.float32)
            grad = (diff / den[:, None]).astype(np.float32)
            rev = ((y - x) / den[:, None]).astype(np.float32)
            with np.errstate(divide="ignore"):
                pw = np.power(dist, f(f(2) * b)).astype(np.float32)
            w = np.where(dist > 0, f(1) / (f(1) + a * pw), f(1)).astype(np.float32)
            gc = ((f(2) * b) * (w - f(1)) / den).astype(np.float32)
            x = (x + np.clip(gc[:, None] * grad, -4, 4) * alpha).astype(np.float32)
            c[part] = (y + np.clip(gc[:, None] * rev, -4, 4) * alpha).astype(np.float32)
        else:
            with np.errstate(divide="ignore", invalid="ignore"):
                pb = np.power(ds, b).astype(np.float32)
                gc = ((((f(-2) * a) * b) * pb) / ds).astype(np.float32)
                gc = (gc / ((a * pb) * ds + f(1))).astype(np.float32)
            gc = np.where(ds > 0, gc, f(0)).astype(np.float32)
            g = np.clip(gc[:, None] * diff, -4, 4).astype(np.float32)
            x = (x + g * alpha).astype(np.float32)
            c[part] = (y - g * alpha).astype(np.float32)
    return x


@pytest.mark.parametrize("generic", [False, True])
@pytest.mark.parametrize("dim", [1, 2, 3, 5])
def test_update_rules_known_answer(oracle, generic, dim):
    """Both SGD rules of the oracle against a numpy restatement on an order-independent case."""
    from conftest import pairs_fixture
    idx, dist, init = pairs_fixture(200, dim, seed=dim)
    cfg = oracle.OracleConfig(n_neighbors=2, negative_sample_rate=0, n_epochs=12)
    m = oracle.learn_manifold(idx, dist, cfg)
    ip, ix, dt = m.graph()
    assert np.array_equal(np.diff(ip), np.ones(len(idx), np.int64)) and (dt == 1).all()
    opt = oracle.Optimizer(m, init, 12, cfg, seed=3, metric_type=int(generic))
    x0 = opt.embedding()
    opt.step_epochs(12)
    a, b = m.info()["a"], m.info()["b"]
    expect = np_pairs_epochs(x0, a, b, cfg.repulsion_strength, cfg.learning_rate, 12, 12, generic)
    got = opt.embedding()
    assert np.array_equal(got, expect) or np.allclose(got, expect, rtol=2e-6, atol=2e-6)
    assert not np.allclose(got, x0)


def test_generic_rule_schedule_matches_euclidean(oracle):
    """The generic rule changes the force law only: the same edges fire and draw the same
    number of negatives (optimize_layout_generic.rs:57-121 vs optimize_layout_euclidean.rs)."""
    idx, dist, init = small_gauss(600, 10, seed=5)
    cfg = oracle.OracleConfig(n_neighbors=10)
    m = oracle.learn_manifold(idx, dist, cfg)
    F0, N0 = oracle.Optimizer(m, init, 40, cfg, seed=1).step_epochs(40, counts=True)
    og = oracle.Optimizer(m, init, 40, cfg, seed=1, metric_type=1)
    F1, N1 = og.step_epochs(40, counts=True)
    assert np.array_equal(F0, F1) and np.array_equal(N0, N1)
    e = og.embedding()
    assert np.isfinite(e).all()


# ---------------------------------------------------------------- kNN producer
def np_knn_bruteforce(X, k):
    """mnist_demo.rs:203-239 in numpy float32: per row, (x - y)^2 summed column by column, sqrt,
    a stable sort by distance (ties in index order), self excluded, zeros past n - 1."""
    X = np.asarray(X, np.float32)
    n, d = X.shape
    idx = np.zeros((n, k), np.uint32)
    dist = np.zeros((n, k), np.float32)
    for i in range(n):
        acc = np.zeros(n, np.float32)
        for c in range(d):
            df = (X[i, c] - X[:, c]).astype(np.float32)
            acc = (acc + df * df).astype(np.float32)
        dd = np.sqrt(acc)
        others = np.delete(np.arange(n), i)
        order = others[np.argsort(dd[others], kind="stable")][:k]
        idx[i, :len(order)] = order
        dist[i, :len(order)] = dd[order]
    return idx, dist


@pytest.mark.parametrize("n,d,k", [(1, 3, 4), (2, 1, 3), (7, 3, 10), (60, 5, 15), (300, 17, 32)])
def test_knn_oracle_matches_numpy(oracle, n, d, k):
    g = np.random.Generator(np.random.PCG64(n * 31 + d))
    X = g.normal(0, 1, (n, d)).astype(np.float32)
    if n >= 60:
        X[::3] = np.round(X[::3])       # exact ties and duplicate rows
        X[5] = X[2]
    i1, d1 = oracle.knn_bruteforce(X, k)
    i2, d2 = np_knn_bruteforce(X, k)
    assert np.array_equal(i1, i2) and np.array_equal(d1, d2)
