"""Statistics of the SGD epoch's negative-sample generator.

The reference draws each negative sample as `rng.random_range(0..n_vertices)` from an
unseeded thread-local generator (optimize_layout_euclidean.rs:313-314): uniform over the
vertices and independent between draws.  The GPU kernel draws from a counter-based
generator instead: firing (entry e, epoch n) draws its negatives in pairs, pair t being the
SplitMix64 finaliser (Steele, Lea, Flood, OOPSLA 2014) of
    seed ^ e*0x9E3779B97F4A7C15 ^ n*0xC2B2AE3D27D4EB4F  +  t*0xD1B54A32D192ED03,
each 32-bit half mapped into [lo, lo + range) by a multiply-high.  `draws_numpy` restates
that in numpy; the CPU tests pin the restatement (a published SplitMix64 output) and test
its statistics at 10^6-10^7 draws, and the GPU tests check that the kernel's own draws
(umap_sgd_negative_draws_device) equal the restatement and pass the same tests at 10^8.

Bars: chi-square statistics within 5 standard deviations of their degrees of freedom
(z = (chi2 - dof) / sqrt(2 dof), |z| < 5); correlations within 5 / sqrt(samples).
"""
import ctypes as C

import numpy as np
import pytest

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
K_IDX = np.uint64(0x9E3779B97F4A7C15)
K_EPOCH = np.uint64(0xC2B2AE3D27D4EB4F)
K_PAIR = np.uint64(0xD1B54A32D192ED03)


def mix64(z):
    z = np.asarray(z, np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def draws_numpy(seed, first, count, epoch, per, lo, rng_range):
    """[count, per] negative samples of entries first..first+count-1 at `epoch`."""
    e = np.arange(first, first + count, dtype=np.uint64)
    with np.errstate(over="ignore"):
        base = np.uint64(seed) ^ (e * K_IDX) ^ (np.uint64(epoch) * K_EPOCH)
        out = np.empty((count, per), np.uint32)
        for q in range(per):
            r = mix64(base + np.uint64(q >> 1) * K_PAIR)
            rv = (r >> np.uint64(32)) if q & 1 else (r & np.uint64(0xFFFFFFFF))
            out[:, q] = np.uint64(lo) + ((rv * np.uint64(rng_range)) >> np.uint64(32))
    return out


def chi2_z(counts, expected):
    counts = np.asarray(counts, np.float64)
    expected = np.asarray(expected, np.float64)
    chi2 = float(((counts - expected) ** 2 / expected).sum())
    dof = counts.size - 1
    return (chi2 - dof) / np.sqrt(2.0 * dof)


def uniform_bins_expected(n, bins, total):
    """Expected counts when [0, n) is cut into `bins` bins by floor(v * bins / n)."""
    v_edges = np.ceil(np.arange(bins + 1) * n / bins).astype(np.int64)
    return total * np.diff(v_edges) / n


def corr(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.corrcoef(a, b)[0, 1])


# ------------------------------------------------------------------ CPU: the restatement
def test_splitmix64_finaliser_known_answer():
    # SplitMix64's first output from state 0 is mix64(0 + 0x9E3779B97F4A7C15) (Vigna's
    # splitmix64.c, the generator's published reference code).
    assert int(mix64(np.uint64(0x9E3779B97F4A7C15))) == 0xE220A8397B1DCDAF


def test_restated_draws_are_uniform_and_in_range():
    n = 2_000_003
    d = draws_numpy(seed=7, first=0, count=1_000_000, epoch=37, per=5, lo=1000, rng_range=n)
    assert d.min() >= 1000 and d.max() < 1000 + n
    v = (d.astype(np.int64) - 1000).ravel()
    bins = 2000
    counts = np.bincount(v * bins // n, minlength=bins)
    assert abs(chi2_z(counts, uniform_bins_expected(n, bins, v.size))) < 5
    small = draws_numpy(seed=7, first=0, count=500_000, epoch=3, per=4, lo=0, rng_range=7).ravel()
    assert abs(chi2_z(np.bincount(small, minlength=7), np.full(7, small.size / 7))) < 5


def test_restated_draws_are_independent_across_entries_epochs_and_draws():
    n = 1 << 20
    m = 1_000_000
    a = draws_numpy(seed=1, first=0, count=m + 1, epoch=20, per=4, lo=0, rng_range=n).astype(np.float64) / n
    b = draws_numpy(seed=1, first=0, count=m + 1, epoch=21, per=4, lo=0, rng_range=n).astype(np.float64) / n
    lim = 5.0 / np.sqrt(m)
    assert abs(corr(a[:-1, 0], a[1:, 0])) < lim       # adjacent entries, same epoch
    assert abs(corr(a[:, 0], b[:, 0])) < lim          # same entry, next epoch
    assert abs(corr(a[:, 0], a[:, 1])) < lim          # the two halves of one pair
    assert abs(corr(a[:, 1], a[:, 2])) < lim          # consecutive pairs
    # joint distribution of adjacent entries' draws: 32 x 32 cells
    cells = (np.floor(a[:-1, 0] * 32) * 32 + np.floor(a[1:, 0] * 32)).astype(np.int64)
    assert abs(chi2_z(np.bincount(cells, minlength=1024), np.full(1024, m / 1024))) < 5


# ------------------------------------------------------------------ GPU: the kernel's draws
def _gpu_draws(ub, seed, first, count, epoch, per, lo, rng_range):
    import torch
    out = torch.empty(count * per, dtype=torch.int32, device="cuda")
    rc = ub.lib().umap_sgd_negative_draws_device(seed, first, count, epoch, per, lo, rng_range,
                                                 C.c_void_p(out.data_ptr()))
    assert rc == 0, ub.lib().umap_last_error()
    return out


@pytest.mark.gpu
def test_kernel_draws_equal_the_restatement(ub):
    for seed, first, epoch, per, lo, rng in ((0, 0, 1, 6, 0, 10_000), (12345, 987_654_321, 499, 7, 500, 2_000_003),
                                             (2 ** 63 + 5, 2 ** 40, 17, 1, 3, 1)):
        got = _gpu_draws(ub, seed, first, 20_000, epoch, per, lo, rng).cpu().numpy().view(np.uint32)
        want = draws_numpy(seed, first, 20_000, epoch, per, lo, rng).ravel()
        assert np.array_equal(got, want)


@pytest.mark.gpu
def test_kernel_draws_pass_uniformity_and_independence_at_1e8(ub):
    """10^8 draws over the 2M workload's vertex range: 10,000-bin chi-square, exact per-value
    counts on a 13-value range, lag correlations between adjacent entries, consecutive
    epochs and draws within a firing, and a 64 x 64 joint chi-square of adjacent entries."""
    import torch
    n = 2_000_003
    m = 20_000_000
    per = 5
    d = _gpu_draws(ub, 99, 0, m, 40, per, 0, n).view(m, per).to(torch.int64)
    assert int(d.min()) >= 0 and int(d.max()) < n
    bins = 10_000
    counts = torch.bincount((d.flatten() * bins) // n, minlength=bins).cpu().numpy()
    assert abs(chi2_z(counts, uniform_bins_expected(n, bins, m * per))) < 5
    small = _gpu_draws(ub, 99, 0, m, 40, per, 0, 13).to(torch.int64)
    assert abs(chi2_z(torch.bincount(small, minlength=13).cpu().numpy(), np.full(13, m * per / 13))) < 5
    u = d.double() / n
    nxt = _gpu_draws(ub, 99, 0, m, 41, per, 0, n).view(m, per).double() / n
    lim = 5.0 / np.sqrt(m)

    def c(x, y):
        return float(torch.corrcoef(torch.stack([x, y]))[0, 1])

    assert abs(c(u[:-1, 0], u[1:, 0])) < lim
    assert abs(c(u[:, 0], nxt[:, 0])) < lim
    assert abs(c(u[:, 0], u[:, 1])) < lim
    assert abs(c(u[:, 1], u[:, 2])) < lim
    assert abs(c(u[:, 4], nxt[:, 4])) < lim
    cells = (torch.floor(u[:-1, 0] * 64) * 64 + torch.floor(u[1:, 0] * 64)).to(torch.int64)
    assert abs(chi2_z(torch.bincount(cells, minlength=4096).cpu().numpy(), np.full(4096, (m - 1) / 4096))) < 5


# ------------------------------------------------------------------ negatives per firing
def negatives_per_firing_exact(q, n, neg):
    """The schedule's closed form in exact integers: with Q = q + 1, firing m happens at epoch
    e_m = ceil(m 2^32 / Q), and the firing at epoch n (m = floor(n Q / 2^32)) draws
    y(n) - y(e_{m-1}) negatives, y(x) = floor(x neg Q / 2^32), or y(n) - 1 for m = 1."""
    Q = q.astype(np.uint64) + np.uint64(1)
    n64 = n.astype(np.uint64)
    m = (n64 * Q) >> np.uint64(32)
    fires = m > ((n64 - np.uint64(1)) * Q >> np.uint64(32))
    prev_e = (((m - np.uint64(1)) << np.uint64(32)) + Q - np.uint64(1)) // Q
    y = (n64 * np.uint64(neg) * Q) >> np.uint64(32)
    yp = np.where(m > 1, (prev_e * np.uint64(neg) * Q) >> np.uint64(32), np.uint64(1))
    out = np.where(y > yp, y - yp, np.uint64(0))
    return np.where(fires & (n64 > 0), out, np.uint64(0)).astype(np.uint32)


@pytest.mark.gpu
def test_kernel_negative_counts_per_firing_are_exact(ub):
    """The epoch kernel's per-firing negative count against the exact closed form, on firing
    epochs of edges with epochs_per_sample in [1, 500] (the prune keeps eps <= total_epochs),
    on non-firing epochs (0), at Q = 2^32 (an edge that fires every epoch), and for
    epochs_per_sample up to 2^20 with firing epochs below 2^21 (the largest total_epochs an
    optimizer accepts), where the kernel's float estimate of the firing gap is least exact."""
    import torch
    g = np.random.Generator(np.random.PCG64(5))
    neg = 5
    eps = np.concatenate([g.uniform(1.0, 500.0, 400_000), np.round(g.uniform(1, 60, 20_000)),
                          2.0 ** g.uniform(14, 19.9, 2_000)])
    with np.errstate(over="ignore"):
        Q = np.minimum(np.ceil(2.0 ** 32 / eps), 2.0 ** 32).astype(np.uint64)
    Q[:1000] = 1 << 32
    q = (Q - np.uint64(1)).astype(np.uint32)
    m = g.integers(1, 40, q.size).astype(np.uint64)
    m[-2000:] = g.integers(1, 3, 2000)                        # n = e_m < 2^21
    n = ((m << np.uint64(32)) + Q - np.uint64(1)) // Q        # firing epochs
    n[: 50_000] += np.uint64(1)                               # mostly not firing
    n = n.astype(np.uint32)
    assert int(n.max()) < 2 ** 21 and int(n.max()) * neg < 2 ** 32
    want = negatives_per_firing_exact(q, n, neg)
    tq = torch.from_numpy(q.view(np.int32)).cuda()
    tn = torch.from_numpy(n.view(np.int32)).cuda()
    out = torch.empty(q.size, dtype=torch.int32, device="cuda")
    rc = ub.lib().umap_sgd_negatives_per_firing_device(C.c_void_p(tq.data_ptr()), C.c_void_p(tn.data_ptr()), q.size,
                                                       neg, C.c_void_p(out.data_ptr()))
    assert rc == 0, ub.lib().umap_last_error()
    got = out.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, want), np.flatnonzero(got != want)[:10]
    assert (want[50_000:] > 0).mean() > 0.99
