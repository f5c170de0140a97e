"""Seeded synthetic workloads for the UMAP fit path, and an exact kNN producer.

No public dataset is used.  Each generator reproduces the shapes, sizes and value
distributions of one benchmark configuration of the fit path:

* ``gaussians_10k``   n=10,000, D=32, 10 isotropic Gaussians (centres ~N(0, 5^2 I), std 1,
  equal weights), seed 0; 200 epochs.
* ``gaussians_2m``    n=2,000,000, D=64, 50 anisotropic Gaussians (centres ~N(0, 8^2 I),
  per-cluster diagonal std ~U[0.5, 2], Dirichlet(1) weights), seed 1; 500 epochs.
* ``swiss_roll``      3-D noisy swiss roll (t~U[1.5pi, 4.5pi], height~U[0, 20], noise std
  0.05), seed 2.
* ``instances``       many independent datasets, sizes log-uniform in [500, 50,000], D=32,
  5 Gaussians each (centres ~N(0, 5^2 I), std 1), per-instance seed.

Every workload's kNN is exact (self first at distance 0): candidates come from a
||x||^2 + ||y||^2 - 2 x.y distance matrix, then the final k distances are recomputed
directly in f32 as sqrt(sum((x - y)^2)) and sorted by (distance, index).  A per-row
certificate checks that no point outside the candidate list can beat the k-th
neighbour; rows that fail it are redone by direct brute force.

Init is uniform in [-10, 10]^dim (f32), like the reference's random-init examples.
"""
from __future__ import annotations

import math

import numpy as np


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def gaussian_mixture(n: int, d: int, n_clusters: int, centre_std: float, seed: int,
                     anisotropic: bool = False, dirichlet: bool = False):
    """Returns (X f32[n, d], labels i32[n])."""
    g = _rng(seed)
    centres = g.normal(0.0, centre_std, size=(n_clusters, d))
    if anisotropic:
        stds = g.uniform(0.5, 2.0, size=(n_clusters, d))
    else:
        stds = np.ones((n_clusters, d))
    if dirichlet:
        w = g.dirichlet(np.ones(n_clusters))
    else:
        w = np.full(n_clusters, 1.0 / n_clusters)
    labels = g.choice(n_clusters, size=n, p=w).astype(np.int32)
    X = np.empty((n, d), np.float32)
    chunk = 1 << 20
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        lab = labels[s:e]
        X[s:e] = (centres[lab] + g.standard_normal((e - s, d)) * stds[lab]).astype(np.float32)
    return X, labels


def gaussians_10k():
    return gaussian_mixture(10_000, 32, 10, 5.0, seed=0)


def gaussians_2m(n: int = 2_000_000):
    return gaussian_mixture(n, 64, 50, 8.0, seed=1, anisotropic=True, dirichlet=True)


def digits_like(n: int = 70_000, side: int = 28, n_classes: int = 10, seed: int = 5):
    """Synthetic stand-in with MNIST's shape and value distribution (no dataset is read):
    n images of side x side pixels in [0, 1], mostly zero.  Each class is a prototype of a few
    Gaussian strokes; a sample is its prototype shifted by up to 2 pixels, scaled in
    intensity, with pixel noise, clipped to [0, 1] and zeroed below 0.2.  Returns
    (X f32[n, side * side], labels i32[n])."""
    g = _rng(seed)
    yy, xx = np.mgrid[0:side, 0:side].astype(np.float32)
    protos = np.zeros((n_classes, side, side), np.float32)
    for c in range(n_classes):
        for _ in range(g.integers(3, 7)):
            cy, cx = g.uniform(6, side - 6, 2)
            sy, sx = g.uniform(1.0, 4.0, 2)
            protos[c] += np.exp(-((yy - cy) ** 2 / (2 * sy * sy) + (xx - cx) ** 2 / (2 * sx * sx)))
        protos[c] /= protos[c].max()
    labels = g.integers(0, n_classes, n).astype(np.int32)
    X = np.empty((n, side * side), np.float32)
    chunk = 8192
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        m = e - s
        sh = g.integers(-2, 3, (m, 2))
        img = np.empty((m, side, side), np.float32)
        for i in range(m):
            img[i] = np.roll(protos[labels[s + i]], (sh[i, 0], sh[i, 1]), axis=(0, 1))
        img *= g.uniform(0.6, 1.0, (m, 1, 1)).astype(np.float32)
        img += g.normal(0, 0.1, img.shape).astype(np.float32)
        np.clip(img, 0.0, 1.0, out=img)
        img[img < 0.2] = 0.0
        X[s:e] = img.reshape(m, -1)
    return X, labels


def swiss_roll(n: int, seed: int = 2):
    g = _rng(seed)
    t = g.uniform(1.5 * math.pi, 4.5 * math.pi, size=n)
    h = g.uniform(0.0, 20.0, size=n)
    X = np.stack([t * np.cos(t), h, t * np.sin(t)], axis=1)
    X += g.normal(0.0, 0.05, size=X.shape)
    return X.astype(np.float32), t.astype(np.float32)


def instance_sizes(count: int = 4096, lo: int = 500, hi: int = 50_000, seed: int = 4):
    g = _rng(seed)
    return np.exp(g.uniform(math.log(lo), math.log(hi), size=count)).astype(np.int64)


def instance(i: int, n: int, seed_base: int = 1000):
    return gaussian_mixture(int(n), 32, 5, 5.0, seed=seed_base + i)


def uniform_init(n: int, dim: int = 2, seed: int = 0) -> np.ndarray:
    g = _rng(10_000 + seed)
    return g.uniform(-10.0, 10.0, size=(n, dim)).astype(np.float32)


# ------------------------------------------------------------------ exact kNN
def _finalize_rows(X, rows, cand, k):
    """Exact f32 distances for candidate lists, sorted by (distance, index), k kept."""
    xi = X[rows][:, None, :]
    xc = X[cand]
    d = np.sqrt(((xi - xc) ** 2).sum(axis=2, dtype=np.float32)).astype(np.float32)
    o1 = np.argsort(cand, axis=1, kind="stable")
    cand = np.take_along_axis(cand, o1, 1)
    d = np.take_along_axis(d, o1, 1)
    o2 = np.argsort(d, axis=1, kind="stable")
    cand = np.take_along_axis(cand, o2, 1)
    d = np.take_along_axis(d, o2, 1)
    return cand[:, :k], d[:, :k]


def knn_exact_numpy(X: np.ndarray, k: int, margin: int = 8, chunk: int = 1024):
    """Exact kNN on the CPU (f64 distance matrix for candidates)."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    n = X.shape[0]
    X64 = X.astype(np.float64)
    sq = (X64 * X64).sum(1)
    kc = min(n, k + margin)
    idx = np.empty((n, k), np.uint32)
    dst = np.empty((n, k), np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        D = sq[s:e, None] + sq[None, :] - 2.0 * (X64[s:e] @ X64.T)
        D[np.arange(e - s), np.arange(s, e)] = -1.0  # self first
        cand = np.argpartition(D, kc - 1, axis=1)[:, :kc]
        ci, cd = _finalize_rows(X, np.arange(s, e), cand, k)
        idx[s:e] = ci
        dst[s:e] = cd
    return idx, dst


def knn_exact_torch(X: np.ndarray, k: int, device="cuda", margin: int = 8, chunk: int = 2048):
    """Exact kNN with torch on the GPU (harness-side producer, not part of the fit path).

    Candidates: top-(k+margin) of the fp32 (TF32 off) expansion distance.  Exactness
    certificate per row: the (k+margin)-th candidate's approximate squared distance minus
    an fp32 rounding bound must exceed the exact k-th squared distance; failing rows are
    recomputed by direct brute force."""
    import torch

    torch.backends.cuda.matmul.allow_tf32 = False
    X0 = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).to(device)
    Xt = X0 - X0.mean(0, keepdim=True)   # centred copy: candidate search only
    n, dim = Xt.shape
    sq = (Xt * Xt).sum(1)
    kc = min(n, k + margin)
    idx = torch.empty((n, k), dtype=torch.int64, device=device)
    dst = torch.empty((n, k), dtype=torch.float32, device=device)
    bad_rows = []
    eps = 4.0 * dim * 2.0 ** -23
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        D = sq[s:e, None] + sq[None, :] - 2.0 * (Xt[s:e] @ Xt.T)
        ar = torch.arange(e - s, device=device)
        D[ar, ar + s] = -1.0
        vals, cand = torch.topk(D, kc, dim=1, largest=False, sorted=True)
        xc = X0[cand]                                   # [m, kc, dim]
        ex = torch.sqrt(((X0[s:e, None, :] - xc) ** 2).sum(2))
        # sort by (distance, index): stable sort on index first, then distance
        o1 = torch.argsort(cand, dim=1, stable=True)
        cand = torch.gather(cand, 1, o1)
        ex = torch.gather(ex, 1, o1)
        o2 = torch.argsort(ex, dim=1, stable=True)
        cand = torch.gather(cand, 1, o2)
        ex = torch.gather(ex, 1, o2)
        idx[s:e] = cand[:, :k]
        dst[s:e] = ex[:, :k]
        if kc < n:
            bound = eps * (sq[s:e] + sq[cand[:, kc - 1]] + 1.0)
            kth = ex[:, k - 1] ** 2
            bad = (vals[:, kc - 1] - bound) <= kth * (1.0 + 1e-6)
            if bool(bad.any()):
                bad_rows.extend((torch.nonzero(bad).flatten() + s).tolist())
    for r in bad_rows:
        d = torch.sqrt(((X0 - X0[r]) ** 2).sum(1))
        d[r] = -1.0
        v, c = torch.topk(d, kc, largest=False, sorted=True)
        o1 = torch.argsort(c, stable=True)
        c, v = c[o1], v[o1]
        o2 = torch.argsort(v, stable=True)
        c, v = c[o2], v[o2]
        v[c == r] = 0.0
        idx[r] = c[:k]
        dst[r] = v[:k]
    return idx.to(torch.int32).cpu().numpy().astype(np.uint32), dst.cpu().numpy(), len(bad_rows)


def knn_exact_gpu(X: np.ndarray, k: int, device="cuda"):
    """Exact kNN with the point itself first (self + k - 1 others), the others from the
    library's tensor-core brute force (umap_knn_bruteforce: the reference example's f32
    distance, ties in index order).  Returns (idx u32[n,k], dist f32[n,k], rows recomputed)."""
    import torch
    import umap_b200 as ub
    n = X.shape[0]
    t = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).to(device)
    i, d, rec = ub.knn_bruteforce(t, k - 1, return_stats=True)
    idx = np.empty((n, k), np.uint32)
    dist = np.zeros((n, k), np.float32)
    idx[:, 0] = np.arange(n, dtype=np.uint32)
    idx[:, 1:] = i.cpu().numpy().view(np.uint32)
    dist[:, 1:] = d.cpu().numpy()
    return idx, dist, rec


def _torch_knn_block(torch, Xq0, Xq, Xc0, Xc, sqq, sqc, k, kc, self_offset):
    """Top-(k) exact neighbours of query rows among candidate rows (both on the GPU).
    X*0 are the original coordinates (exact distances), X* the centred copies (search)."""
    D = sqq[:, None] + sqc[None, :] - 2.0 * (Xq @ Xc.T)
    if self_offset is not None:
        ar = torch.arange(Xq.shape[0], device=Xq.device)
        D[ar, ar + self_offset] = -1.0
    vals, cand = torch.topk(D, kc, dim=1, largest=False, sorted=True)
    ex = torch.sqrt(((Xq0[:, None, :] - Xc0[cand]) ** 2).sum(2))
    o1 = torch.argsort(cand, dim=1, stable=True)
    cand = torch.gather(cand, 1, o1)
    ex = torch.gather(ex, 1, o1)
    o2 = torch.argsort(ex, dim=1, stable=True)
    return torch.gather(cand, 1, o2)[:, :k], torch.gather(ex, 1, o2)[:, :k], vals[:, kc - 1]


def knn_exact_clustered_torch(X: np.ndarray, labels: np.ndarray, k: int, device="cuda",
                              margin: int = 8, chunk: int = 4096):
    """Exact kNN for clustered data: search inside each cluster, then certify every row.

    Certificate for row x in cluster A: for every other cluster B, ||x - c_B|| - R_B (c_B
    the cluster mean, R_B its radius) must exceed the k-th neighbour distance found in A,
    so no point outside A can be closer.  The in-cluster candidate list is certified like
    knn_exact_torch.  Rows failing either test are recomputed by global brute force.
    Returns (idx u32[n,k], dist f32[n,k], n_recomputed)."""
    import torch

    torch.backends.cuda.matmul.allow_tf32 = False
    n, dim = X.shape
    X0 = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).to(device)
    lab = torch.from_numpy(np.ascontiguousarray(labels, dtype=np.int64)).to(device)
    idx = torch.empty((n, k), dtype=torch.int64, device=device)
    dst = torch.empty((n, k), dtype=torch.float32, device=device)
    bad = torch.zeros(n, dtype=torch.bool, device=device)
    eps = 4.0 * dim * 2.0 ** -23
    C = int(labels.max()) + 1
    centres = torch.zeros((C, dim), dtype=torch.float64, device=device)
    radius = torch.zeros(C, dtype=torch.float64, device=device)
    for c in range(C):
        members = torch.nonzero(lab == c).flatten()
        if members.numel() == 0:
            continue
        Xc0 = X0[members]
        centres[c] = Xc0.double().mean(0)
        radius[c] = torch.sqrt(((Xc0.double() - centres[c]) ** 2).sum(1)).max()
        mu = Xc0.mean(0, keepdim=True)
        Xc = Xc0 - mu
        sq = (Xc * Xc).sum(1)
        m = members.numel()
        kc = min(m, k + margin)
        for s in range(0, m, chunk):
            e = min(m, s + chunk)
            ci, cd, last = _torch_knn_block(torch, Xc0[s:e], Xc[s:e], Xc0, Xc, sq[s:e], sq, min(k, kc), kc, s)
            gi = members[ci]
            if ci.shape[1] < k:
                bad[members[s:e]] = True
                continue
            idx[members[s:e]] = gi
            dst[members[s:e]] = cd
            if kc < m:
                bound = eps * (sq[s:e] + sq.max() + 1.0)
                bad[members[s:e]] |= (last - bound) <= cd[:, k - 1] ** 2 * (1.0 + 1e-6)
            else:
                pass
    # cross-cluster certificate
    for s in range(0, n, 1 << 18):
        e = min(n, s + (1 << 18))
        dc = torch.cdist(X0[s:e].double(), centres) - radius[None, :]
        dc[torch.arange(e - s, device=device), lab[s:e]] = float("inf")
        bad[s:e] |= dc.min(1).values <= dst[s:e, k - 1].double() * (1.0 + 1e-6) + 1e-6
    bad_rows = torch.nonzero(bad).flatten()
    Xg = X0 - X0.mean(0, keepdim=True)
    sqg = (Xg * Xg).sum(1)
    for s in range(0, bad_rows.numel(), 1024):
        r = bad_rows[s:s + 1024]
        D = sqg[r, None] + sqg[None, :] - 2.0 * (Xg[r] @ Xg.T)
        D[torch.arange(r.numel(), device=device), r] = -1.0
        kc = min(n, k + 64)
        _, cand = torch.topk(D, kc, dim=1, largest=False, sorted=True)
        ex = torch.sqrt(((X0[r][:, None, :] - X0[cand]) ** 2).sum(2))
        o1 = torch.argsort(cand, dim=1, stable=True)
        cand = torch.gather(cand, 1, o1)
        ex = torch.gather(ex, 1, o1)
        o2 = torch.argsort(ex, dim=1, stable=True)
        idx[r] = torch.gather(cand, 1, o2)[:, :k]
        dst[r] = torch.gather(ex, 1, o2)[:, :k]
    return (idx.to(torch.int32).cpu().numpy().astype(np.uint32), dst.cpu().numpy(),
            int(bad_rows.numel()))


def instances_torch(count: int = 4096, k: int = 15, seed: int = 4, device="cuda", lo=500, hi=50_000,
                    which: range | None = None):
    """The batched workload on the GPU: `count` datasets with sizes log-uniform in [lo, hi],
    each D=32, 5 Gaussians (centres ~N(0, 5^2 I), std 1), per-instance seed; exact kNN k
    (self first, local ids) by brute force per instance; init U[-10, 10]^2.  `which` (a
    range of instance ids) generates only those instances, exactly as in the full set.
    Returns (sizes i64[m], idx i32 CUDA [N, k], dist f32 CUDA [N, k], init f32 CUDA [N, 2])."""
    import torch

    torch.backends.cuda.matmul.allow_tf32 = False
    all_sizes = instance_sizes(count, lo, hi, seed)
    which = range(count) if which is None else which
    sizes = all_sizes[which.start:which.stop]
    N = int(sizes.sum())
    idx = torch.empty((N, k), dtype=torch.int32, device=device)
    dst = torch.empty((N, k), dtype=torch.float32, device=device)
    off = 0
    for i, n in zip(which, sizes.tolist()):
        g = torch.Generator(device=device).manual_seed(1000 + i)
        centres = torch.randn((5, 32), generator=g, device=device) * 5.0
        lab = torch.randint(0, 5, (n,), generator=g, device=device)
        X0 = centres[lab] + torch.randn((n, 32), generator=g, device=device)
        Xc = X0 - X0.mean(0, keepdim=True)
        sq = (Xc * Xc).sum(1)
        kc = min(n, k + 8)
        for s in range(0, n, 4096):
            e = min(n, s + 4096)
            ci, cd, _ = _torch_knn_block(torch, X0[s:e], Xc[s:e], X0, Xc, sq[s:e], sq, k, kc, s)
            idx[off + s:off + e] = ci.to(torch.int32)
            dst[off + s:off + e] = cd
        off += n
    g = torch.Generator(device=device).manual_seed(77)
    init = torch.rand((int(all_sizes.sum()), 2), generator=g, device=device) * 20.0 - 10.0
    first = int(all_sizes[:which.start].sum())
    init = init[first:first + N].contiguous()
    return sizes, idx, dst, init


# ------------------------------------------------------------------ 100M-point swiss roll
def swiss_roll_torch(n: int, seed: int = 2, device="cuda"):
    """``swiss_roll`` generated on the GPU in chunks (t~U[1.5pi, 4.5pi], height~U[0, 20],
    Gaussian noise std 0.05); returns f32 CUDA [n, 3]."""
    import torch
    X = torch.empty((n, 3), dtype=torch.float32, device=device)
    g = torch.Generator(device=device).manual_seed(seed)
    chunk = 1 << 24
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        m = e - s
        t = torch.rand(m, generator=g, device=device, dtype=torch.float64) * (3.0 * math.pi) + 1.5 * math.pi
        h = torch.rand(m, generator=g, device=device, dtype=torch.float64) * 20.0
        P = torch.stack([t * torch.cos(t), h, t * torch.sin(t)], dim=1)
        P += torch.randn((m, 3), generator=g, device=device, dtype=torch.float64) * 0.05
        X[s:e] = P.to(torch.float32)
    return X


def _grid_keys(torch, X, lo, h, dims):
    c = torch.floor((X - lo) / h).to(torch.int64)
    c = torch.minimum(torch.clamp(c, min=0), dims - 1)
    return (c[:, 0] * dims[1] + c[:, 1]) * dims[2] + c[:, 2], c


def _grid_pass(torch, X, rows, k, h, chunk):
    """Candidates from the 27 cells around each query row on a grid of cell size h.
    Returns (idx [m, k] int64, dist [m, k] f32, certified [m] bool): a row is certified when
    its k-th distance is <= h, so no point outside the 27 cells can be closer."""
    dev = X.device
    lo = X.min(0).values
    dims = (torch.floor((X.max(0).values - lo) / h).to(torch.int64) + 1)
    keys, _ = _grid_keys(torch, X, lo, h, dims)
    keys_sorted, order = torch.sort(keys)
    uniq, counts = torch.unique_consecutive(keys_sorted, return_counts=True)
    starts = torch.cumsum(counts, 0) - counts
    M = int(counts.max())
    Xs = X[order]
    offs = torch.tensor([(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)],
                        dtype=torch.int64, device=dev)
    ar = torch.arange(M, device=dev)
    m = rows.numel()
    out_i = torch.empty((m, k), dtype=torch.int64, device=dev)
    out_d = torch.empty((m, k), dtype=torch.float32, device=dev)
    q_chunk = max(1024, min(chunk, int(2e8 // (27 * M))))
    for s in range(0, m, q_chunk):
        e = min(m, s + q_chunk)
        q = X[rows[s:e]]
        _, qc = _grid_keys(torch, q, lo, h, dims)
        nc = qc[:, None, :] + offs[None, :, :]                                   # [Q, 27, 3]
        inside = ((nc >= 0) & (nc < dims)).all(-1)
        nk = (nc[..., 0] * dims[1] + nc[..., 1]) * dims[2] + nc[..., 2]
        pos = torch.searchsorted(uniq, nk).clamp(max=uniq.numel() - 1)
        found = inside & (uniq[pos] == nk)
        cnt = torch.where(found, counts[pos], torch.zeros_like(pos))
        cand = starts[pos][..., None] + ar                                       # [Q, 27, M]
        valid = ar < cnt[..., None]
        cand = torch.where(valid, cand, torch.zeros_like(cand)).reshape(e - s, -1)
        valid = valid.reshape(e - s, -1)
        diff = Xs[cand] - q[:, None, :]
        d2 = (diff * diff).sum(-1)
        d2 = torch.where(valid, d2, torch.full_like(d2, float("inf")))
        kk = min(k, d2.shape[1])
        vals, p = torch.topk(d2, kk, dim=1, largest=False, sorted=True)
        gid = order[torch.gather(cand, 1, p)]
        out_i[s:e, :kk] = gid
        out_d[s:e, :kk] = torch.sqrt(vals)
        if kk < k:
            out_i[s:e, kk:] = 0
            out_d[s:e, kk:] = float("inf")
    ok = out_d[:, k - 1] <= h
    return out_i, out_d, ok


def knn_grid_torch(X, k: int, chunk: int = 1 << 17, occupancy: float = 6.0):
    """Exact kNN (self first at distance 0) of low-dimensional points (CUDA f32 [n, d]) with
    a uniform grid: each query searches the 3^d cells around its own.  The cell size is set
    so that occupied cells hold about `occupancy` points; rows whose k-th distance exceeds
    the cell size are redone on a grid with twice the cell size until every row is
    certified.  Returns (idx int32 CUDA [n, k], dist f32 CUDA [n, k], rows redone)."""
    import torch
    n, d = X.shape
    lo = X.min(0).values
    ext = (X.max(0).values - lo).clamp(min=1e-6)
    h = float((ext.prod() / max(n, 1) * occupancy) ** (1.0 / d))
    for _ in range(8):  # refine h towards the target occupancy of occupied cells
        dims = (torch.floor(ext / h).to(torch.int64) + 1)
        keys, _ = _grid_keys(torch, X, lo, h, dims)
        occ = n / float(torch.unique(keys).numel())
        if 0.7 * occupancy <= occ <= 1.4 * occupancy:
            break
        h *= (occupancy / occ) ** (1.0 / d)
        del keys
    rows = torch.arange(n, device=X.device)
    idx = torch.empty((n, k), dtype=torch.int32, device=X.device)
    dst = torch.empty((n, k), dtype=torch.float32, device=X.device)
    redone = 0
    first = True
    while rows.numel():
        oi, od, ok = _grid_pass(torch, X, rows, k, h, chunk)
        idx[rows[ok]] = oi[ok].to(torch.int32)
        dst[rows[ok]] = od[ok]
        rows = rows[~ok]
        if not first:
            redone += int(ok.sum())
        first = False
        h *= 2.0
    return idx, dst, redone
