"""Embedding quality scores used to compare two UMAP embeddings of the same input.

The reference computes no quality metric, so both scores are defined here and applied
identically to every embedding being compared:

* ``knn_recall``: for each scored point i, the overlap between the non-self members of
  its input kNN list (the high-dimensional neighbours) and its nearest neighbours in the
  embedding (same count, self excluded), divided by that count, averaged over points.
  With k = 15 (self first) this is the overlap of 14-element sets ("15-NN recall").
  Rows containing NaN (disconnected vertices) are skipped.
* ``fuzzy_cross_entropy``: sum over the optimised edges (head, tail, weight w) of
  w log(w/q) + (1-w) log((1-w)/(1-q)), plus sum over a fixed seeded set of 5*E random
  vertex pairs of -log(1-q), with q = 1 / (1 + a d^(2b)), clamped to [1e-12, 1-1e-12].
"""
from __future__ import annotations

import numpy as np

EPS = 1e-12


def _nn_lowdim_numpy(emb: np.ndarray, rows: np.ndarray, m: int, chunk: int = 2048) -> np.ndarray:
    e = emb.astype(np.float64)
    sq = (e * e).sum(1)
    out = np.empty((len(rows), m), np.int64)
    for s in range(0, len(rows), chunk):
        r = rows[s:s + chunk]
        D = sq[r, None] + sq[None, :] - 2.0 * (e[r] @ e.T)
        D[np.arange(len(r)), r] = np.inf
        D[~np.isfinite(D)] = np.inf
        idx = np.argpartition(D, m - 1, axis=1)[:, :m]
        out[s:s + chunk] = idx
    return out


def _nn_lowdim_torch(emb: np.ndarray, rows: np.ndarray, m: int, chunk: int = 4096) -> np.ndarray:
    import torch
    e = torch.from_numpy(np.ascontiguousarray(emb, np.float32)).cuda().double()
    e = torch.nan_to_num(e, nan=1e30)
    sq = (e * e).sum(1)
    rr = torch.from_numpy(rows).cuda()
    out = torch.empty((len(rows), m), dtype=torch.int64, device="cuda")
    chunk = max(1, min(chunk, int(4e9 // (8 * e.shape[0]))))  # distance block of at most ~4 GB
    for s in range(0, len(rows), chunk):
        r = rr[s:s + chunk]
        D = sq[r, None] + sq[None, :] - 2.0 * (e[r] @ e.T)
        D[torch.arange(len(r), device="cuda"), r] = float("inf")
        out[s:s + chunk] = torch.topk(D, m, dim=1, largest=False).indices
    return out.cpu().numpy()


def knn_recall(emb: np.ndarray, knn_indices: np.ndarray, sample: int | None = None, seed: int = 0,
               use_torch: bool | None = None) -> float:
    n = emb.shape[0]
    rows = np.arange(n)
    if sample is not None and sample < n:
        rows = np.sort(np.random.Generator(np.random.PCG64(seed)).choice(n, sample, replace=False))
    ok = ~np.isnan(emb[rows]).any(1)
    rows = rows[ok]
    knn = np.asarray(knn_indices)[rows].astype(np.int64)
    m = knn.shape[1] - 1 if (knn[:, 0] == rows).all() else knn.shape[1]
    if use_torch is None:
        try:
            import torch
            use_torch = torch.cuda.is_available()
        except Exception:
            use_torch = False
    low = (_nn_lowdim_torch if use_torch else _nn_lowdim_numpy)(emb, rows, m)
    total = 0
    for i in range(len(rows)):
        hi = knn[i]
        hi = hi[hi != rows[i]][:m]
        total += len(np.intersect1d(hi, low[i], assume_unique=False))
    return total / (m * len(rows))


def fuzzy_cross_entropy(emb: np.ndarray, head: np.ndarray, tail: np.ndarray, weight: np.ndarray,
                        a: float, b: float, neg_factor: int = 5, seed: int = 0) -> float:
    emb = emb.astype(np.float64)
    head = np.asarray(head, np.int64)
    tail = np.asarray(tail, np.int64)
    w = np.asarray(weight, np.float64)
    ok = ~(np.isnan(emb[head]).any(1) | np.isnan(emb[tail]).any(1))
    head, tail, w = head[ok], tail[ok], w[ok]

    def q_of(i, j):
        d2 = ((emb[i] - emb[j]) ** 2).sum(1)
        q = 1.0 / (1.0 + a * np.power(d2, b))
        return np.clip(q, EPS, 1.0 - EPS)

    q = q_of(head, tail)
    with np.errstate(divide="ignore", invalid="ignore"):
        pos = np.where(w > 0, w * np.log(np.clip(w, EPS, 1) / q), 0.0)
        neg = np.where(w < 1, (1 - w) * np.log(np.clip(1 - w, EPS, 1) / (1 - q)), 0.0)
    g = np.random.Generator(np.random.PCG64(seed))
    n = emb.shape[0]
    m = neg_factor * len(head)
    ri = g.integers(0, n, m)
    rj = g.integers(0, n, m)
    keep = (ri != rj) & ~(np.isnan(emb[ri]).any(1) | np.isnan(emb[rj]).any(1))
    qr = q_of(ri[keep], rj[keep])
    return float(pos.sum() + neg.sum() + (-np.log(1.0 - qr)).sum())


def fuzzy_cross_entropy_torch(emb, head, tail, weight, a: float, b: float, neg_factor: int = 5, seed: int = 0,
                              chunk: int = 1 << 24) -> float:
    """``fuzzy_cross_entropy`` evaluated on the GPU in float64 (same definition; the random
    pairs come from a seeded torch generator, so the value differs from the numpy scorer's
    by the sampling of the non-edge pairs only)."""
    import torch
    dev = "cuda"
    e = torch.as_tensor(np.asarray(emb) if not hasattr(emb, "is_cuda") else emb).to(dev, torch.float64)
    h = torch.as_tensor(np.asarray(head, np.int64) if not hasattr(head, "is_cuda") else head).to(dev, torch.int64)
    t = torch.as_tensor(np.asarray(tail, np.int64) if not hasattr(tail, "is_cuda") else tail).to(dev, torch.int64)
    w = torch.as_tensor(np.asarray(weight) if not hasattr(weight, "is_cuda") else weight).to(dev, torch.float64)
    bad = torch.isnan(e).any(1)
    ok = ~(bad[h] | bad[t])
    h, t, w = h[ok], t[ok], w[ok]

    def q_of(i, j):
        d2 = ((e[i] - e[j]) ** 2).sum(1)
        return torch.clamp(1.0 / (1.0 + a * torch.pow(d2, b)), EPS, 1.0 - EPS)

    total = 0.0
    for s in range(0, h.numel(), chunk):
        q = q_of(h[s:s + chunk], t[s:s + chunk])
        ww = w[s:s + chunk]
        pos = torch.where(ww > 0, ww * torch.log(torch.clamp(ww, EPS, 1.0) / q), torch.zeros_like(q))
        neg = torch.where(ww < 1, (1 - ww) * torch.log(torch.clamp(1 - ww, EPS, 1.0) / (1 - q)), torch.zeros_like(q))
        total += float(pos.sum() + neg.sum())
    g = torch.Generator(device=dev).manual_seed(seed)
    n = e.shape[0]
    m = neg_factor * h.numel()
    for s in range(0, m, chunk):
        c = min(chunk, m - s)
        ri = torch.randint(0, n, (c,), device=dev, generator=g)
        rj = torch.randint(0, n, (c,), device=dev, generator=g)
        keep = (ri != rj) & ~(bad[ri] | bad[rj])
        total += float((-torch.log(1.0 - q_of(ri[keep], rj[keep]))).sum())
    return total


def pruned_edges(manifold, total_epochs: int):
    """(head, tail, weight) of the graph edges an optimiser for `total_epochs` keeps
    (weight >= max weight / total_epochs, or the 500 / 200 default when total_epochs <= 10;
    optimizer.rs:90-117), as host arrays."""
    g = manifold.graph()
    indptr = np.asarray(g.indptr, np.int64)
    w = np.asarray(g.data, np.float32)
    n = len(indptr) - 1
    epochs = total_epochs if total_epochs > 10 else (500 if n <= 10000 else 200)
    thr = np.float32(max(float(w.max()), 0.0) / np.float32(epochs)) if w.size else np.float32(0)
    keep = w >= thr
    head = np.repeat(np.arange(len(indptr) - 1, dtype=np.int64), np.diff(indptr))
    return head[keep], np.asarray(g.indices, np.int64)[keep], w[keep]
