"""TEST INFRASTRUCTURE ONLY: a CPU (numpy) restatement of the warm-start MLP, used by the
tests to check the GPU forward, backward and Adam kernels.  Nothing in the product imports it.

The reference has no network (its caller supplies the initial embedding, umap-rs
src/embedding.rs:274); this oracle states the network's own mathematics:

  x' = bf16((x - shift) * scale)
  z1 = x' W1^T + b1,   h1 = bf16(gelu(z1))          (W* used as bf16(W*))
  z2 = h1 W2^T + b2,   h2 = bf16(gelu(z2))
  y  = h2 W3^T + b3,   loss = sum((y - t)^2) / (rows * out)
  dy = 2 (y - t) / (rows * out)
  dz2 = (dy W3) * gelu'(z2)          db2 = sum_rows dz2 (before rounding),  dW3 = dy^T h2
  dz1 = (bf16(dz2) W2) * gelu'(z1)   db1 = sum_rows dz1 (before rounding),  dW2 = bf16(dz2)^T h1
  dW1 = bf16(dz1)^T x'               db3 = sum_rows dy

gelu(x) = x * Phi(x) with the exact normal CDF; gelu'(x) = Phi(x) + x * phi(x).  With
`bf16=False` every rounding is dropped and float64 is used throughout: that form is checked
against central finite differences, which pins the derivative formulas above.
Flat parameter order: W1 [256, in], b1 [256], W2 [256, 256], b2 [256], W3 [out, 256], b3 [out].
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

HIDDEN = 256


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)


def unpack(params: np.ndarray, in_dim: int, out_dim: int, hidden: int = HIDDEN):
    o = 0
    out = []
    for rows, cols in ((hidden, in_dim), (hidden, 0), (hidden, hidden), (hidden, 0), (out_dim, hidden), (out_dim, 0)):
        n = rows * cols if cols else rows
        a = params[o:o + n]
        out.append(a.reshape(rows, cols) if cols else a)
        o += n
    assert o == params.size, (o, params.size)
    return out


def pack(parts) -> np.ndarray:
    return np.concatenate([np.asarray(p).ravel() for p in parts])


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def forward_backward(params, X, T, in_dim, out_dim, shift=None, scale=None, bf16=True, hidden=HIDDEN):
    """Returns (loss, flat gradients, y).  bf16=True mirrors the GPU's rounding points
    (products in float64, each result rounded to float32 like an fp32 accumulator)."""
    if bf16:
        f = lambda a: np.asarray(a, dtype=np.float32)  # noqa: E731
        r = bf16_round
    else:
        f = lambda a: np.asarray(a, dtype=np.float64)  # noqa: E731
        r = lambda a: np.asarray(a, dtype=np.float64)  # noqa: E731
    mm = lambda a, b: f(np.asarray(a, np.float64) @ np.asarray(b, np.float64))  # noqa: E731
    W1, b1, W2, b2, W3, b3 = unpack(np.asarray(params), in_dim, out_dim, hidden)
    W1b, W2b, W3b = r(W1), r(W2), r(W3)
    x = f(X)
    if scale is not None:
        x = f((x - f(shift)) * f(scale))
    xb = r(x)
    z1 = f(mm(xb, W1b.T) + f(b1))
    h1 = r(f(gelu(np.asarray(z1, np.float64))))
    z2 = f(mm(h1, W2b.T) + f(b2))
    h2 = r(f(gelu(np.asarray(z2, np.float64))))
    y = f(mm(h2, W3b.T) + f(b3))
    rows = X.shape[0]
    e = f(y - f(T))
    loss = float(np.sum(np.asarray(e, np.float64) ** 2) / (rows * out_dim))
    dy = f(2.0 * e / (rows * out_dim))
    dz2 = f(mm(dy, W3b) * gelu_grad(np.asarray(z2, np.float64)))
    dz2b = r(dz2)
    dz1 = f(mm(dz2b, W2b) * gelu_grad(np.asarray(z1, np.float64)))
    dz1b = r(dz1)
    grads = pack([mm(dz1b.T, xb), dz1.sum(0, dtype=np.float64), mm(dz2b.T, h1), dz2.sum(0, dtype=np.float64),
                  mm(dy.T, h2), dy.sum(0, dtype=np.float64)])
    return loss, f(grads), y


def loss_only(params, X, T, in_dim, out_dim, hidden=HIDDEN):
    return forward_backward(params, X, T, in_dim, out_dim, bf16=False, hidden=hidden)[0]


def adam_step(w, m, v, g, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (Kingma & Ba 2015, bias-corrected) in float32; returns (w, m, v)."""
    w, m, v, g = (np.asarray(a, np.float32) for a in (w, m, v, g))
    m = np.float32(b1) * m + np.float32(1 - b1) * g
    v = np.float32(b2) * v + np.float32(1 - b2) * g * g
    c1 = np.float32(1 - b1 ** t)
    c2 = np.float32(1 - b2 ** t)
    w = w - np.float32(lr) * (m / c1) / (np.sqrt(v / c2) + np.float32(eps))
    return w.astype(np.float32), m, v
