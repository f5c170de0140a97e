"""Learned warm start (no counterpart in the reference, whose `Umap::fit` takes `init` from
the caller, embedding.rs:274).

A small MLP (in -> 256 -> 256 -> n_components, GELU; bf16 weights and activations, fp32
accumulation on the tensor cores) is trained with Adam on the plain-fit embedding of a
subsample, predicts an initial embedding for every point, and a shortened fit
(`n_epochs` = 100 by default) refines it.  The shortened fit keeps the reference's
semantics for that epoch count: `Optimizer::new` prunes at max_w / total_epochs
(optimizer.rs:96-102) and the learning rate decays from `learning_rate` over the shorter run.

Everything here runs through the library's C ABI: `umap_mlp_*` for the network (forward,
backward and Adam are the library's own kernels) and `umap_fit_device` / `umap_learn_manifold_device` + `umap_fit_manifold_device` for the
fits.  The
caller supplies the subsample's kNN, as it supplies the kNN of the full data set.
"""
from __future__ import annotations

import copy
import ctypes as C
import time

import numpy as np

from . import _lib
from . import (ERR_INVALID_ARGUMENT, FittedUmap, Umap, UmapConfig, UmapError, _check, _Handle)

HIDDEN = 256


def param_count(in_dim: int, out_dim: int) -> int:
    v = C.c_uint64()
    _check(_lib.load().umap_mlp_param_count(in_dim, out_dim, C.byref(v)))
    return v.value


def init_params(in_dim: int, out_dim: int, seed: int = 0) -> np.ndarray:
    """Flat fp32 parameters W1, b1, W2, b2, W3, b3 drawn like a default linear layer:
    U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((in_dim, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, out_dim)):
        bound = 1.0 / np.sqrt(fan_in)
        parts.append(rng.uniform(-bound, bound, size=fan_out * fan_in))
        parts.append(rng.uniform(-bound, bound, size=fan_out))
    return np.concatenate(parts).astype(np.float32)


def _cuda_f32(x, name):
    import torch
    if not (hasattr(x, "is_cuda") and x.is_cuda):
        raise UmapError(ERR_INVALID_ARGUMENT, f"{name} must be a CUDA tensor")
    t = x.contiguous()
    if t.dtype != torch.float32:
        t = t.float()
    return t


class Mlp(_Handle):
    """The warm-start network (umap_mlp_* in include/umap_b200.h)."""
    _free = "umap_mlp_free"

    @staticmethod
    def create(in_dim: int, out_dim: int, params: np.ndarray | None = None, seed: int = 0) -> "Mlp":
        if params is None:
            params = init_params(in_dim, out_dim, seed)
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != param_count(in_dim, out_dim):
            raise UmapError(ERR_INVALID_ARGUMENT, f"expected {param_count(in_dim, out_dim)} parameters, got {p.size}")
        h = C.c_void_p()
        _check(_lib.load().umap_mlp_new(in_dim, out_dim, p.ctypes.data_as(C.c_void_p), C.byref(h)))
        return Mlp(h.value)

    def dims(self):
        a, b = C.c_uint64(), C.c_uint64()
        _check(_lib.load().umap_mlp_dims(self._get(), C.byref(a), C.byref(b)))
        return a.value, b.value

    def params(self) -> np.ndarray:
        i, o = self.dims()
        out = np.empty(param_count(i, o), np.float32)
        _check(_lib.load().umap_mlp_get_params(self._get(), out.ctypes.data_as(C.c_void_p)))
        return out

    def set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        i, o = self.dims()
        if p.size != param_count(i, o):
            raise UmapError(ERR_INVALID_ARGUMENT, f"expected {param_count(i, o)} parameters, got {p.size}")
        _check(_lib.load().umap_mlp_set_params(self._get(), p.ctypes.data_as(C.c_void_p)))

    def fit_input_norm(self, x):
        x = _cuda_f32(x, "x")
        _check(_lib.load().umap_mlp_fit_input_norm_device(self._get(), C.c_void_p(x.data_ptr()), x.shape[0]))

    def input_norm(self):
        i, _ = self.dims()
        sh, sc = np.empty(i, np.float32), np.empty(i, np.float32)
        _check(_lib.load().umap_mlp_input_norm(self._get(), sh.ctypes.data_as(C.c_void_p),
                                               sc.ctypes.data_as(C.c_void_p)))
        return sh, sc

    def set_input_norm(self, shift, scale):
        sh = np.ascontiguousarray(shift, np.float32)
        sc = np.ascontiguousarray(scale, np.float32)
        _check(_lib.load().umap_mlp_set_input_norm(self._get(), sh.ctypes.data_as(C.c_void_p),
                                                   sc.ctypes.data_as(C.c_void_p)))

    def _check_shapes(self, x, y=None):
        i, o = self.dims()
        if x.dim() != 2 or x.shape[1] != i:
            raise UmapError(ERR_INVALID_ARGUMENT, f"x must be [rows, {i}], got {list(x.shape)}")
        if y is not None and (y.dim() != 2 or y.shape[1] != o or y.shape[0] != x.shape[0]):
            raise UmapError(ERR_INVALID_ARGUMENT, f"y must be [{x.shape[0]}, {o}], got {list(y.shape)}")

    def gradients(self, x, y):
        """Mean-squared-error gradients (flat parameter order) and loss of one batch."""
        x, y = _cuda_f32(x, "x"), _cuda_f32(y, "y")
        self._check_shapes(x, y)
        i, o = self.dims()
        g = np.empty(param_count(i, o), np.float32)
        loss = C.c_float()
        _check(_lib.load().umap_mlp_gradients_device(self._get(), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                                     x.shape[0], g.ctypes.data_as(C.c_void_p), C.byref(loss)))
        return g, loss.value

    def train(self, x, y, epochs: int = 20, batch: int = 4096, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        """Adam on shuffled mini-batches; returns each epoch's mean batch loss."""
        x, y = _cuda_f32(x, "x"), _cuda_f32(y, "y")
        self._check_shapes(x, y)
        losses = np.zeros(max(epochs, 1), np.float32)
        _check(_lib.load().umap_mlp_train_device(self._get(), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                                 x.shape[0], epochs, batch, lr, seed,
                                                 losses.ctypes.data_as(C.c_void_p)))
        return losses[:epochs]

    def predict(self, x):
        import torch
        x = _cuda_f32(x, "x")
        self._check_shapes(x)
        _, o = self.dims()
        y = torch.empty((x.shape[0], o), dtype=torch.float32, device=x.device)
        _check(_lib.load().umap_mlp_predict_device(self._get(), C.c_void_p(x.data_ptr()), x.shape[0],
                                                   C.c_void_p(y.data_ptr())))
        return y


def gemm_bf16(a, b, k_splits: int = 1):
    """C = A B^T on the library's tensor-core GEMM (A [m, k], B [n, k] bf16 CUDA tensors)."""
    import torch
    if a.dtype != torch.bfloat16 or b.dtype != torch.bfloat16 or not a.is_cuda or not b.is_cuda:
        raise UmapError(ERR_INVALID_ARGUMENT, "a and b must be bf16 CUDA tensors")
    a, b = a.contiguous(), b.contiguous()
    if a.shape[1] != b.shape[1]:
        raise UmapError(ERR_INVALID_ARGUMENT, "a and b must have the same k")
    c = torch.zeros((a.shape[0], b.shape[0]), dtype=torch.float32, device=a.device)
    _check(_lib.load().umap_gemm_bf16_device(C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
                                             C.c_void_p(c.data_ptr()), a.shape[0], b.shape[0], a.shape[1], k_splits))
    return c


def _pad64(x):
    """Zero-pads feature columns to a multiple of 64 (the network's input tile)."""
    import torch
    d = x.shape[1]
    if d % 64 == 0:
        return x
    return torch.nn.functional.pad(x, (0, 64 - d % 64))


def _with_epochs(config: UmapConfig, n_epochs: int, learning_rate: float | None) -> UmapConfig:
    c = copy.deepcopy(config)
    c.optimization.n_epochs = n_epochs
    if learning_rate is not None:
        c.optimization.learning_rate = learning_rate
    return c


def warm_start_fit(config: UmapConfig, data, knn_indices, knn_dists, sub_index, sub_knn_indices, sub_knn_dists,
                   *, sub_init=None, sub_epochs: int = 500, epochs: int = 100, mlp_epochs: int = 20,
                   batch: int = 4096, mlp_lr: float = 1e-3, learning_rate: float | None = None, seed: int = 0,
                   info: dict | None = None) -> FittedUmap:
    """Fit with a learned initial embedding.

    data: CUDA f32 [n, d]; knn_*: the full data set's kNN (as for `Umap.fit`); sub_index:
    CUDA int64 rows of the subsample; sub_knn_*: the subsample's own kNN (local ids).
    The subsample is fitted plainly for `sub_epochs` from `sub_init` (uniform [-10, 10]^2,
    seeded, when None); the network is trained on (data[sub_index], that embedding) for
    `mlp_epochs` epochs of Adam; its predictions initialise a fit of all points for `epochs`
    epochs.  `info`, when given, receives per-phase wall times (ms) and the loss curve.
    """
    import threading

    import torch
    data = _cuda_f32(data, "data")
    t = {}
    dev = data.device

    def mark(name, t0):
        torch.cuda.synchronize(dev)
        t[name] = (time.perf_counter() - t0) * 1e3
        return time.perf_counter()

    torch.cuda.synchronize(dev)
    t_start = t0 = time.perf_counter()
    cfg_full = _with_epochs(config, epochs, learning_rate)
    # The full graph does not depend on the initial embedding: build it on its own stream
    # (another handle, another host thread) while the subsample is fitted and the network
    # trained.
    full = {}

    def build_full_graph():
        try:
            tg = time.perf_counter()
            full["manifold"] = Umap(cfg_full).learn_manifold(data, knn_indices, knn_dists)
            full["ms"] = (time.perf_counter() - tg) * 1e3
        except BaseException as e:  # re-raised on the calling thread
            full["error"] = e

    worker = threading.Thread(target=build_full_graph, name="umap-b200-full-graph")
    worker.start()
    try:
        x = _pad64(data)
        sub = x[sub_index]
        n_sub = sub.shape[0]
        dim = config.n_components
        if sub_init is None:
            g = np.random.default_rng(seed)
            sub_init = torch.from_numpy(g.uniform(-10.0, 10.0, size=(n_sub, dim)).astype(np.float32)).to(dev)
        t0 = mark("prepare", t0)
        fitted_sub = Umap(_with_epochs(config, sub_epochs, None)).fit(sub, sub_knn_indices, sub_knn_dists, sub_init)
        y = torch.from_numpy(fitted_sub.embedding()).to(dev)
        del fitted_sub
        keep = torch.isfinite(y).all(dim=1)  # rows with an empty graph row come back NaN
        if not bool(keep.all()):
            sub, y = sub[keep].contiguous(), y[keep].contiguous()
        t0 = mark("subsample_fit", t0)
        net = Mlp.create(x.shape[1], dim, seed=seed)
        net.fit_input_norm(sub)
        losses = net.train(sub, y, epochs=mlp_epochs, batch=min(batch, sub.shape[0] // 128 * 128), lr=mlp_lr,
                           seed=seed)
        t0 = mark("mlp_train", t0)
        init = net.predict(x)
        t0 = mark("mlp_predict", t0)
    finally:
        worker.join()
    if "error" in full:
        raise full["error"]
    t0 = mark("wait_full_graph", t0)
    fitted = Umap(cfg_full).fit_manifold(full.pop("manifold"), init)
    mark("fit", t0)
    t["full_graph_overlapped"] = full.get("ms", 0.0)
    t["total"] = (time.perf_counter() - t_start) * 1e3
    if info is not None:
        info["ms"] = t
        info["mlp_losses"] = losses.tolist()
        info["n_sub"] = int(n_sub)
    return fitted
