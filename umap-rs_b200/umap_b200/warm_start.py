"""Learned warm start (no counterpart in the reference, whose `Umap::fit` takes `init` from
the caller, embedding.rs:274).

A small MLP (in -> 256 -> 256 -> n_components, GELU; bf16 weights and activations, fp32
accumulation on the tensor cores) is trained with Adam on the plain-fit embedding of a
subsample, predicts an initial embedding for every point, and a shortened fit
(`n_epochs` = 100 by default) refines it.  The shortened fit keeps the reference's
semantics for that epoch count: `Optimizer::new` prunes at max_w / total_epochs
(optimizer.rs:96-102) and the learning rate decays from `learning_rate` over the shorter run.

Everything here runs through the library's C ABI: `umap_mlp_*` for the network (forward,
backward and Adam are the library's own kernels) and `umap_warm_start_fit_device` for the
whole pipeline.  The caller supplies the subsample's kNN, as it supplies the kNN of the full
data set.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from . import (ERR_INVALID_ARGUMENT, FittedUmap, UmapConfig, UmapError, _check, _Handle)

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


def warm_start_fit(config: UmapConfig, data, knn_indices, knn_dists, sub_index, sub_knn_indices, sub_knn_dists,
                   *, sub_init=None, sub_epochs: int = 500, epochs: int = 100, mlp_epochs: int = 20,
                   batch: int = 4096, mlp_lr: float = 1e-3, learning_rate: float | None = None, seed: int = 0,
                   info: dict | None = None) -> FittedUmap:
    """Fit with a learned initial embedding (umap_warm_start_fit_device: one call into the
    library, which builds the full graph on another stream while it fits the subsample and
    trains the network).

    data: CUDA f32 [n, d]; knn_*: the full data set's kNN (as for `Umap.fit`); sub_index:
    CUDA integer rows of the subsample; sub_knn_*: the subsample's own kNN (local ids).
    The subsample is fitted plainly for `sub_epochs` from `sub_init` (uniform [-10, 10]^2
    from `seed` when None); the network is trained on (data[sub_index], that embedding) for
    `mlp_epochs` epochs of Adam; its predictions initialise a fit of all points for `epochs`
    epochs.  `info`, when given, receives per-phase wall times (ms) and the loss curve.
    """
    import torch
    data = _cuda_f32(data, "data")
    n, d = data.shape
    dev = data.device
    ki, pki = _dev_u32(knn_indices, dev)
    kd = _dev_f32(knn_dists, dev)
    rows, prows = _dev_u32(sub_index, dev)
    si, psi = _dev_u32(sub_knn_indices, dev)
    sd = _dev_f32(sub_knn_dists, dev)
    n_sub = int(rows.shape[0])
    sinit = None
    if sub_init is not None:
        sinit = _dev_f32(sub_init, dev)
    wp = _lib.WarmStartParamsC()
    L = _lib.load()
    _check(L.umap_warm_start_params_default(C.byref(wp)))
    wp.sub_epochs, wp.epochs, wp.mlp_epochs, wp.batch = sub_epochs, epochs, mlp_epochs, batch
    wp.mlp_learning_rate = mlp_lr
    wp.has_learning_rate = int(learning_rate is not None)
    wp.learning_rate = 1.0 if learning_rate is None else learning_rate
    wp.seed = seed
    ph = np.zeros(len(_lib.WARM_START_PHASES), np.float32)
    losses = np.zeros(max(mlp_epochs, 1), np.float32)
    cfg = config.to_c()
    out = C.c_void_p()
    torch.cuda.synchronize(dev)
    _check(L.umap_warm_start_fit_device(
        C.byref(cfg), C.byref(wp), C.c_void_p(data.data_ptr()), n, d, pki, C.c_void_p(kd.data_ptr()),
        int(kd.shape[1]), prows, n_sub, psi, C.c_void_p(sd.data_ptr()),
        C.c_void_p(sinit.data_ptr()) if sinit is not None else None, C.byref(out),
        ph.ctypes.data_as(C.c_void_p), losses.ctypes.data_as(C.c_void_p)))
    fitted = FittedUmap(out.value)
    if info is not None:
        info["ms"] = {k: float(v) for k, v in zip(_lib.WARM_START_PHASES, ph)}
        info["mlp_losses"] = losses[:mlp_epochs].tolist()
        info["n_sub"] = n_sub
    return fitted


def _dev_f32(x, dev):
    """A contiguous CUDA f32 copy (or view) of a CUDA tensor or a host array."""
    import torch
    t = x if hasattr(x, "is_cuda") else torch.from_numpy(np.ascontiguousarray(np.asarray(x, np.float32)))
    return t.to(dev).float().contiguous()


def _dev_u32(x, dev):
    """A CUDA int32 view of integer ids (u32 values; int64 input narrowed) and its pointer."""
    import torch
    t = x if hasattr(x, "is_cuda") else torch.from_numpy(np.ascontiguousarray(np.asarray(x).astype(np.int64)))
    t = t.to(dev)
    if t.dtype != torch.int32:
        t = t.to(torch.int64).to(torch.int32)
    t = t.contiguous()
    return t, C.c_void_p(t.data_ptr())
