"""umap_b200: the B200 UMAP fit path behind the API of wilsonzlin/umap-rs.

Python mirror of the reference's Rust API (umap-rs/src/lib.rs:53-82) over the C ABI of
libumap_b200.so (include/umap_b200.h).  Names, argument meanings and error behaviour follow
the reference: every condition where the reference panics raises ``UmapError`` carrying the
reference's panic text.

    config = UmapConfig()
    umap = Umap(config)
    manifold = umap.learn_manifold(data, knn_indices, knn_dists)      # embedding.rs:149
    opt = Optimizer(manifold, init, 500, config, MetricType.Euclidean) # optimizer.rs:74
    while opt.remaining_epochs() > 0:
        opt.step_epochs(min(10, opt.remaining_epochs()), EuclideanMetric())
    fitted = opt.into_fitted(config)                                   # optimizer.rs:397
    fitted.embedding()

Inputs may be numpy arrays (host; copied to the GPU by the library) or CUDA torch tensors
(device-resident; the *_device entry points are used).  All compute runs on the GPU.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field

import numpy as np

from . import _lib

__all__ = [
    "ManifoldParams", "GraphParams", "OptimizationParams", "UmapConfig", "MetricType",
    "EuclideanMetric", "GenericEuclideanMetric", "Metric", "OUTPUT_METRIC_EUCLIDEAN", "Umap", "LearnedManifold", "Optimizer", "FittedUmap",
    "SparseMat", "UmapError", "find_ab_params", "lib", "knn_bruteforce", "knn_last_profile", "KNN_MAX_K", "KNN_MAX_K_TENSOR",
]

lib = _lib.load


class UmapError(RuntimeError):
    """A call into the library failed.  ``code`` is the C status (UMAP_ERR_*); for the
    reference's panic sites the message is the reference's panic text."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


ERR_INVALID_ARGUMENT, ERR_OVERSTEP, ERR_CUDA, ERR_OOM, ERR_FORMAT = 1, 2, 3, 4, 5
ERR_IO, ERR_NULL, ERR_UNSUPPORTED = 6, 7, 8


def _check(rc: int):
    if rc != 0:
        raise UmapError(rc, _lib.load().umap_last_error().decode())


def _f32(v) -> float:
    """An f32 field as the shortest decimal that round-trips (0.1f32 -> 0.1)."""
    return float(str(np.float32(v)))


# ------------------------------------------------------------------ config (config.rs)
@dataclass
class ManifoldParams:
    min_dist: float = 0.1
    spread: float = 1.0
    a: float | None = None
    b: float | None = None


@dataclass
class GraphParams:
    n_neighbors: int = 15
    local_connectivity: float = 1.0
    set_op_mix_ratio: float = 1.0
    disconnection_distance: float | None = None
    symmetrize: bool = True


@dataclass
class OptimizationParams:
    n_epochs: int | None = None
    learning_rate: float = 1.0
    negative_sample_rate: int = 5
    repulsion_strength: float = 1.0


@dataclass
class UmapConfig:
    n_components: int = 2
    manifold: ManifoldParams = field(default_factory=ManifoldParams)
    graph: GraphParams = field(default_factory=GraphParams)
    optimization: OptimizationParams = field(default_factory=OptimizationParams)

    def to_c(self) -> _lib.UmapConfigC:
        c = _lib.UmapConfigC()
        c.n_components = self.n_components
        c.min_dist = self.manifold.min_dist
        c.spread = self.manifold.spread
        c.has_a = int(self.manifold.a is not None)
        c.a = self.manifold.a or 0.0
        c.has_b = int(self.manifold.b is not None)
        c.b = self.manifold.b or 0.0
        c.n_neighbors = self.graph.n_neighbors
        c.local_connectivity = self.graph.local_connectivity
        c.set_op_mix_ratio = self.graph.set_op_mix_ratio
        c.has_disconnection_distance = int(self.graph.disconnection_distance is not None)
        c.disconnection_distance = self.graph.disconnection_distance or 0.0
        c.symmetrize = int(self.graph.symmetrize)
        c.has_n_epochs = int(self.optimization.n_epochs is not None)
        c.n_epochs = self.optimization.n_epochs or 0
        c.learning_rate = self.optimization.learning_rate
        c.negative_sample_rate = self.optimization.negative_sample_rate
        c.repulsion_strength = self.optimization.repulsion_strength
        return c

    @staticmethod
    def from_c(c: _lib.UmapConfigC) -> "UmapConfig":
        f = _f32
        return UmapConfig(
            n_components=int(c.n_components),
            manifold=ManifoldParams(f(c.min_dist), f(c.spread),
                                    f(c.a) if c.has_a else None, f(c.b) if c.has_b else None),
            graph=GraphParams(int(c.n_neighbors), f(c.local_connectivity), f(c.set_op_mix_ratio),
                              f(c.disconnection_distance) if c.has_disconnection_distance else None,
                              bool(c.symmetrize)),
            optimization=OptimizationParams(int(c.n_epochs) if c.has_n_epochs else None,
                                            f(c.learning_rate), int(c.negative_sample_rate),
                                            f(c.repulsion_strength)))


# ------------------------------------------------------------------ metrics (metric.rs)
class MetricType(enum.IntEnum):
    Euclidean = 0
    Generic = 1


OUTPUT_METRIC_EUCLIDEAN = 0   # umap_output_metric (include/umap_b200.h)


class Metric:
    """Output-space metric (metric.rs:19-62).  `metric_type()` picks the SGD rule: the
    Euclidean specialisation or the generic rule (layout/optimize_layout_generic.rs), which
    needs the metric's distance and gradient on the device.  `device_metric()` names that
    device implementation (an umap_output_metric id), or None for a metric that has none:
    a Generic optimizer stepped with such a metric raises UMAP_ERR_UNSUPPORTED."""

    def metric_type(self) -> MetricType:
        return MetricType.Generic

    def disconnection_threshold(self) -> float:
        return float("inf")

    def device_metric(self) -> int | None:
        return None


class EuclideanMetric(Metric):
    """distances.rs:10-50."""

    def metric_type(self) -> MetricType:
        return MetricType.Euclidean

    def device_metric(self) -> int | None:
        return OUTPUT_METRIC_EUCLIDEAN

    def distance(self, x, y):
        """(sqrt(sum (x - y)^2), (x - y) / (distance + 1e-6)) in f32 (distances.rs:22-37)."""
        x = np.asarray(x, np.float32)
        y = np.asarray(y, np.float32)
        s = np.float32(0)
        for v in x - y:
            s = np.float32(s + v * v)
        d = np.sqrt(s)
        return d, (x - y) / np.float32(d + np.float32(1e-6))


class GenericEuclideanMetric(EuclideanMetric):
    """EuclideanMetric's distance and gradient through the generic rule: what a Rust caller
    gets from a Metric impl that computes the Euclidean distance but keeps the trait's default
    `metric_type()` (Generic), so Optimizer::step_epochs takes optimize_layout_generic.rs."""

    def metric_type(self) -> MetricType:
        return MetricType.Generic


def kernel_launches() -> int:
    """Number of this library's kernel launches so far in this process."""
    v = C.c_uint64()
    _check(_lib.load().umap_kernel_launches(C.byref(v)))
    return v.value


def batch_fit(config: UmapConfig, offsets, knn_indices, knn_dists, init):
    """Umap::fit for many independent instances at once (no counterpart in the reference).
    Returns f32[total points, n_components] (host) or writes into a CUDA tensor when the
    inputs are CUDA tensors (returned)."""
    L = _lib.load()
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    n_inst = len(off) - 1
    cfg = config.to_c()
    k = int(knn_dists.shape[1])
    d = int(init.shape[1])
    if _is_cuda_tensor(knn_dists):
        import torch
        ti, pi = _device(knn_indices, torch.int32)
        td, pd = _device(knn_dists, torch.float32)
        tn, pn = _device(init, torch.float32)
        out = torch.empty((int(off[-1]), d), dtype=torch.float32, device=knn_dists.device)
        _check(L.umap_batch_fit_device(C.byref(cfg), n_inst, off.ctypes.data_as(C.c_void_p), pi, pd, k, pn, d,
                                       C.c_void_p(out.data_ptr())))
        return out
    ai, pi = _host(knn_indices, np.uint32)
    ad, pd = _host(knn_dists, np.float32)
    an, pn = _host(init, np.float32)
    out = np.empty((int(off[-1]), d), np.float32)
    _check(L.umap_batch_fit(C.byref(cfg), n_inst, off.ctypes.data_as(C.c_void_p), pi, pd, k, pn, d,
                            out.ctypes.data_as(C.c_void_p)))
    return out


KNN_MAX_K = 128       # largest k; above 32 every row takes the exact CUDA-core path
KNN_MAX_K_TENSOR = 32  # largest k through the tensor-core candidate pass


def knn_bruteforce(data, k: int, return_stats: bool = False):
    """Exact k nearest neighbours of every row of `data` [n, dim] (numpy f32 or a CUDA
    tensor), as the reference's example computes them (examples/src/bin/mnist_demo.rs:203-229):
    f32 Euclidean distance summed in coordinate order, self excluded, ordered by distance then
    index, missing slots 0 / 0.0 when n - 1 < k.  Returns (indices u32 [n, k], distances f32
    [n, k]) of the input's kind (numpy, or int32/float32 CUDA tensors), plus the number of rows
    recomputed exactly after a failed certificate when `return_stats`."""
    L = _lib.load()
    n, dim = int(data.shape[0]), int(data.shape[1])
    rec = C.c_uint64()
    if _is_cuda_tensor(data):
        import torch
        t, p = _device(data, torch.float32)
        idx = torch.empty((n, k), dtype=torch.int32, device=t.device)
        dist = torch.empty((n, k), dtype=torch.float32, device=t.device)
        _check(L.umap_knn_bruteforce_device(p, n, dim, k, C.c_void_p(idx.data_ptr() if n else 1),
                                            C.c_void_p(dist.data_ptr() if n else 1), C.byref(rec)))
    else:
        a, p = _host(data, np.float32)
        idx = np.zeros((n, k), np.uint32)
        dist = np.zeros((n, k), np.float32)
        _check(L.umap_knn_bruteforce(p, n, dim, k, idx.ctypes.data_as(C.c_void_p) if n else C.c_void_p(1),
                                     dist.ctypes.data_as(C.c_void_p) if n else C.c_void_p(1), C.byref(rec)))
    return (idx, dist, rec.value) if return_stats else (idx, dist)


def knn_last_profile():
    """(candidate-pass ms, rows recomputed, scanned in locality order) of this thread's last
    knn_bruteforce call."""
    ms, rec, ro = C.c_float(), C.c_uint64(), C.c_uint32()
    _check(_lib.load().umap_knn_last_profile(C.byref(ms), C.byref(rec), C.byref(ro)))
    return ms.value, rec.value, bool(ro.value)


def release_cached_memory() -> int:
    """Return the library's cached device blocks to the CUDA pool; returns their bytes."""
    v = C.c_uint64()
    _check(_lib.load().umap_release_cached_memory(C.byref(v)))
    return v.value


def find_ab_params(spread: float, min_dist: float):
    """umap/find_ab_params.rs:9-82 (host code inside the library)."""
    a, b = C.c_float(), C.c_float()
    _check(_lib.load().umap_find_ab_params(spread, min_dist, C.byref(a), C.byref(b)))
    return a.value, b.value


# ------------------------------------------------------------------ array helpers
def _is_cuda_tensor(x) -> bool:
    return hasattr(x, "is_cuda") and bool(x.is_cuda)


def _n_samples(data) -> int:
    if isinstance(data, (int, np.integer)):
        return int(data)
    return int(data.shape[0])


def _host(x, dtype):
    a = np.ascontiguousarray(x, dtype=dtype)
    return a, a.ctypes.data_as(C.c_void_p)


def _device(x, torch_dtype):
    t = x.contiguous()
    if t.dtype != torch_dtype:
        t = t.to(torch_dtype)
    return t, C.c_void_p(t.data_ptr())


class SparseMat:
    """CSR graph (sprs CsMatI<f32, u32, usize>): indptr u64[n+1], indices u32[nnz], data f32[nnz]."""

    def __init__(self, n: int, indptr, indices, data):
        self.shape = (n, n)
        self.indptr, self.indices, self.data = indptr, indices, data

    def nnz(self) -> int:
        return int(self.indices.shape[0])

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.data, self.indices.astype(np.int64), self.indptr.astype(np.int64)),
                             shape=self.shape)


class _Handle:
    _free = None

    def __init__(self, h):
        self._h = h

    def _get(self):
        if not self._h:
            raise UmapError(ERR_NULL, f"{type(self).__name__} has been moved or freed")
        return self._h

    def _take(self):
        h = self._get()
        self._h = None
        return h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and self._free:
            try:
                getattr(_lib.load(), self._free)(h)
            except Exception:
                pass
            self._h = None


# ------------------------------------------------------------------ LearnedManifold
class LearnedManifold(_Handle):
    """manifold.rs:14-55."""
    _free = "umap_manifold_free"

    def __init__(self, h, owner=None):
        super().__init__(h)
        self._owner = owner  # borrowed views keep their owner alive and are not freed
        if owner is not None:
            self._free = None

    def n_vertices(self) -> int:
        v = C.c_uint64()
        _check(_lib.load().umap_manifold_n_vertices(self._get(), C.byref(v)))
        return v.value

    def curve_params(self):
        a, b = C.c_float(), C.c_float()
        _check(_lib.load().umap_manifold_curve_params(self._get(), C.byref(a), C.byref(b)))
        return a.value, b.value

    def graph(self) -> SparseMat:
        L = _lib.load()
        n = self.n_vertices()
        nnz = C.c_uint64()
        _check(L.umap_manifold_graph_nnz(self._get(), C.byref(nnz)))
        ip = np.empty(n + 1, np.uint64)
        ix = np.empty(nnz.value, np.uint32)
        dt = np.empty(nnz.value, np.float32)
        _check(L.umap_manifold_graph_copy(self._get(), ip.ctypes.data_as(C.c_void_p),
                                          ix.ctypes.data_as(C.c_void_p), dt.ctypes.data_as(C.c_void_p)))
        return SparseMat(n, ip, ix, dt)

    def sigmas_rhos(self):
        n = self.n_vertices()
        s = np.empty(n, np.float32)
        r = np.empty(n, np.float32)
        _check(_lib.load().umap_manifold_sigmas_rhos(self._get(), s.ctypes.data_as(C.c_void_p),
                                                     r.ctypes.data_as(C.c_void_p)))
        return s, r

    def disconnection_counts(self):
        e, v = C.c_uint64(), C.c_uint64()
        _check(_lib.load().umap_manifold_disconnection_counts(self._get(), C.byref(e), C.byref(v)))
        return e.value, v.value

    def clone(self) -> "LearnedManifold":
        out = C.c_void_p()
        _check(_lib.load().umap_manifold_clone(self._get(), C.byref(out)))
        return LearnedManifold(out.value)

    def to_bytes(self) -> bytes:
        return _serialize("umap_manifold_serialize", self._get())

    @staticmethod
    def from_bytes(b: bytes) -> "LearnedManifold":
        return LearnedManifold(_deserialize("umap_manifold_deserialize", b))

    def to_bincode(self) -> bytes:
        """The reference's own bytes: bincode::serialize(&manifold)."""
        return _serialize("umap_manifold_serialize_bincode", self._get())

    @staticmethod
    def from_bincode(b: bytes) -> "LearnedManifold":
        return LearnedManifold(_deserialize("umap_manifold_deserialize_bincode", b))


def _serialize(fn, h) -> bytes:
    L = _lib.load()
    need = C.c_uint64()
    _check(getattr(L, fn)(h, None, 0, C.byref(need)))
    buf = (C.c_uint8 * need.value)()
    _check(getattr(L, fn)(h, C.cast(buf, C.c_void_p), need.value, C.byref(need)))
    return bytes(buf)


def _deserialize(fn, b: bytes):
    L = _lib.load()
    arr = (C.c_uint8 * len(b)).from_buffer_copy(b) if len(b) else (C.c_uint8 * 1)()
    out = C.c_void_p()
    _check(getattr(L, fn)(C.cast(arr, C.c_void_p), len(b), C.byref(out)))
    return out.value


# ------------------------------------------------------------------ Umap (embedding.rs)
class Umap:
    def __init__(self, config: UmapConfig | None = None):
        self.config = config or UmapConfig()
        self.metric = EuclideanMetric()
        self.output_metric = EuclideanMetric()

    @staticmethod
    def with_metrics(config: UmapConfig, metric: Metric, output_metric: Metric) -> "Umap":
        u = Umap(config)
        u.metric, u.output_metric = metric, output_metric
        return u

    def _cfg(self):
        c = self.config.to_c()
        if self.config.graph.disconnection_distance is None:
            thr = self.metric.disconnection_threshold()
            if thr != float("inf"):
                c.has_disconnection_distance = 1
                c.disconnection_distance = thr
        return c

    def learn_manifold(self, data, knn_indices, knn_dists) -> LearnedManifold:
        """embedding.rs:149-240."""
        L = _lib.load()
        n = _n_samples(data)
        rows, cols = int(knn_dists.shape[0]), int(knn_dists.shape[1])
        if tuple(knn_indices.shape) != tuple(knn_dists.shape):
            raise UmapError(ERR_INVALID_ARGUMENT,
                            f"knn_dists and knn_indices must have the same shape, got "
                            f"{list(knn_dists.shape)} vs {list(knn_indices.shape)}")
        cfg = self._cfg()
        out = C.c_void_p()
        if _is_cuda_tensor(knn_dists):
            import torch
            ti, pi = _device(knn_indices, torch.int32)
            td, pd = _device(knn_dists, torch.float32)
            _check(L.umap_learn_manifold_device(C.byref(cfg), n, pi, pd, rows, cols, C.byref(out)))
        else:
            ai, pi = _host(knn_indices, np.uint32)
            ad, pd = _host(knn_dists, np.float32)
            _check(L.umap_learn_manifold(C.byref(cfg), n, pi, pd, rows, cols, C.byref(out)))
        return LearnedManifold(out.value)

    def _output_metric_ids(self):
        mt = self.output_metric.metric_type()
        dm = self.output_metric.device_metric()
        if mt == MetricType.Generic and dm is None:
            raise UmapError(ERR_UNSUPPORTED, f"output metric {type(self.output_metric).__name__} has no "
                                             "device implementation")
        return int(mt), OUTPUT_METRIC_EUCLIDEAN if dm is None else int(dm)

    def fit(self, data, knn_indices, knn_dists, init) -> "FittedUmap":
        """embedding.rs:274-337."""
        L = _lib.load()
        if self._output_metric_ids()[0] != MetricType.Euclidean:
            # generic rule: learn_manifold, then the rest of fit with the metric's device id
            irows, icols = int(init.shape[0]), int(init.shape[1])
            n = _n_samples(data)
            if icols != self.config.n_components:
                raise UmapError(ERR_INVALID_ARGUMENT, f"init has {icols} components but n_components is "
                                                      f"{self.config.n_components}")
            if irows != n:
                raise UmapError(ERR_INVALID_ARGUMENT, f"init has {irows} samples but data has {n} samples")
            return self.fit_manifold(self.learn_manifold(data, knn_indices, knn_dists), init)
        n = _n_samples(data)
        rows, cols = int(knn_dists.shape[0]), int(knn_dists.shape[1])
        if tuple(knn_indices.shape) != tuple(knn_dists.shape):
            raise UmapError(ERR_INVALID_ARGUMENT,
                            f"knn_dists and knn_indices must have the same shape, got "
                            f"{list(knn_dists.shape)} vs {list(knn_indices.shape)}")
        irows, icols = int(init.shape[0]), int(init.shape[1])
        cfg = self._cfg()
        out = C.c_void_p()
        if _is_cuda_tensor(knn_dists):
            import torch
            ti, pi = _device(knn_indices, torch.int32)
            td, pd = _device(knn_dists, torch.float32)
            tn, pn = _device(init, torch.float32)
            _check(L.umap_fit_device(C.byref(cfg), n, pi, pd, rows, cols, pn, irows, icols, C.byref(out)))
        else:
            ai, pi = _host(knn_indices, np.uint32)
            ad, pd = _host(knn_dists, np.float32)
            an, pn = _host(init, np.float32)
            _check(L.umap_fit(C.byref(cfg), n, pi, pd, rows, cols, pn, irows, icols, C.byref(out)))
        return FittedUmap(out.value)


    def fit_manifold(self, manifold: "LearnedManifold", init) -> "FittedUmap":
        """embedding.rs:299-337: `fit` after its learn_manifold step.  Consumes `manifold`."""
        L = _lib.load()
        mt, dm = self._output_metric_ids()
        cfg = self._cfg()
        irows, icols = int(init.shape[0]), int(init.shape[1])
        mh = manifold._take()
        out = C.c_void_p()
        if _is_cuda_tensor(init):
            import torch
            tn, pn = _device(init, torch.float32)
            _check(L.umap_fit_manifold_metric_device(mh, C.byref(cfg), pn, irows, icols, mt, dm, C.byref(out)))
        else:
            an, pn = _host(init, np.float32)
            _check(L.umap_fit_manifold_metric(mh, C.byref(cfg), pn, irows, icols, mt, dm, C.byref(out)))
        return FittedUmap(out.value)


# ------------------------------------------------------------------ Optimizer (optimizer.rs)
class Optimizer(_Handle):
    _free = "umap_optimizer_free"

    def __init__(self, manifold: LearnedManifold | None, init=None, total_epochs: int = 0,
                 config: UmapConfig | None = None, metric_type: MetricType = MetricType.Euclidean,
                 _handle=None):
        """optimizer.rs:74-290.  Consumes `manifold` (the reference moves it in)."""
        if _handle is not None:
            super().__init__(_handle)
            return
        L = _lib.load()
        config = config or UmapConfig()
        cfg = config.to_c()
        mh = manifold._take()
        rows, dims = int(init.shape[0]), int(init.shape[1])
        out = C.c_void_p()
        if _is_cuda_tensor(init):
            import torch
            t, p = _device(init, torch.float32)
            rc = L.umap_optimizer_new_device(mh, p, rows, dims, total_epochs, C.byref(cfg), int(metric_type),
                                             C.byref(out))
        else:
            a, p = _host(init, np.float32)
            rc = L.umap_optimizer_new(mh, p, rows, dims, total_epochs, C.byref(cfg), int(metric_type),
                                      C.byref(out))
        super().__init__(out.value)
        _check(rc)

    def step_epochs(self, n: int, output_metric: Metric | None = None):
        """optimizer.rs:297-366.  A Generic optimizer uses `output_metric` (Euclidean when
        omitted); one without a device implementation raises UMAP_ERR_UNSUPPORTED."""
        dm = OUTPUT_METRIC_EUCLIDEAN if output_metric is None else output_metric.device_metric()
        _check(_lib.load().umap_optimizer_step_epochs_metric(self._get(), n, -1 if dm is None else int(dm)))

    def _u64(self, fn):
        v = C.c_uint64()
        _check(getattr(_lib.load(), fn)(self._get(), C.byref(v)))
        return v.value

    def current_epoch(self) -> int:
        return self._u64("umap_optimizer_current_epoch")

    def total_epochs(self) -> int:
        return self._u64("umap_optimizer_total_epochs")

    def remaining_epochs(self) -> int:
        return self._u64("umap_optimizer_remaining_epochs")

    def n_edges(self) -> int:
        return self._u64("umap_optimizer_n_edges")

    def dims(self):
        n, d = C.c_uint64(), C.c_uint64()
        _check(_lib.load().umap_optimizer_dims(self._get(), C.byref(n), C.byref(d)))
        return n.value, d.value

    def embedding(self) -> np.ndarray:
        n, d = self.dims()
        out = np.empty((n, d), np.float32)
        _check(_lib.load().umap_optimizer_embedding(self._get(), out.ctypes.data_as(C.c_void_p)))
        return out

    def embedding_device_ptr(self) -> int:
        p = C.c_void_p()
        _check(_lib.load().umap_optimizer_embedding_device(self._get(), C.byref(p)))
        return p.value

    def manifold(self) -> LearnedManifold:
        p = C.c_void_p()
        _check(_lib.load().umap_optimizer_manifold(self._get(), C.byref(p)))
        return LearnedManifold(p.value, owner=self)

    def last_step_ms(self) -> float:
        """CUDA-event time of the last step_epochs epoch loop (library stream)."""
        v = C.c_float()
        _check(_lib.load().umap_optimizer_last_step_ms(self._get(), C.byref(v)))
        return v.value

    def set_seed(self, seed: int):
        _check(_lib.load().umap_optimizer_set_seed(self._get(), seed))

    def export_edges(self):
        """The reference's per-edge arrays: head, tail, epochs_per_sample and the schedule
        state (epoch_of_next_sample, epoch_of_next_negative_sample, epochs_per_negative_sample)."""
        E = self.n_edges()
        head = np.empty(E, np.uint32)
        tail = np.empty(E, np.uint32)
        arrs = [np.empty(E, np.float64) for _ in range(4)]
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        _check(_lib.load().umap_optimizer_export_edges(self._get(), ptr(head), ptr(tail), *[ptr(a) for a in arrs]))
        return head, tail, arrs[0], arrs[1], arrs[2], arrs[3]

    def schedule_totals(self, start: int, end: int):
        f, g = C.c_uint64(), C.c_uint64()
        _check(_lib.load().umap_optimizer_schedule_totals(self._get(), start, end, C.byref(f), C.byref(g)))
        return f.value, g.value

    @staticmethod
    def batch(config: UmapConfig, offsets, knn_indices, knn_dists, init, total_epochs: int) -> "Optimizer":
        """Batched instances (no counterpart in the reference): instance s owns points
        [offsets[s], offsets[s+1]) of the concatenated arrays; kNN ids are local to each
        instance.  Returns one optimizer over all instances (one kernel launch per epoch)."""
        L = _lib.load()
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        n_inst = len(off) - 1
        cfg = config.to_c()
        out = C.c_void_p()
        k = int(knn_dists.shape[1])
        d = int(init.shape[1])
        if _is_cuda_tensor(knn_dists):
            import torch
            ti, pi = _device(knn_indices, torch.int32)
            td, pd = _device(knn_dists, torch.float32)
            tn, pn = _device(init, torch.float32)
            _check(L.umap_batch_optimizer_new_device(C.byref(cfg), n_inst, off.ctypes.data_as(C.c_void_p),
                                                     pi, pd, k, pn, d, total_epochs, C.byref(out)))
        else:
            ai, pi = _host(knn_indices, np.uint32)
            ad, pd = _host(knn_dists, np.float32)
            an, pn = _host(init, np.float32)
            _check(L.umap_batch_optimizer_new(C.byref(cfg), n_inst, off.ctypes.data_as(C.c_void_p),
                                              pi, pd, k, pn, d, total_epochs, C.byref(out)))
        return Optimizer(None, _handle=out.value)

    def layout(self) -> dict:
        """How the SGD layout is laid out: lane-major entries, the 8-negatives register
        budget, vertices renamed into a locality order, the order tasks are dealt to warps
        ("length", "length+rate", "row blocks" or "rows"); and the epoch kernel it selects."""
        f = C.c_uint32()
        _check(_lib.load().umap_optimizer_layout_flags(self._get(), C.byref(f)))
        bit = _lib.LAYOUT_FLAGS
        lm, eight, renamed, generic, twelve = (bool(f.value & bit[k]) for k in
                                               ("LANE_MAJOR", "EIGHT_NEGATIVES", "RENAMED", "GENERIC_RULE",
                                                "TWELVE_NEGATIVES"))
        _, dim = self.dims()
        eight = eight and dim <= 2 and not generic  # the generic rule keeps the 4-negatives budget
        twelve = twelve and dim <= 2 and not generic
        nb, minb = (12, 3) if twelve else (8, 4) if eight else (4, 5)
        gen = "true" if generic else "false"
        kernel = (f"sgd_epoch_kernel2<{dim}, {gen}, {nb}, {minb}, {'true' if lm else 'false'}>" if dim <= 4
                  else f"sgd_epoch_anydim<{gen}>")
        order = ("length+rate" if f.value & bit["RATE_ORDER"] else "row blocks" if f.value & bit["BLOCK_ORDER"]
                 else "rows" if f.value & bit["ROW_ORDER"] else "length")
        return {"lane_major": lm, "eight_negatives": eight, "twelve_negatives": twelve, "renamed": renamed,
                "generic_rule": generic, "task_order": order, "kernel": kernel}

    def tuning(self):
        """(task length, threads per block) of the SGD kernel in use."""
        c, b = C.c_uint32(), C.c_uint32()
        _check(_lib.load().umap_optimizer_tuning(self._get(), C.byref(c), C.byref(b)))
        return c.value, b.value

    def into_fitted(self, config: UmapConfig | None = None) -> "FittedUmap":
        """optimizer.rs:397-403.  Consumes the optimizer."""
        cfg = (config or UmapConfig()).to_c()
        out = C.c_void_p()
        _check(_lib.load().umap_optimizer_into_fitted(self._take(), C.byref(cfg), C.byref(out)))
        return FittedUmap(out.value)

    def to_bytes(self) -> bytes:
        return _serialize("umap_optimizer_serialize", self._get())

    @staticmethod
    def from_bytes(b: bytes) -> "Optimizer":
        return Optimizer(None, _handle=_deserialize("umap_optimizer_deserialize", b))

    def to_bincode(self) -> bytes:
        """The reference's own bytes: bincode::serialize(&optimizer)."""
        return _serialize("umap_optimizer_serialize_bincode", self._get())

    @staticmethod
    def from_bincode(b: bytes) -> "Optimizer":
        return Optimizer(None, _handle=_deserialize("umap_optimizer_deserialize_bincode", b))


# ------------------------------------------------------------------ FittedUmap
class FittedUmap(_Handle):
    """embedding.rs:438-524."""
    _free = "umap_fitted_free"

    def dims(self):
        n, d = C.c_uint64(), C.c_uint64()
        _check(_lib.load().umap_fitted_dims(self._get(), C.byref(n), C.byref(d)))
        return n.value, d.value

    def embedding(self) -> np.ndarray:
        n, d = self.dims()
        out = np.empty((n, d), np.float32)
        _check(_lib.load().umap_fitted_embedding(self._get(), out.ctypes.data_as(C.c_void_p)))
        return out

    def into_embedding(self) -> np.ndarray:
        e = self.embedding()
        h = self._take()
        _lib.load().umap_fitted_free(h)
        return e

    def manifold(self) -> LearnedManifold:
        p = C.c_void_p()
        _check(_lib.load().umap_fitted_manifold(self._get(), C.byref(p)))
        return LearnedManifold(p.value, owner=self)

    def config(self) -> UmapConfig:
        c = _lib.UmapConfigC()
        _check(_lib.load().umap_fitted_config(self._get(), C.byref(c)))
        return UmapConfig.from_c(c)

    def transform(self, new_data, new_knn_indices, new_knn_dists):
        """embedding.rs:516-523: `todo!()` in the reference."""
        raise NotImplementedError("Transform not yet implemented - contributions welcome!")

    def to_bytes(self) -> bytes:
        return _serialize("umap_fitted_serialize", self._get())

    @staticmethod
    def from_bytes(b: bytes) -> "FittedUmap":
        return FittedUmap(_deserialize("umap_fitted_deserialize", b))

    def to_bincode(self) -> bytes:
        """The reference's own bytes: bincode::serialize(&fitted)."""
        return _serialize("umap_fitted_serialize_bincode", self._get())

    @staticmethod
    def from_bincode(b: bytes) -> "FittedUmap":
        return FittedUmap(_deserialize("umap_fitted_deserialize_bincode", b))


# ------------------------------------------------------------------ learned warm start
from .warm_start import Mlp, gemm_bf16, init_params as mlp_init_params, warm_start_fit  # noqa: E402
