"""ctypes binding of the CPU oracle (liborc_umap.so) -- TEST INFRASTRUCTURE ONLY.

The oracle restates the reference UMAP fit path (wilsonzlin/umap-rs, Rust) in C++; see the
header of umap_oracle.cpp for what each function follows and for its parity status
("parity unpinned": the Rust reference cannot be built here and its own tests pin no
numeric value).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs
import this module; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liborc_umap.so")
_lib = None

u64, u32, f32, i32 = C.c_uint64, C.c_uint32, C.c_float, C.c_int
P = C.c_void_p


def build(force: bool = False) -> str:
    """Compile liborc_umap.so with the committed Makefile (g++, no GPU needed)."""
    src = os.path.join(_HERE, "umap_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liborc_umap.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_last_error.restype = C.c_char_p
        L.orc_set_threads.argtypes = [i32]
        L.orc_get_threads.restype = i32
        L.orc_find_ab_params.argtypes = [f32, f32, P, P]
        L.orc_ndarray_mean.argtypes = [P, u64]
        L.orc_ndarray_mean.restype = f32
        L.orc_smooth_knn_dist.argtypes = [P, u64, u64, u64, f32, f32, P, P]
        L.orc_learn_manifold.argtypes = [u64, u64, u64, P, P, u64, f32, f32, i32, f32, i32, f32,
                                         f32, f32, i32, f32, i32, f32, f32, u64]
        L.orc_learn_manifold.restype = P
        L.orc_manifold_free.argtypes = [P]
        for fn in ("orc_manifold_nnz", "orc_manifold_directed_nnz"):
            getattr(L, fn).argtypes = [P]
            getattr(L, fn).restype = u64
        L.orc_manifold_graph.argtypes = [P, P, P, P]
        L.orc_manifold_directed.argtypes = [P, P, P, P]
        L.orc_manifold_sigmas_rhos.argtypes = [P, P, P]
        L.orc_manifold_info.argtypes = [P, P, P, P, P, P]
        L.orc_optimizer_new.argtypes = [P, P, u64, u64, u64, f32, f32, u64, u64]
        L.orc_optimizer_new.restype = P
        L.orc_optimizer_free.argtypes = [P]
        for fn in ("orc_optimizer_n_edges", "orc_optimizer_current_epoch", "orc_optimizer_total_epochs"):
            getattr(L, fn).argtypes = [P]
            getattr(L, fn).restype = u64
        L.orc_optimizer_threshold.argtypes = [P, P, P]
        L.orc_optimizer_edges.argtypes = [P, P, P, P]
        L.orc_optimizer_state.argtypes = [P, P, P, P]
        L.orc_optimizer_embedding.argtypes = [P, P]
        L.orc_optimizer_set_embedding.argtypes = [P, P]
        L.orc_optimizer_set_metric_type.argtypes = [P, i32]
        L.orc_knn_bruteforce.argtypes = [P, u64, u64, u64, P, P]
        L.orc_knn_bruteforce.restype = None
        L.orc_knn_bruteforce_rows.argtypes = [P, u64, u64, u64, u64, u64, P, P]
        L.orc_knn_bruteforce_rows.restype = None
        L.orc_optimizer_step_epochs.argtypes = [P, u64, P, P]
        L.orc_optimizer_step_epochs.restype = i32
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class OracleError(RuntimeError):
    pass


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


def find_ab_params(spread: float, min_dist: float):
    a, b = C.c_float(), C.c_float()
    lib().orc_find_ab_params(spread, min_dist, C.byref(a), C.byref(b))
    return a.value, b.value


def ndarray_mean(x: np.ndarray) -> np.float32:
    x = np.ascontiguousarray(x, dtype=np.float32)
    return np.float32(lib().orc_ndarray_mean(_ptr(x), x.size))


def smooth_knn_dist(dists: np.ndarray, k: int | None = None, n_iter: int = 64,
                    local_connectivity: float = 1.0, bandwidth: float = 1.0):
    d = np.ascontiguousarray(dists, dtype=np.float32)
    n, kk = d.shape
    sig = np.empty(n, np.float32)
    rho = np.empty(n, np.float32)
    lib().orc_smooth_knn_dist(_ptr(d), n, kk if k is None else k, n_iter, local_connectivity,
                              bandwidth, _ptr(sig), _ptr(rho))
    return sig, rho


@dataclass
class OracleConfig:
    n_neighbors: int = 15
    min_dist: float = 0.1
    spread: float = 1.0
    a: float | None = None
    b: float | None = None
    local_connectivity: float = 1.0
    set_op_mix_ratio: float = 1.0
    disconnection_distance: float | None = None
    symmetrize: bool = True
    repulsion_strength: float = 1.0
    learning_rate: float = 1.0
    negative_sample_rate: int = 5
    n_components: int = 2
    n_epochs: int | None = None


class Manifold:
    def __init__(self, handle):
        self.h = handle

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_manifold_free(self.h)
            self.h = None

    def info(self):
        n, ed, vd = C.c_uint64(), C.c_uint64(), C.c_uint64()
        a, b = C.c_float(), C.c_float()
        lib().orc_manifold_info(self.h, C.byref(n), C.byref(a), C.byref(b), C.byref(ed), C.byref(vd))
        return dict(n_vertices=n.value, a=a.value, b=b.value, edges_removed=ed.value,
                    vertices_disconnected=vd.value)

    @property
    def n_vertices(self):
        return self.info()["n_vertices"]

    def graph(self):
        n = self.n_vertices
        nnz = lib().orc_manifold_nnz(self.h)
        ip = np.empty(n + 1, np.uint64)
        ix = np.empty(nnz, np.uint32)
        dt = np.empty(nnz, np.float32)
        lib().orc_manifold_graph(self.h, _ptr(ip), _ptr(ix), _ptr(dt))
        return ip, ix, dt

    def directed(self):
        n = self.n_vertices
        nnz = lib().orc_manifold_directed_nnz(self.h)
        ip = np.empty(n + 1, np.uint64)
        ix = np.empty(nnz, np.uint32)
        dt = np.empty(nnz, np.float32)
        lib().orc_manifold_directed(self.h, _ptr(ip), _ptr(ix), _ptr(dt))
        return ip, ix, dt

    def sigmas_rhos(self):
        n = self.n_vertices
        s = np.empty(n, np.float32)
        r = np.empty(n, np.float32)
        lib().orc_manifold_sigmas_rhos(self.h, _ptr(s), _ptr(r))
        return s, r


def learn_manifold(knn_idx: np.ndarray, knn_dist: np.ndarray, cfg: OracleConfig | None = None,
                   n_samples: int | None = None) -> Manifold:
    cfg = cfg or OracleConfig()
    idx = np.ascontiguousarray(knn_idx, dtype=np.uint32)
    dst = np.ascontiguousarray(knn_dist, dtype=np.float32)
    rows, cols = dst.shape
    n = rows if n_samples is None else n_samples
    h = lib().orc_learn_manifold(
        n, rows, cols, _ptr(idx), _ptr(dst), cfg.n_neighbors, cfg.min_dist, cfg.spread,
        int(cfg.a is not None), 0.0 if cfg.a is None else cfg.a,
        int(cfg.b is not None), 0.0 if cfg.b is None else cfg.b,
        cfg.local_connectivity, cfg.set_op_mix_ratio,
        int(cfg.disconnection_distance is not None),
        0.0 if cfg.disconnection_distance is None else cfg.disconnection_distance,
        int(cfg.symmetrize), cfg.repulsion_strength, cfg.learning_rate, cfg.n_components)
    if not h:
        raise OracleError(lib().orc_last_error().decode())
    return Manifold(h)


class Optimizer:
    def __init__(self, manifold: Manifold, init: np.ndarray, total_epochs: int,
                 cfg: OracleConfig | None = None, seed: int = 0, metric_type: int = 0):
        """metric_type 0 = Euclidean specialisation (optimize_layout_euclidean.rs), 1 = the
        generic-metric rule with the built-in Euclidean output metric
        (optimize_layout_generic.rs + distances.rs)."""
        cfg = cfg or OracleConfig()
        x = np.ascontiguousarray(init, dtype=np.float32)
        self.n, self.dim = x.shape
        self.h = lib().orc_optimizer_new(manifold.h, _ptr(x), self.n, self.dim, total_epochs,
                                         cfg.repulsion_strength, cfg.learning_rate,
                                         cfg.negative_sample_rate, seed)
        if not self.h:
            raise OracleError(lib().orc_last_error().decode())
        lib().orc_optimizer_set_metric_type(self.h, int(metric_type))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_optimizer_free(self.h)
            self.h = None

    def n_edges(self):
        return int(lib().orc_optimizer_n_edges(self.h))

    def current_epoch(self):
        return int(lib().orc_optimizer_current_epoch(self.h))

    def total_epochs(self):
        return int(lib().orc_optimizer_total_epochs(self.h))

    def remaining_epochs(self):
        return self.total_epochs() - self.current_epoch()

    def threshold(self):
        mv, th = C.c_float(), C.c_float()
        lib().orc_optimizer_threshold(self.h, C.byref(mv), C.byref(th))
        return mv.value, th.value

    def edges(self):
        e = self.n_edges()
        head = np.empty(e, np.uint32)
        tail = np.empty(e, np.uint32)
        eps = np.empty(e, np.float64)
        lib().orc_optimizer_edges(self.h, _ptr(head), _ptr(tail), _ptr(eps))
        return head, tail, eps

    def state(self):
        e = self.n_edges()
        a, b, c = (np.empty(e, np.float64) for _ in range(3))
        lib().orc_optimizer_state(self.h, _ptr(a), _ptr(b), _ptr(c))
        return a, b, c

    def embedding(self):
        out = np.empty((self.n, self.dim), np.float32)
        lib().orc_optimizer_embedding(self.h, _ptr(out))
        return out

    def set_embedding(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        lib().orc_optimizer_set_embedding(self.h, _ptr(x))

    def step_epochs(self, n: int, counts: bool = False):
        fires = np.zeros(max(n, 1), np.uint64)
        negs = np.zeros(max(n, 1), np.uint64)
        rc = lib().orc_optimizer_step_epochs(self.h, n, _ptr(fires), _ptr(negs))
        if rc != 0:
            raise OracleError(lib().orc_last_error().decode())
        if counts:
            return fires[:n], negs[:n]


def fit(knn_idx, knn_dist, init, cfg: OracleConfig | None = None, seed: int = 0, metric_type: int = 0):
    """embedding.rs:274-337: learn_manifold -> Optimizer::new -> one step_epochs call ->
    rows whose graph row sums to zero become NaN."""
    cfg = cfg or OracleConfig()
    n = knn_idx.shape[0]
    m = learn_manifold(knn_idx, knn_dist, cfg)
    total = cfg.n_epochs if cfg.n_epochs is not None else (500 if n <= 10000 else 200)
    opt = Optimizer(m, init, total, cfg, seed=seed, metric_type=metric_type)
    opt.step_epochs(total)
    emb = opt.embedding()
    ip, _, _ = m.graph()
    empty = (ip[1:] - ip[:-1]) == 0
    emb[empty] = np.nan
    return emb, m, opt


def knn_bruteforce(X, k: int, rows=None):
    """examples/src/bin/mnist_demo.rs:203-229 (brute force, self excluded, stable by distance).
    `rows` = (r0, r1) computes only those query rows (against all points)."""
    x = np.ascontiguousarray(X, dtype=np.float32)
    n, d = x.shape
    r0, r1 = (0, n) if rows is None else rows
    idx = np.zeros((r1 - r0, k), np.uint32)
    dist = np.zeros((r1 - r0, k), np.float32)
    if r1 > r0:
        lib().orc_knn_bruteforce_rows(_ptr(x), n, d, k, r0, r1, _ptr(idx), _ptr(dist))
    return idx, dist
