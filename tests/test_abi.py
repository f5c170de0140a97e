"""CPU tests of the C ABI boundary: the library loads without a GPU, exports every symbol
include/umap_b200.h declares, and its host-only logic (defaults, curve fit, validation with
the reference's panic texts) behaves like the reference.  No compute call is made here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "umap_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(umap_\w+)\s*\(", txt, re.M)))


def test_every_declared_symbol_is_exported(ub):
    L = ub.lib()
    names = declared_functions()
    assert len(names) >= 40
    for n in names:
        assert hasattr(L, n), n


def test_python_binding_covers_header(ub):
    from umap_b200 import _lib
    names = set(declared_functions()) - {"umap_last_error", "umap_abi_version"}
    assert names == set(_lib.SIGNATURES)


def test_layout_flag_bits_match_header(ub):
    """The layout flags the Python binding decodes are the header's UMAP_LAYOUT_* values."""
    from umap_b200 import _lib
    txt = open(HEADER).read()
    defs = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define UMAP_LAYOUT_(\w+) (\d+)u", txt)}
    assert defs == _lib.LAYOUT_FLAGS


@pytest.mark.parametrize("flags,dims,expect", [
    (1 | 2 | 32, 2, {"lane_major": True, "eight_negatives": True, "task_order": "length+rate",
                     "kernel": "sgd_epoch_kernel2<2, false, 8, 4, true>"}),
    (4 | 16 | 64, 2, {"renamed": True, "twelve_negatives": True, "task_order": "row blocks",
                      "kernel": "sgd_epoch_kernel2<2, false, 12, 3, false>"}),
    (1, 2, {"task_order": "length", "kernel": "sgd_epoch_kernel2<2, false, 4, 5, true>"}),
    (1 | 8 | 2, 2, {"generic_rule": True, "eight_negatives": False,
                    "kernel": "sgd_epoch_kernel2<2, true, 4, 5, true>"}),
    (128, 5, {"task_order": "rows", "kernel": "sgd_epoch_anydim<false>"}),
])
def test_layout_flags_decoded_without_gpu(ub, monkeypatch, flags, dims, expect):
    """Optimizer.layout() turns umap_optimizer_layout_flags into the kernel it selects."""
    from umap_b200 import _lib

    class StubLib:
        def umap_optimizer_layout_flags(self, h, out):
            out._obj.value = flags
            return 0

    opt = ub.Optimizer.__new__(ub.Optimizer)
    monkeypatch.setattr(_lib, "load", lambda: StubLib())
    monkeypatch.setattr(type(opt), "_get", lambda self: None)
    monkeypatch.setattr(type(opt), "dims", lambda self: (10, dims))
    got = opt.layout()
    for k, v in expect.items():
        assert got[k] == v, (k, got)


def test_config_default_matches_reference(ub):
    # config.rs:43-52, :117-127, :171-180, :226-235
    c = ub._lib.UmapConfigC()
    assert ub.lib().umap_config_default(C.byref(c)) == 0
    py = ub.UmapConfig.from_c(c)
    assert py == ub.UmapConfig()
    assert (py.n_components, py.manifold.min_dist, py.manifold.spread) == (2, np.float32(0.1), 1.0)
    assert (py.graph.n_neighbors, py.graph.local_connectivity, py.graph.set_op_mix_ratio) == (15, 1.0, 1.0)
    assert py.graph.disconnection_distance is None and py.graph.symmetrize is True
    assert py.optimization == ub.OptimizationParams(None, 1.0, 5, 1.0)


def test_config_roundtrip(ub):
    cfg = ub.UmapConfig(n_components=3, manifold=ub.ManifoldParams(0.25, 1.5, 1.2, 0.8),
                        graph=ub.GraphParams(30, 2.0, 0.5, 7.5, False),
                        optimization=ub.OptimizationParams(123, 0.5, 7, 2.0))
    assert ub.UmapConfig.from_c(cfg.to_c()) == cfg


@pytest.mark.parametrize("spread,min_dist", [(1.0, 0.1), (1.0, 0.0), (2.0, 0.5), (0.5, 0.25), (1.0, 0.99)])
def test_find_ab_params_bit_identical_to_oracle(ub, oracle, spread, min_dist):
    assert ub.find_ab_params(spread, min_dist) == oracle.find_ab_params(spread, min_dist)


def test_find_ab_params_memo_concurrent(ub, oracle):
    """The library memoises (a, b) per (spread, min_dist) for the process: concurrent callers
    (ctypes drops the GIL) with a mix of cached and new arguments all get the oracle's bits."""
    import threading
    args = [(1.0, 0.1), (1.5, 0.3), (0.7, 0.05), (2.0, 0.5), (1.25, 0.0)]
    want = {a: oracle.find_ab_params(*a) for a in args}
    got, errors = [], []

    def worker(k):
        try:
            for i in range(12):
                a = args[(k + i) % len(args)]
                got.append((a, ub.find_ab_params(*a)))
        except Exception as e:  # surfaced below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    assert len(got) == 8 * 12
    for a, ab in got:
        assert ab == want[a], (a, ab, want[a])


def _learn(ub, cfg, n, rows, cols):
    idx = np.zeros((rows, cols), np.uint32)
    dist = np.zeros((rows, cols), np.float32)
    return ub.Umap(cfg).learn_manifold(n, idx, dist)


@pytest.mark.parametrize("mutate,message", [
    (lambda c: setattr(c.graph, "set_op_mix_ratio", 1.5), "set_op_mix_ratio must be between 0.0 and 1.0, got 1.5"),
    (lambda c: setattr(c.graph, "n_neighbors", 1), "n_neighbors must be >= 2, got 1"),
    (lambda c: setattr(c.optimization, "repulsion_strength", -0.5), "repulsion_strength cannot be negative, got -0.5"),
    (lambda c: setattr(c.manifold, "min_dist", 2.0), "min_dist (2) must be <= spread (1)"),
    (lambda c: (setattr(c.manifold, "min_dist", -0.1)), "min_dist cannot be negative, got -0.1"),
    (lambda c: setattr(c.optimization, "learning_rate", -1.0), "learning_rate must be positive, got -1"),
    (lambda c: setattr(c, "n_components", 0), "n_components must be >= 1, got 0"),
])
def test_validation_messages(ub, mutate, message):
    # embedding.rs:339-429: each panic becomes UMAP_ERR_INVALID_ARGUMENT with the same text.
    cfg = ub.UmapConfig()
    mutate(cfg)
    with pytest.raises(ub.UmapError) as e:
        _learn(ub, cfg, 100, 100, cfg.graph.n_neighbors)
    assert e.value.code == ub.ERR_INVALID_ARGUMENT
    assert str(e.value) == message


def test_shape_messages(ub):
    cfg = ub.UmapConfig()
    with pytest.raises(ub.UmapError, match=r"^knn_dists has 10 neighbors but n_neighbors is 15$"):
        _learn(ub, cfg, 100, 100, 10)
    with pytest.raises(ub.UmapError, match=r"^knn_dists has 99 samples but data has 100 samples$"):
        _learn(ub, cfg, 100, 99, 15)
    with pytest.raises(ub.UmapError, match=r"^Number of samples \(15\) must be > n_neighbors \(15\)$"):
        _learn(ub, cfg, 15, 15, 15)
    with pytest.raises(ub.UmapError, match=r"^knn_dists and knn_indices must have the same shape"):
        ub.Umap(cfg).learn_manifold(100, np.zeros((100, 15), np.uint32), np.zeros((100, 14), np.float32))


def test_fit_init_shape_messages(ub):
    # embedding.rs:284-297 (checked before the manifold is learned)
    cfg = ub.UmapConfig()
    idx = np.zeros((100, 15), np.uint32)
    dist = np.zeros((100, 15), np.float32)
    with pytest.raises(ub.UmapError, match=r"^init has 3 components but n_components is 2$"):
        ub.Umap(cfg).fit(100, idx, dist, np.zeros((100, 3), np.float32))
    with pytest.raises(ub.UmapError, match=r"^init has 50 samples but data has 100 samples$"):
        ub.Umap(cfg).fit(100, idx, dist, np.zeros((50, 2), np.float32))


def test_null_and_moved_handles(ub):
    L = ub.lib()
    v = C.c_uint64()
    assert L.umap_manifold_n_vertices(None, C.byref(v)) == ub.ERR_NULL
    assert "NULL" in L.umap_last_error().decode()
    m = ub.LearnedManifold(None)
    with pytest.raises(ub.UmapError, match="moved or freed"):
        m.n_vertices()
    assert L.umap_manifold_free(None) == 0


def test_deserialize_rejects_garbage_without_gpu(ub):
    for fn in (ub.LearnedManifold.from_bytes, ub.Optimizer.from_bytes, ub.FittedUmap.from_bytes):
        with pytest.raises(ub.UmapError) as e:
            fn(b"not a checkpoint at all")
        assert e.value.code == ub.ERR_FORMAT
        with pytest.raises(ub.UmapError) as e:
            fn(b"")
        assert e.value.code == ub.ERR_FORMAT


def test_transform_is_todo_like_reference(ub):
    f = ub.FittedUmap(None)
    with pytest.raises(NotImplementedError, match="Transform not yet implemented"):
        f.transform(None, None, None)


def test_batch_validation_names_the_instance(ub):
    # checked on the host before any device work
    off = np.array([0, 100, 110], np.uint64)
    idx = np.zeros((110, 15), np.uint32)
    dist = np.zeros((110, 15), np.float32)
    init = np.zeros((110, 2), np.float32)
    with pytest.raises(ub.UmapError, match=r"^instance 1: Number of samples \(10\) must be > n_neighbors \(15\)$"):
        ub.Optimizer.batch(ub.UmapConfig(), off, idx, dist, init, 10)


def test_rust_ffi_is_generated_from_the_header():
    """include/umap_b200_ffi.rs (the Rust crate's extern "C" block) is current with the header:
    regenerating it changes nothing, every header entry point has a declaration, and the
    config struct lists the header's fields in order (the ctypes mirror's order too)."""
    import importlib.util
    import os
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("gen_rust_ffi", os.path.join(root, "include", "gen_rust_ffi.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    header = open(os.path.join(root, "include", "umap_b200.h")).read()
    committed = open(os.path.join(root, "include", "umap_b200_ffi.rs")).read()
    assert gen.render(header) == committed
    decl = set(re.findall(r"^(?:int|const char\s*\*)\s*(umap_\w+)\s*\(", gen._strip_comments(header), re.M))
    rust = set(re.findall(r"pub fn (umap_\w+)\(", committed))
    assert decl == rust and len(rust) > 60
    from umap_b200._lib import UmapConfigC
    fields = re.findall(r"^    pub (\w+): ", committed.split("pub struct umap_config {")[1].split("}")[0], re.M)
    assert fields == [f[0] for f in UmapConfigC._fields_]


def test_output_metric_checks_without_gpu(ub):
    """metric.rs / distances.rs on the host side: EuclideanMetric's distance and gradient
    (distances.rs:22-37, f32), the metric types and device ids that route Optimizer and
    Umap.fit, and the refusal of a metric with no device form before any GPU work."""
    import numpy as np
    x = np.float32([1.5, -2.0, 0.25])
    y = np.float32([0.5, 1.0, 0.25])
    d, g = ub.EuclideanMetric().distance(x, y)
    assert d == np.float32(np.sqrt(np.float32(1.0) + np.float32(9.0)))
    assert np.array_equal(g, (x - y) / np.float32(d + np.float32(1e-6)))
    assert ub.EuclideanMetric().metric_type() == ub.MetricType.Euclidean
    assert ub.GenericEuclideanMetric().metric_type() == ub.MetricType.Generic
    assert ub.GenericEuclideanMetric().device_metric() == ub.OUTPUT_METRIC_EUCLIDEAN
    assert ub.Metric().metric_type() == ub.MetricType.Generic and ub.Metric().device_metric() is None
    idx = np.zeros((20, 3), np.uint32)
    dist = np.zeros((20, 3), np.float32)
    init = np.zeros((20, 2), np.float32)
    with pytest.raises(ub.UmapError) as e:
        ub.Umap.with_metrics(ub.UmapConfig(), ub.EuclideanMetric(), ub.Metric()).fit(20, idx, dist, init)
    assert e.value.code == ub.ERR_UNSUPPORTED


@pytest.mark.parametrize("change,message", [
    ({"n_sub": 100}, "the subsample must have 128..n_samples rows"),
    ({"n_sub": 2000}, "the subsample must have 128..n_samples rows"),
    ({"data_dim": 0}, "data_dim must be 1..4096, got 0"),
    ({"data_dim": 5000}, "data_dim must be 1..4096, got 5000"),
    ({"n_components": 5}, "the warm start's network predicts 1..4 components"),
    ({"mlp_epochs": 0}, "sub_epochs, epochs and mlp_epochs must be positive"),
    # the config's own validation (embedding.rs:339-429) runs next
    ({"knn_cols": 1}, "knn_dists has 1 neighbors but n_neighbors is 15"),
])
def test_warm_start_argument_checks_without_gpu(ub, change, message):
    """umap_warm_start_fit_device refuses arguments that need no device before it touches
    the GPU: subsample size, feature count, component count, epoch counts, then the
    config's own validation."""
    from umap_b200 import _lib
    L = ub.lib()
    cfg = ub.UmapConfig()
    cfg.n_components = change.get("n_components", 2)
    c = cfg.to_c()
    wp = _lib.WarmStartParamsC()
    assert L.umap_warm_start_params_default(C.byref(wp)) == 0
    wp.mlp_epochs = change.get("mlp_epochs", wp.mlp_epochs)
    n, k = 1000, change.get("knn_cols", 15)
    buf_f = np.zeros(64, np.float32)   # never read: the call returns before any pointer is used
    buf_u = np.zeros(64, np.uint32)
    pf, pu = buf_f.ctypes.data_as(C.c_void_p), buf_u.ctypes.data_as(C.c_void_p)
    out = C.c_void_p()
    rc = L.umap_warm_start_fit_device(C.byref(c), C.byref(wp), pf, n, change.get("data_dim", 64), pu, pf, k, pu,
                                      change.get("n_sub", 300), pu, pf, None, C.byref(out), None, None)
    assert rc == ub.ERR_INVALID_ARGUMENT and not out.value
    assert L.umap_last_error().decode() == message
