"""Checkpoints in the reference's own encoding (serde derive + bincode 1.3, as its tests use:
umap-rs/src/tests.rs:150, :179, :207).  The expected bytes are built here field by field
from the documented layout with numpy (little-endian fixed-width numbers, u64 sequence
lengths, u8 Option tags, u32 unit-enum indices; ndarray {v: 1, dim, data}; sprs CSR
{storage 0, nrows, ncols, indptr, indices, data}), so a change of field order or encoding
fails here.  No Rust-written file exists to compare with: parity with the reference's bytes
is unpinned beyond this restatement."""
import struct

import numpy as np
import pytest


def _seq(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    return struct.pack("<Q", a.size) + a.tobytes()


def _nd1(a, dtype):
    a = np.asarray(a)
    return struct.pack("<BQ", 1, a.size) + _seq(a, dtype)


def _nd2(a, dtype):
    a = np.asarray(a)
    return struct.pack("<BQQ", 1, a.shape[0], a.shape[1]) + _seq(a.ravel(), dtype)


def manifold_bytes(indptr, indices, data, sigmas, rhos, a, b):
    n = len(indptr) - 1
    return (struct.pack("<IQQ", 0, n, n) + _seq(indptr, "<u8") + _seq(indices, "<u4") + _seq(data, "<f4")
            + _nd1(sigmas, "<f4") + _nd1(rhos, "<f4") + struct.pack("<Qff", n, a, b))


def opt_f32(v):
    return struct.pack("<B", 0) if v is None else struct.pack("<Bf", 1, v)


def config_bytes(c):
    m, g, o = c.manifold, c.graph, c.optimization
    return (struct.pack("<Q", c.n_components) + struct.pack("<ff", m.min_dist, m.spread) + opt_f32(m.a)
            + opt_f32(m.b) + struct.pack("<Qff", g.n_neighbors, g.local_connectivity, g.set_op_mix_ratio)
            + opt_f32(g.disconnection_distance) + struct.pack("<B", int(g.symmetrize))
            + (struct.pack("<B", 0) if o.n_epochs is None else struct.pack("<BQ", 1, o.n_epochs))
            + struct.pack("<fQf", o.learning_rate, o.negative_sample_rate, o.repulsion_strength))


def test_garbage_rejected_without_gpu(ub):
    for fn in (ub.LearnedManifold.from_bincode, ub.Optimizer.from_bincode, ub.FittedUmap.from_bincode):
        for b in (b"", b"\x01\x00", b"not a checkpoint at all, just text"):
            with pytest.raises(ub.UmapError) as e:
                fn(b)
            assert e.value.code == ub.ERR_FORMAT


@pytest.mark.gpu
def test_manifold_bytes_match_layout_and_round_trip(ub, ring):
    idx, dist, init = ring
    cfg = ub.UmapConfig()
    cfg.graph.n_neighbors = 10
    m = ub.Umap(cfg).learn_manifold(50, idx, dist)
    G = m.graph()
    s, r = m.sigmas_rhos()
    a, b = m.curve_params()
    got = m.to_bincode()
    assert got == manifold_bytes(G.indptr, G.indices, G.data, s, r, a, b)
    m2 = ub.LearnedManifold.from_bincode(got)
    G2 = m2.graph()
    assert np.array_equal(G2.indptr, G.indptr) and np.array_equal(G2.indices, G.indices)
    assert np.array_equal(G2.data, G.data) and m2.curve_params() == (a, b)
    assert m2.to_bincode() == got


@pytest.mark.gpu
def test_fitted_bytes_match_layout_and_round_trip(ub, ring):
    idx, dist, init = ring
    cfg = ub.UmapConfig()
    cfg.graph.n_neighbors = 10
    cfg.optimization.n_epochs = 10
    cfg.graph.disconnection_distance = 5.0
    f = ub.Umap(cfg).fit(50, idx, dist, init)
    man = f.manifold()
    G = man.graph()
    s, r = man.sigmas_rhos()
    a, b = man.curve_params()
    expect = (_nd2(f.embedding(), "<f4") + manifold_bytes(G.indptr, G.indices, G.data, s, r, a, b)
              + config_bytes(f.config()))
    got = f.to_bincode()
    assert got == expect
    f2 = ub.FittedUmap.from_bincode(got)
    assert np.array_equal(f2.embedding(), f.embedding())
    assert f2.config() == f.config()
    assert f2.to_bincode() == got


@pytest.mark.gpu
def test_optimizer_round_trip_resumes(ub, ring):
    """Checkpoint mid-fit in the reference's encoding, load, and continue: the loaded
    optimizer carries the same epoch counters, edges and schedule and finishes the fit."""
    idx, dist, init = ring
    cfg = ub.UmapConfig()
    cfg.graph.n_neighbors = 10
    cfg.optimization.n_epochs = 40
    opt = ub.Optimizer(ub.Umap(cfg).learn_manifold(50, idx, dist), init, 40, cfg)
    opt.step_epochs(15)
    raw = opt.to_bincode()
    h, t, e, eons, eonns, epns = opt.export_edges()
    man = opt.manifold()
    G = man.graph()
    s, r = man.sigmas_rhos()
    a, b = man.curve_params()
    expect = (manifold_bytes(G.indptr, G.indices, G.data, s, r, a, b) + _nd1(h, "<u4") + _nd1(t, "<u4")
              + _nd1(e, "<f8") + _nd2(opt.embedding(), "<f4") + _nd1(eons, "<f8") + _nd1(eonns, "<f8")
              + _nd1(epns, "<f8") + struct.pack("<QQffdI", 15, 40, cfg.optimization.repulsion_strength,
                                                cfg.optimization.learning_rate, 5.0, 0))
    assert raw == expect
    opt2 = ub.Optimizer.from_bincode(raw)
    assert (opt2.current_epoch(), opt2.total_epochs(), opt2.n_edges()) == (15, 40, len(h))
    assert np.array_equal(opt2.embedding(), opt.embedding())
    h2, t2, e2, eons2, eonns2, epns2 = opt2.export_edges()
    assert np.array_equal(h2, h) and np.array_equal(t2, t) and np.array_equal(e2, e)
    assert np.array_equal(eons2, eons) and np.array_equal(eonns2, eonns)
    opt2.step_epochs(25)
    assert opt2.remaining_epochs() == 0 and np.isfinite(opt2.embedding()).all()
    with pytest.raises(ub.UmapError) as err:
        ub.Optimizer.from_bincode(raw[:-3])
    assert err.value.code == ub.ERR_FORMAT
