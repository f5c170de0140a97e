"""GPU test of the allocation-free sort entry point (umap_radix_sort_pairs_device_noalloc).

That entry point serves callers that cannot allocate device memory when they sort (a host
application whose allocator owns the whole GPU heap, or a loop that must not enter the CUDA
allocator): its scratch is a static device array, so it makes no allocation.  Here it is
called through the C ABI and its output is compared with the allocating entry point's on
two consecutive calls (the second one reuses the scratch the first one left behind).  The
sort is integer work, so the comparison is exact.  This file is collected last so that a
run stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _warm_up(ub):
    """The per-device first call a caller that reserves the heap makes up front: n = 0 with
    NULL buffers loads the scratch array and looks up its address, and queues no work."""
    assert ub.lib().umap_radix_sort_pairs_device_noalloc(None, None, None, None, 0, 32, None) == 0, \
        ub.lib().umap_last_error()


def _sort(ub, fn, keys, vals, bits, noalloc, stream=None):
    import torch
    n = keys.size
    tk = torch.from_numpy(keys.view(np.int32)).cuda()
    tv = torch.from_numpy(vals.view(np.int32)).cuda() if vals is not None else None
    ok = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    ov = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    args = [C.c_void_p(tk.data_ptr()), C.c_void_p(tv.data_ptr()) if tv is not None else None,
            C.c_void_p(ok.data_ptr()), C.c_void_p(ov.data_ptr()), n, bits]
    if noalloc:
        args.append(C.c_void_p(stream.cuda_stream) if stream is not None else None)  # NULL: default stream
    torch.cuda.synchronize()
    rc = getattr(ub.lib(), fn)(*args)
    assert rc == 0, ub.lib().umap_last_error()
    return ok[:n].cpu().numpy().view(np.uint32), ov[:n].cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_allocating_sort_on_two_calls(ub):
    _warm_up(ub)
    g = np.random.Generator(np.random.PCG64(2024))
    cases = [
        (g.integers(0, 1 << 21, 1_000_003, dtype=np.uint64).astype(np.uint32),
         g.integers(0, 1 << 32, 1_000_003, dtype=np.uint64).astype(np.uint32), 21),
        (g.integers(0, 1 << 32, 777_777, dtype=np.uint64).astype(np.uint32), None, 32),
    ]
    for keys, vals, bits in cases:
        ref_k, ref_v = _sort(ub, "umap_radix_sort_pairs_device", keys, vals, bits, noalloc=False)
        got_k, got_v = _sort(ub, "umap_radix_sort_pairs_device_noalloc", keys, vals, bits, noalloc=True)
        assert np.array_equal(got_k, ref_k)
        assert np.array_equal(got_v, ref_v)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(got_k, keys[order])


def test_noalloc_sort_rejects_sizes_beyond_its_scratch(ub):
    import torch
    L = ub.lib()
    mx = C.c_uint64()
    assert L.umap_radix_sort_noalloc_max_pairs(C.byref(mx)) == 0
    assert mx.value == 1 << 20
    buf = torch.empty(16, dtype=torch.int32, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    rc = L.umap_radix_sort_pairs_device_noalloc(p, p, p, p, mx.value + 1, 32, None)
    assert rc == ub.ERR_INVALID_ARGUMENT
    assert "at most 1048576 pairs" in L.umap_last_error().decode()


def test_noalloc_sort_at_its_maximum_size_on_a_side_stream(ub):
    """Exactly umap_radix_sort_noalloc_max_pairs() pairs (the size the scratch carving is laid
    out for) with all 32 key bits, with and without values, queued on a non-default stream;
    two calls in a row, each against the allocating sort and numpy's stable argsort."""
    import torch
    _warm_up(ub)
    mx = C.c_uint64()
    assert ub.lib().umap_radix_sort_noalloc_max_pairs(C.byref(mx)) == 0
    n = mx.value
    g = np.random.Generator(np.random.PCG64(77))
    side = torch.cuda.Stream()
    for with_vals in (True, False):
        keys = g.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
        keys[::1000] = keys[0]  # runs of equal keys: stability is visible
        vals = g.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32) if with_vals else None
        ref_k, ref_v = _sort(ub, "umap_radix_sort_pairs_device", keys, vals, 32, noalloc=False)
        order = np.argsort(keys, kind="stable")
        want_v = vals[order] if with_vals else order.astype(np.uint32)
        for _ in range(2):
            got_k, got_v = _sort(ub, "umap_radix_sort_pairs_device_noalloc", keys, vals, 32, noalloc=True,
                                 stream=side)
            assert np.array_equal(got_k, ref_k) and np.array_equal(got_v, ref_v)
            assert np.array_equal(got_k, keys[order]) and np.array_equal(got_v, want_v)


def test_sorts_reject_overlapping_buffers(ub):
    """An output that shares memory with an input (or the other output) is refused by both
    sort entry points before any work is queued."""
    import torch
    buf = torch.empty(4096, dtype=torch.int32, device="cuda")
    p0 = C.c_void_p(buf.data_ptr())
    p1 = C.c_void_p(buf.data_ptr() + 4 * 1024)
    p2 = C.c_void_p(buf.data_ptr() + 4 * 2048)
    L = ub.lib()
    for fn, extra in (("umap_radix_sort_pairs_device", []), ("umap_radix_sort_pairs_device_noalloc", [None])):
        f = getattr(L, fn)
        assert f(p0, None, p0, p1, 1024, 21, *extra) == ub.ERR_INVALID_ARGUMENT       # keys in place
        assert f(p0, p1, p2, C.c_void_p(buf.data_ptr() + 4 * 2500), 1024, 21, *extra) == ub.ERR_INVALID_ARGUMENT
        assert "must not overlap" in L.umap_last_error().decode()
