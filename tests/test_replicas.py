"""The N > 1 path on CPU: cost-balanced sharding of independent instances, and the rank
plumbing (max-over-ranks timing, sums, barrier) run as two gloo processes on 127.0.0.1."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_by_cost_covers_and_balances():
    from umap_b200 import replicas as R
    from umap_b200 import workloads as W
    sizes = W.instance_sizes(4096)
    for world in (1, 2, 3, 4, 8):
        ranges = R.shard_by_cost(sizes, world)
        assert len(ranges) == world and ranges[0][0] == 0 and ranges[-1][1] == len(sizes)
        assert all(a <= b for a, b in ranges)
        assert all(ranges[i][1] == ranges[i + 1][0] for i in range(world - 1))
        loads = [float(sizes[a:b].sum()) for a, b in ranges]
        assert max(loads) <= sizes.sum() / world + sizes.max(), (world, loads)


def test_shard_by_cost_edge_cases():
    from umap_b200 import replicas as R
    assert R.shard_by_cost([], 3) == [(0, 0), (0, 0), (0, 0)]
    r = R.shard_by_cost([5.0], 4)
    assert sum(b - a for a, b in r) == 1
    r = R.shard_by_cost(np.zeros(10), 3)
    assert r[0][0] == 0 and r[-1][1] == 10 and sum(b - a for a, b in r) == 10
    with pytest.raises(ValueError):
        R.shard_by_cost([1.0, -1.0], 2)


def _worker(rank, world, port, costs, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "umap-rs_b200"))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        from umap_b200 import replicas as R
        assert R.env() == (rank, world, rank)
        assert R.init("gloo", timeout_s=60)
        a, b = R.shard_by_cost(costs, world)[rank]
        mine = float(np.sum(costs[a:b]))
        total = R.sum_over_ranks(mine)
        slowest = R.max_over_ranks(10.0 + rank)
        n_units = R.sum_over_ranks(b - a)
        R.barrier()
        q.put((rank, a, b, total, slowest, n_units))
        R.finalize()
    except BaseException as e:  # reported to the parent
        q.put((rank, "error", repr(e)))


def test_two_gloo_ranks_shard_and_reduce():
    import torch.multiprocessing as mp
    costs = np.random.default_rng(0).integers(500, 50000, 37).astype(np.float64)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert all(o[1] != "error" for o in out), out
    (r0, a0, b0, t0, s0, n0), (r1, a1, b1, t1, s1, n1) = out
    assert (a0, b1) == (0, len(costs)) and b0 == a1
    assert t0 == t1 == float(costs.sum())
    assert s0 == s1 == 11.0
    assert n0 == n1 == len(costs)
