"""Multi-GPU plumbing: one process per GPU (torchrun / torch.distributed).

A single fit does not shard: its Hogwild epochs update one embedding in place, and splitting
it across GPUs would need a per-epoch exchange of the whole embedding that changes the
reference's update semantics (optimizer.rs:297-366).  Several GPUs therefore run independent
work with no data-path collective:

* replicas: every rank runs the same fit (weak scaling);
* shards: a batch of independent instances is cut into contiguous, cost-balanced ranges of
  instances, one per rank (the batched workload).

The only collectives are the timing reduction (max over ranks), scalar sums and a barrier.
"""
from __future__ import annotations

import datetime
import os

import numpy as np


def env():
    """(rank, world_size, local_rank) from the torchrun environment (defaults 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 600.0) -> bool:
    """Joins the process group when WORLD_SIZE > 1; returns whether it did."""
    _, world, _ = env()
    if world <= 1:
        return False
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return True


def shard_by_cost(costs, world: int):
    """Contiguous ranges [(start, end)] of the units 0..len(costs)-1, one per rank, cut at
    the cost quantiles: rank r gets the units whose cost prefix lies in
    [r * total / world, (r + 1) * total / world).  Every unit lands in exactly one range;
    a range can be empty when there are fewer units than ranks."""
    c = np.asarray(costs, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    if c.ndim != 1 or (c < 0).any():
        raise ValueError("costs must be a 1-D array of non-negative values")
    n = len(c)
    prefix = np.concatenate([[0.0], np.cumsum(c)])
    total = prefix[-1]
    cuts = [0]
    for r in range(1, world):
        # first unit whose cost midpoint reaches the quantile
        mid = (prefix[:-1] + prefix[1:]) / 2.0
        cuts.append(int(np.searchsorted(mid, r * total / world, side="left")) if total > 0 else (r * n) // world)
    cuts.append(n)
    cuts = np.maximum.accumulate(np.asarray(cuts))
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(world)]


def _reduce(x: float, op, device):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x: float, device="cpu") -> float:
    """Maximum of a per-rank value (device times: the job is done when its slowest rank is)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX, device)


def sum_over_ranks(x: float, device="cpu") -> float:
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM, device)


def barrier(device=None):
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        if device is not None and dist.get_backend() == "nccl":
            dist.barrier(device_ids=[device.index if hasattr(device, "index") else int(device)])
        else:
            dist.barrier()


def finalize():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
