"""Multi-GPU layout of the path: replicas, one process per GPU.

Primaries are independent, so a scan shards by primary with no exchange
during transport (the reference runs one driver per device over a shared
host queue, gpu_main.cu:284-295).  Two layouts:

* weak: every rank runs the whole workload with its own seed (per-GPU work
  fixed as ranks are added) -- what bench.py reports;
* strong: the scan's primaries are split into contiguous ranges, one per
  rank, and the per-pixel tallies are summed once at the end.

The only collectives are the end-of-run ones below (max of the per-rank
device time, sum of tallies); nothing crosses GPUs on the data path.
"""
from __future__ import annotations

import numpy as np


def shard(n, rank, world):
    """Contiguous [start, stop) of n items for rank (sizes differ by <= 1)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def replica_seed(base_seed, rank):
    """Seed of a weak-scaling replica (independent Philox key per rank)."""
    return (int(base_seed) + 0x9E3779B97F4A7C15 * (rank + 1)) & 0xFFFFFFFFFFFFFFFF


def max_over_ranks(value, dist, device=None):
    """Max of a float over all ranks (the timing rule: slowest rank)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_tallies(arrays, dist, device=None):
    """Element-wise sum of per-rank tallies (uint32/float arrays)."""
    import torch
    out = []
    for a in arrays:
        t = torch.from_numpy(np.ascontiguousarray(a).astype(np.float64)).to(device if device else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        out.append(t.cpu().numpy())
    return out
