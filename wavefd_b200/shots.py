"""Shot-level parallelism across GPUs (one process per GPU, torch.distributed).

The path shards by shot: shots are independent units, so ranks share no data during
propagation; the only collective is the reduction of the image (or of per-rank timings) at the
end of a batch.
"""
from __future__ import annotations

import numpy as np


def partition_shots(nshots: int, world: int, rank: int):
    """Contiguous, balanced split of shot indices 0..nshots-1 over `world` ranks."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(nshots, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def partition_by_cost(costs, world: int, rank: int):
    """Greedy longest-processing-time assignment of shots with uneven costs (cells x steps)."""
    order = np.argsort(-np.asarray(costs, dtype=np.float64), kind="stable")
    load = np.zeros(world)
    owner = np.empty(len(costs), dtype=np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += costs[i]
    return [int(i) for i in range(len(costs)) if owner[i] == rank]


def reduce_max(value: float, device=None) -> float:
    """Max over ranks of a per-rank number (e.g. elapsed device time)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_image(image, dst: int = 0):
    """Sum the per-rank partial images into rank `dst` (in place), one collective per batch."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return image
    dist.reduce(image, dst=dst, op=dist.ReduceOp.SUM)
    return image
