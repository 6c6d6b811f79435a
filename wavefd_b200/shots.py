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


class ShotLedger:
    """Shot-level resume: an append-only file of the shots whose results are saved.

    The reference keeps no record of finished work (a run that stops is run again). Here each rank
    records a shot after its contribution is safely stored (`done`, one line written and flushed to
    disk per shot), and a restarted job asks for the shots still to do (`pending`). Lines are
    "rank shot" text; a line cut short by a crash is ignored (and dropped when that rank's ledger is
    opened again, before it appends). Ranks write to their own file
    (path + ".rank<r>"), so no locking is needed; `pending` reads every rank's file.
    """

    def __init__(self, path: str, rank: int = 0):
        import os
        self.base = str(path)
        self.rank = int(rank)
        self.path = f"{self.base}.rank{self.rank}"
        d = os.path.dirname(self.path)
        if d:
            os.makedirs(d, exist_ok=True)
        # a record cut short by a crash (no newline) is dropped before this rank appends again
        if os.path.exists(self.path):
            with open(self.path, "rb+") as f:
                data = f.read()
                if data and not data.endswith(b"\n"):
                    f.truncate(data.rfind(b"\n") + 1)

    def done(self, shot: int):
        import os
        with open(self.path, "a") as f:
            f.write(f"{self.rank} {int(shot)}\n")
            f.flush()
            os.fsync(f.fileno())

    def finished(self):
        import glob
        out = set()
        for p in glob.glob(f"{self.base}.rank*"):
            with open(p) as f:
                for line in f:
                    if not line.endswith("\n"):
                        continue  # cut short
                    parts = line.split()
                    if len(parts) == 2 and parts[1].lstrip("-").isdigit():
                        out.add(int(parts[1]))
        return out

    def pending(self, shots):
        fin = self.finished()
        return [s for s in shots if s not in fin]
