"""Events across GPUs: one process per GPU, each running its own share of a
batch; no collective on the data path.

The reference's Monte Carlo events are independent (one grid each, echo.f90
events loop), so a many-event workload shards by events: every rank takes a
subset whose cell counts are balanced (greedy longest-processing-time
assignment), runs it as its own batch, and only scalars cross ranks
afterwards -- the total of cell-updates, the slowest rank's time, the
per-event status gathered on rank 0.  The helpers take the process group
torch.distributed was initialised with (NCCL on the GPUs, gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def partition_by_cells(cells, world: int) -> list[np.ndarray]:
    """Event indices of every rank: events in decreasing cell count, each to
    the rank with the fewest cells so far (ties to the lower rank); every
    rank's indices sorted.  The largest rank load exceeds the mean by less
    than the largest event."""
    cells = np.asarray(cells, dtype=np.int64)
    if world < 1:
        raise ValueError("world must be >= 1")
    load = np.zeros(world, dtype=np.int64)
    owner = np.empty(len(cells), dtype=np.int64)
    for e in np.argsort(-cells, kind="stable"):
        r = int(np.argmin(load))
        owner[e] = r
        load[r] += cells[e]
    return [np.sort(np.nonzero(owner == r)[0]) for r in range(world)]


def _tensor(x, device):
    import torch

    return torch.tensor([float(x)], dtype=torch.float64, device=device)


def reduce_max(x: float, device="cpu") -> float:
    """Maximum of x over the ranks (the slowest rank's time)."""
    import torch.distributed as dist

    t = _tensor(x, device)
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x: float, device="cpu") -> float:
    """Sum of x over the ranks (cell-updates of the whole job)."""
    import torch.distributed as dist

    t = _tensor(x, device)
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_status(local_idx, local_status: list[dict], nev: int) -> list[dict] | None:
    """Every event's status on rank 0, in event order (None on other ranks).
    local_idx[i] is the global index of this rank's i-th event."""
    import torch.distributed as dist

    mine = list(zip([int(i) for i in local_idx], local_status))
    if not (dist.is_initialized() and dist.get_world_size() > 1):
        parts = [mine]
    else:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, mine)
        if dist.get_rank() != 0:
            return None
    out: list = [None] * nev
    for part in parts:
        for i, st in part:
            out[i] = st
    if any(s is None for s in out):
        raise RuntimeError("an event has no status: the shards do not cover the batch")
    return out
