"""Events across ranks (no GPU): the cell-balanced partition, and the
host-side reductions a sharded batched run ends with, on two gloo ranks
(processes started with spawn, rendezvous on 127.0.0.1)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from echo_gpu import events as EV
from echo_gpu import shard as SH


def test_partition_covers_and_balances():
    cells = EV.batched_viscous().cells
    for world in (1, 2, 3, 8):
        parts = SH.partition_by_cells(cells, world)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(len(cells)))
        loads = np.array([cells[p].sum() for p in parts])
        assert loads.max() - cells.sum() / world < cells.max()
        assert all(np.all(np.diff(p) > 0) for p in parts)
    with pytest.raises(ValueError):
        SH.partition_by_cells(cells, 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cells = EV.batched_viscous(nev=40).cells
        mine = SH.partition_by_cells(cells, world)[rank]
        # stand-in results of this rank's batch: steps = 10 + event index
        status = [{"steps": 10 + int(e), "state": 1} for e in mine]
        cu = float(sum(cells[e] * (10 + int(e)) for e in mine))
        total = SH.reduce_sum(cu)
        slowest = SH.reduce_max(1.0 + rank)
        full = SH.gather_status(mine, status, len(cells))
        if rank == 0:
            q.put((total, slowest, [s["steps"] for s in full]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    total, slowest, steps = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cells = EV.batched_viscous(nev=40).cells
    assert total == float(sum(cells[e] * (10 + e) for e in range(40)))
    assert slowest == 2.0
    assert steps == [10 + e for e in range(40)]
