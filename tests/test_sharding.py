"""Scene-parallel placement and metric reduction across ranks (gloo, CPU)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from mpm_b200 import scenes
from mpm_b200.sharding import partition, reduce_step_metrics, scenes_for_rank


def test_partition_covers_and_balances():
    w = np.random.default_rng(0).integers(1, 1000, 200)
    for ws in (1, 2, 3, 8):
        parts = partition(w, ws)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(w)))
        loads = [w[p].sum() for p in parts]
        assert max(loads) - min(loads) <= w.max()
    assert partition([5, 5, 5], 2) == partition([5, 5, 5], 2)  # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    import torch
    scs = scenes.batched_scenes(count=12, scale=0.01)
    mine = scenes_for_rank(scs, rank, ws)
    names = [s.name for s in mine]
    gathered = [None] * ws
    dist.all_gather_object(gathered, names)

    def allsum(x):
        t = torch.tensor([x], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def allmax(x):
        t = torch.tensor([x], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    work = sum(s.n for s in mine) * 10
    rate, total, t = reduce_step_metrics(work, 1.0 + rank, allsum, allmax)
    if rank == 0:
        out.put((gathered, rate, total, t, [s.name for s in scs], sum(s.n for s in scs) * 10))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_scene_placement_gloo():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    gathered, rate, total, t, all_names, all_work = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    flat = sorted(n for part in gathered for n in part)
    assert flat == sorted(all_names) and not set(gathered[0]) & set(gathered[1])
    assert total == pytest.approx(all_work) and t == pytest.approx(2.0) and rate == pytest.approx(all_work / 2.0)
