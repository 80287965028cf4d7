"""Sharding across ranks (one process per GPU) with gloo on CPU, world size 2: every read is owned by
exactly one rank, loads are balanced, and the per-rank scalars combine with one all-reduce."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from marginpolish_b200 import shard, synth


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    jobs = synth.config_small(seed=3, n_reads=11).jobs()
    mine, idx = shard.shard(jobs, rank, world)
    cost = int(shard.estimated_cells(mine, 25).sum())
    t = torch.tensor([cost, mine.n_jobs], dtype=torch.float64)
    tot = t.clone()
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    gathered = [None] * world
    dist.all_gather_object(gathered, idx.tolist())
    if rank == 0:
        q.put((gathered, float(tot[0]), float(tot[1]), float(mx[0]), int(shard.estimated_cells(jobs, 25).sum())))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_covers_every_read_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, tot_cost, tot_jobs, max_cost, all_cost = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    owned = sorted(i for part in gathered for i in part)
    assert owned == list(range(11))
    assert tot_jobs == 11
    assert tot_cost == all_cost
    assert max_cost <= 0.75 * all_cost  # balanced to within a read's worth


def test_lpt_assignment_balances():
    costs = np.array([10, 9, 8, 7, 6, 5, 4, 3, 2, 1])
    parts = shard.assign_lpt(costs, 3)
    loads = [int(costs[p].sum()) for p in parts]
    assert sum(loads) == costs.sum() and max(loads) - min(loads) <= 2
