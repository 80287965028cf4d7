"""Sharding across ranks (one process per GPU) with gloo on CPU, world size 2: whole chunks go to
ranks by LPT over their estimated cells, every read is owned by exactly one rank together with the
rest of its chunk, loads are balanced, and the per-rank scalars combine with one all-reduce."""
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
    wl = synth.config_batched(seed=3, n_chunks=7, chunk_len=2000, coverage=6)
    jobs = wl.jobs()
    off = np.zeros(len(wl.templates) + 1, np.int64)
    off[1:] = np.cumsum(np.bincount(wl.read_template, minlength=len(wl.templates)))
    mine, idx = shard.shard(jobs, rank, world, off)
    cost = int(shard.estimated_cells(mine, 25).sum())
    t = torch.tensor([cost, mine.n_jobs], dtype=torch.float64)
    tot = t.clone()
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    gathered = [None] * world
    dist.all_gather_object(gathered, idx.tolist())
    if rank == 0:
        q.put((gathered, float(tot[0]), float(tot[1]), float(mx[0]), int(shard.estimated_cells(jobs, 25).sum()),
               wl.read_template.tolist(), shard.chunk_costs(jobs, off, 25).tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_chunk_sharding_covers_every_read_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, tot_cost, tot_jobs, max_cost, all_cost, chunk_of, costs = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    n = len(chunk_of)
    owned = sorted(i for part in gathered for i in part)
    assert owned == list(range(n))
    assert tot_jobs == n
    assert tot_cost == all_cost
    # a chunk's reads all live on one rank: the ranks' chunk sets are disjoint
    chunk_sets = [{chunk_of[i] for i in part} for part in gathered]
    assert not (chunk_sets[0] & chunk_sets[1])
    assert max_cost <= 0.5 * all_cost + max(costs)  # LPT: within one chunk of an even split


def test_lpt_assignment_balances():
    costs = np.array([10, 9, 8, 7, 6, 5, 4, 3, 2, 1])
    parts = shard.assign_lpt(costs, 3)
    loads = [int(costs[p].sum()) for p in parts]
    assert sum(loads) == costs.sum() and max(loads) - min(loads) <= 2
