"""Sharding of independent reads across GPUs (one process per GPU).

Reads of different chunks -- and reads within a chunk, up to the POA update --
are independent (the reference runs chunks in parallel, marginPolish.c:436-439),
so a batch splits across ranks with no data-path collective: each rank runs the
posterior pass on its own subset and only per-rank scalars are combined.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence

import numpy as np

from .realign import Jobs


def assign_lpt(costs: Sequence[int], world: int) -> List[np.ndarray]:
    """Longest-processing-time assignment of items to `world` ranks (balanced by cost)."""
    costs = np.asarray(costs, dtype=np.int64)
    order = np.argsort(-costs, kind="stable")
    heap = [(0, r) for r in range(world)]
    owners = np.empty(costs.size, dtype=np.int64)
    for i in order:
        load, r = heapq.heappop(heap)
        owners[i] = r
        heapq.heappush(heap, (load + int(costs[i]), r))
    return [np.sort(np.nonzero(owners == r)[0]) for r in range(world)]


def subset(jobs: Jobs, idx: np.ndarray) -> Jobs:
    """The jobs `idx` of a batch (templates are shared, reads and anchors are copied)."""
    idx = np.asarray(idx, dtype=np.int64)
    ys, yo, an, ao = [], [0], [], [0]
    for j in idx:
        y = jobs.y_symbols[jobs.y_offsets[j]:jobs.y_offsets[j + 1]]
        a = jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]]
        ys.append(y)
        an.append(a)
        yo.append(yo[-1] + y.size)
        ao.append(ao[-1] + a.shape[0])

    def pick(v):
        return None if v is None else v[idx]

    return Jobs(jobs.x_symbols, jobs.x_begin[idx], jobs.x_end[idx],
                np.concatenate(ys) if ys else np.zeros(0, np.uint16), np.asarray(yo, np.int64),
                np.concatenate(an) if an else np.zeros((0, 3), np.int32), np.asarray(ao, np.int64),
                jobs.strand[idx], pick(jobs.ragged_left), pick(jobs.ragged_right), pick(jobs.x_shift))


def estimated_cells(jobs: Jobs, half_width: int) -> np.ndarray:
    """Cheap per-job cost estimate: anti-diagonals x band cells."""
    lx = jobs.x_end - jobs.x_begin
    ly = np.diff(jobs.y_offsets)
    return (lx + ly + 1) * (2 * half_width + 2)


def shard(jobs: Jobs, rank: int, world: int, half_width: int = 25) -> tuple[Jobs, np.ndarray]:
    """This rank's share of a batch and the indices of its jobs in the batch."""
    parts = assign_lpt(estimated_cells(jobs, half_width), world)
    return subset(jobs, parts[rank]), parts[rank]
