"""Sharding of chunks across GPUs (one process per GPU).

Chunks are independent (the reference runs them in parallel, marginPolish.c:436-439),
and a chunk's reads must stay together, since its POA update folds all of them
into one graph. A batch therefore splits across ranks by whole chunks, assigned
greedily longest-processing-time first by their estimated cells, with the model
tables replicated and no data-path collective: each rank runs the posterior pass
(and the polishing loop) on its own chunks, and only per-rank scalars are combined.
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


def chunk_costs(jobs: Jobs, chunk_offsets: np.ndarray, half_width: int) -> np.ndarray:
    """Estimated cells of each chunk (its jobs are chunk_offsets[c] .. chunk_offsets[c+1]-1)."""
    per_job = estimated_cells(jobs, half_width)
    csum = np.concatenate([[0], np.cumsum(per_job)])
    off = np.asarray(chunk_offsets, dtype=np.int64)
    return csum[off[1:]] - csum[off[:-1]]


def shard_chunks(chunk_offsets: np.ndarray, costs: np.ndarray, rank: int, world: int) -> tuple[np.ndarray, np.ndarray]:
    """This rank's chunks (LPT over the chunk costs) and the indices of their jobs, in chunk order."""
    off = np.asarray(chunk_offsets, dtype=np.int64)
    chunks = assign_lpt(costs, world)[rank]
    idx = (np.concatenate([np.arange(off[c], off[c + 1]) for c in chunks]) if chunks.size
           else np.zeros(0, np.int64))
    return chunks, idx


def shard(jobs: Jobs, rank: int, world: int, chunk_offsets: np.ndarray = None,
          half_width: int = 25) -> tuple[Jobs, np.ndarray]:
    """This rank's share of a batch (whole chunks) and the indices of its jobs in the batch.
    chunk_offsets (n_chunks + 1 job offsets) defaults to one chunk per job."""
    if chunk_offsets is None:
        chunk_offsets = np.arange(jobs.n_jobs + 1, dtype=np.int64)
    _, idx = shard_chunks(chunk_offsets, chunk_costs(jobs, chunk_offsets, half_width), rank, world)
    return subset(jobs, idx), idx
