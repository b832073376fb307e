"""Work split across ranks, one process per GPU.

A single problem is not split: its tree and far lists would need a halo
exchange between ranks, so ranks run independent replicas (weak scaling).
A forest of independent problems is split by problem with no collective on
the data path: each rank solves its share and keeps its own results; only
timings are reduced across ranks.
"""
from __future__ import annotations

import heapq

import numpy as np


def forest_shard(sizes, world: int, rank: int) -> np.ndarray:
    """Problem indices assigned to `rank`: largest problem first to the rank
    with the least work so far (longest-processing-time rule, work = points),
    ties to the lower rank.  Every problem lands on exactly one rank, and no
    rank exceeds the even share by more than the largest problem."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    sizes = np.asarray(sizes, dtype=np.int64)
    order = np.argsort(-sizes, kind="stable")
    heap = [(0, r) for r in range(world)]
    owner = np.empty(len(sizes), dtype=np.int64)
    for p in order:
        load, r = heapq.heappop(heap)
        owner[p] = r
        heapq.heappush(heap, (load + int(sizes[p]), r))
    return np.flatnonzero(owner == rank)


def sub_forest(toff, soff, problems):
    """Offsets of the sub-forest made of `problems` (in the given order) and
    the index arrays that gather its targets and sources from the full forest."""
    toff = np.asarray(toff, dtype=np.int64)
    soff = np.asarray(soff, dtype=np.int64)
    tidx = [np.arange(toff[p], toff[p + 1]) for p in problems]
    sidx = [np.arange(soff[p], soff[p + 1]) for p in problems]
    nt = np.array([len(a) for a in tidx], dtype=np.int64)
    ns = np.array([len(a) for a in sidx], dtype=np.int64)
    sub_toff = np.concatenate([[0], np.cumsum(nt)]).astype(np.int64)
    sub_soff = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    cat = lambda parts: np.concatenate(parts) if parts else np.zeros(0, dtype=np.int64)
    return sub_toff, sub_soff, cat(tidx), cat(sidx)


def max_over_ranks(values, device=None):
    """Element-wise maximum of `values` over all ranks of the default process
    group (identity without one).  Every rank must call it, in the same order
    as its other collectives."""
    import torch
    import torch.distributed as dist
    vals = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(vals, op=dist.ReduceOp.MAX)
    return [float(v) for v in vals.cpu()]
