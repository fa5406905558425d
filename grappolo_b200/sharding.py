"""Batches of independent graphs across GPUs: one process per GPU, no collective
on the data path.

A batch of graphs (the 4,096-graph workload) splits into per-rank shards of
about equal work: graphs are taken largest first and each goes to the rank
with the least estimated work so far (longest-processing-time-first, within
4/3 of the best split).  Every rank runs its shard as batched persistent
launches on its own GPU; the per-graph results are then gathered on the host
of every rank, in the batch's original graph order.  The only collectives are
the host-side gather of the results and the timing reduction.
"""
from __future__ import annotations

import heapq

import numpy as np


def shard_by_work(work, world: int) -> list[np.ndarray]:
    """Graph indices of each rank's shard, each in ascending order.

    `work` holds one estimate per graph (expected CSR entries); every graph is
    in exactly one shard.  Deterministic: equal estimates go to the lower
    graph index first and ties between ranks to the lower rank."""
    work = np.asarray(work, dtype=np.float64)
    if world < 1:
        raise ValueError('world must be >= 1')
    order = np.lexsort((np.arange(len(work)), -work))  # largest first, then index
    heap = [(0.0, r) for r in range(world)]
    shards: list[list[int]] = [[] for _ in range(world)]
    for g in order:
        load, r = heapq.heappop(heap)
        shards[r].append(int(g))
        heapq.heappush(heap, (load + float(work[g]), r))
    return [np.array(sorted(s), dtype=np.int64) for s in shards]


def shard_loads(work, shards) -> np.ndarray:
    work = np.asarray(work, dtype=np.float64)
    return np.array([work[s].sum() for s in shards])


def gather_results(local_idx, local_values, num_graphs: int, dist=None) -> np.ndarray:
    """Per-graph values of every rank's shard in the original graph order.

    `local_idx` are this rank's graph indices and `local_values` one row per
    graph (any numeric columns).  With torch.distributed initialised the rows
    of all ranks are exchanged (all_gather_object over the host); without it
    this rank's rows are placed directly."""
    local_idx = np.asarray(local_idx, dtype=np.int64)
    local_values = np.asarray(local_values, dtype=np.float64)
    if local_values.ndim == 1:
        local_values = local_values[:, None]
    parts = [(local_idx, local_values)]
    if dist is not None and dist.is_initialized():
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, (local_idx, local_values))
    ncol = local_values.shape[1]
    out = np.full((num_graphs, ncol), np.nan)
    seen = np.zeros(num_graphs, dtype=bool)
    for idx, vals in parts:
        if np.any(seen[idx]):
            raise ValueError('a graph appears in two shards')
        seen[idx] = True
        out[idx] = vals
    if not seen.all():
        raise ValueError('some graphs are in no shard')
    return out
