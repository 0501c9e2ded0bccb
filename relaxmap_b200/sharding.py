"""Batched mode across GPUs: graphs are independent, so a batch shards by
graph with no collective inside the optimiser. One process per GPU; every
rank optimises its share, then the per-graph results are combined.

lpt_assign   longest-processing-time assignment of graphs to ranks by their
             (estimated) link counts: heaviest first, each to the least-loaded
             rank (ties to the lowest rank), so the slowest rank's load is
             within 4/3 of the optimum.
combine      the per-graph values of all ranks on every rank: each rank writes
             its graphs' entries of a dense vector, one SUM all_reduce.
"""
from __future__ import annotations

import heapq

import numpy as np


def lpt_assign(weights, world: int) -> list:
    """Graph indices per rank (ascending within a rank)."""
    w = np.asarray(weights, dtype=np.float64)
    order = np.argsort(-w, kind="stable")
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for g in order.tolist():
        load, r = heapq.heappop(heap)
        out[r].append(g)
        heapq.heappush(heap, (load + float(w[g]), r))
    return [np.array(sorted(o), dtype=np.int64) for o in out]


def combine(n_graphs: int, mine, values, pg, device) -> np.ndarray:
    """Dense per-graph vector from every rank's (indices, values)."""
    import torch
    v = torch.zeros(n_graphs, dtype=torch.float64, device=device)
    if len(mine):
        v[torch.as_tensor(np.asarray(mine), device=device)] = torch.as_tensor(np.asarray(values, dtype=np.float64),
                                                                               device=device)
    if pg is not None:
        pg.all_reduce(v, op=pg.ReduceOp.SUM)
    return v.cpu().numpy()
