"""Splitting ONE batch of independent SPD matrices across GPUs (one process per GPU).

The matrices of a batch share nothing, so the batch shards with no data-path collective:
every rank factors its own subset as one block-diagonal batch (its own persistent launches
and graph), and only the per-matrix results travel, on the host, after the work.  The
subsets balance the factorization work: each matrix costs its flop count fl = sum_j c_j^2
over the column counts of its factor (the reference's flop measure,
cholesky/ColumnCount.h:492-498, here from the library's own symbolic analysis of the
ordered matrix), and the matrices go, largest first, to the rank with the least work so far
(longest-processing-time list scheduling: the busiest rank carries at most 4/3 of the
optimum).  Ties go to the lower rank, so every rank computes the same split by itself.
"""
from __future__ import annotations

import heapq

import numpy as np

__all__ = ["matrix_flops", "split_by_cost", "gather_results"]


def matrix_flops(mat) -> float:
    """fl = sum_j c_j^2 of an ordered matrix (lower CSC of P A P^T with n, indptr, indices),
    from the library's supernode partition with the reference's relaxation (explicit zeros of
    relaxed supernodes counted: the work the factorization executes)."""
    from . import layout, supernodes
    sup = supernodes(mat.n, mat.indptr, mat.indices)
    lip = layout(mat.n, mat.indptr, mat.indices, sup)["Li_ptr"].astype(np.int64)
    f = sup[:-1].astype(np.int64)
    w = np.diff(sup).astype(np.int64)
    m = lip[sup[1:]] - lip[f]
    # sum_{k < w} (m - k)^2 per supernode, in closed form
    k1 = w * (w - 1) // 2
    k2 = (w - 1) * w * (2 * w - 1) // 6
    return float(np.sum(w * m * m - 2 * m * k1 + k2))


def split_by_cost(costs, world: int) -> list[np.ndarray]:
    """Indices of the matrices of each rank (sorted), balanced by cost."""
    costs = np.asarray(costs, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(costs.size), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def gather_results(local_idx, local_values, count: int, world: int):
    """Per-matrix results of every rank, in the batch's order (on every rank): one host
    all-gather of (indices, values) through torch.distributed (any backend; nothing when
    world is 1).  local_values is a 1-D array aligned with local_idx."""
    local_idx = np.asarray(local_idx, dtype=np.int64)
    local_values = np.asarray(local_values, dtype=np.float64)
    if world == 1:
        pieces = [(local_idx, local_values)]
    else:
        import torch.distributed as dist
        pieces = [None] * world
        dist.all_gather_object(pieces, (local_idx, local_values))
    out = np.full(count, np.nan)
    seen = np.zeros(count, dtype=bool)
    for idx, vals in pieces:
        if np.any(seen[idx]):
            raise RuntimeError("a matrix was assigned to two ranks")
        seen[idx] = True
        out[idx] = vals
    if not seen.all():
        raise RuntimeError("a matrix was assigned to no rank")
    return out
