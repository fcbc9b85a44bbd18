"""Multi-GPU decomposition of the path (one process per GPU).

Density tiles are independent given the points within 3h (the reference's
tile loop, kde_cuda_kdtr_tiled.cu:1146-1517, computes each tile from its halo
points only), so tiles are partitioned across ranks and no collective touches
the density data.  The reference instead split points across GPUs and summed
full tile copies through host memory (ReformGPUAsciiRaster, :2468-2567).

The LOO bandwidth search has one real exchange: each rank sums
log max(loo_j, eps) over its range of query points for every candidate h, and
one all-reduce of the nh partial sums (FP64) gives every rank the totals and
the same argmax.
"""
from __future__ import annotations

import heapq

import numpy as np


def tile_plan(nrows: int, ncols: int, tile: int):
    """Row-major tiles (row0, col0, nr, nc) covering the raster, as the
    reference walks them (:1497-1512)."""
    out = []
    for r0 in range(0, nrows, tile):
        for c0 in range(0, ncols, tile):
            out.append((r0, c0, min(tile, nrows - r0), min(tile, ncols - c0)))
    return out


def assign_tiles(tiles, world: int, costs=None):
    """Deterministic longest-processing-time assignment of tiles to ranks.
    costs: per-tile work estimate (e.g. candidate points x cells); default
    is the cell count.  Returns a list of tile-index lists, one per rank."""
    if costs is None:
        costs = [nr * nc for (_, _, nr, nc) in tiles]
    order = sorted(range(len(tiles)), key=lambda i: (-costs[i], i))
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def query_range(n: int, rank: int, world: int):
    """Contiguous share of the query points for the LOO sum."""
    per = (n + world - 1) // world
    a = min(n, rank * per)
    return a, min(n, a + per)


def allreduce_loglik(partial, group=None):
    """Sums per-rank FP64 partial log likelihoods over ranks (one all-reduce of
    nh doubles); returns (totals, argmax)."""
    import torch
    import torch.distributed as dist

    t = torch.as_tensor(np.asarray(partial, np.float64))
    if dist.is_available() and dist.is_initialized():
        dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        t = t.to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    tot = t.cpu().numpy()
    return tot, int(np.argmax(tot))
