"""Multi-GPU decomposition of the path (one process per GPU).

Density rows are independent given the points within 3h (the reference's
tile loop, kde_cuda_kdtr_tiled.cu:1146-1517, computes each tile from its halo
points only), so one study's raster is split into contiguous row ranges of
balanced work, one per rank (split_rows, row_costs), and each rank runs
mgk_kde_raster_rows on its range: no collective touches the density data.
The reference instead split points across GPUs and summed full tile copies
through host memory (ReformGPUAsciiRaster, :2468-2567).

The LOO bandwidth search has two exchanges (loo_loglik_shared): the edge
weights of every point at every h are computed by point share and
all-gathered (nh x n floats), then each rank sums log max(loo_j, eps) over
its share of the queries for every candidate h, and one all-reduce of the nh
partial sums (FP64) gives every rank the totals and the same argmax.  Only
NCCL (or gloo) collectives move data between ranks.
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


BLOCK_ROWS = 64  # cell rows of one density block: row ranges start on block rows


def row_costs(x, y, h, grid, mask=None):
    """Work estimate per band of BLOCK_ROWS rows: valid cells of the band times
    the points within 3h of its cell centres (the band's candidate pairs)."""
    nb = (grid.nrows + BLOCK_ROWS - 1) // BLOCK_ROWS
    reach = 3.0 * float(h)
    ys = np.sort(np.asarray(y, np.float64))
    cost = np.zeros(nb)
    for b in range(nb):
        r0, r1 = b * BLOCK_ROWS, min(grid.nrows, (b + 1) * BLOCK_ROWS)
        y_top = float(grid.yll) + (grid.nrows - 0.5 - r0) * float(grid.cs)
        y_bot = float(grid.yll) + (grid.nrows - 0.5 - (r1 - 1)) * float(grid.cs)
        npts = np.searchsorted(ys, y_top + reach, "right") - np.searchsorted(ys, y_bot - reach, "left")
        cells = (r1 - r0) * grid.ncols if mask is None else int(np.count_nonzero(mask[r0:r1] != grid.nodata))
        cost[b] = float(cells) * float(npts)
    return cost


def split_rows(nrows: int, world: int, costs=None):
    """Contiguous row ranges [(row0, nrows_r)] of balanced cost, one per rank,
    each starting on a block row.  costs: per band of BLOCK_ROWS rows
    (row_costs); default: equal.  A range may be empty when ranks outnumber
    the bands."""
    nb = (nrows + BLOCK_ROWS - 1) // BLOCK_ROWS
    c = np.ones(nb) if costs is None else np.asarray(costs, np.float64)
    cum = np.concatenate([[0.0], np.cumsum(c)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, world):
        # the band boundary whose prefix is nearest r / world of the total
        t = total * r / world
        b = int(np.searchsorted(cum, t, "left"))
        if b > 0 and (b > nb or t - cum[b - 1] < cum[b] - t):
            b -= 1
        cuts.append(min(max(b, cuts[-1]), nb))
    cuts.append(nb)
    out = []
    for r in range(world):
        a, b = cuts[r] * BLOCK_ROWS, min(nrows, cuts[r + 1] * BLOCK_ROWS)
        out.append((a, max(0, b - a)))
    return out


def share_chunk(n: int, world: int) -> int:
    """Points per rank in the edge-weight exchange (the last rank's share may
    be shorter; every chunk has this many slots)."""
    return (n + world - 1) // world


def gather_edge_chunks(ew_all, rank: int, group=None):
    """All-gathers the edge-weight chunks in place: ew_all is a
    (world, nh, chunk) float32 tensor of which this rank filled ew_all[rank]."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return ew_all
    mine = ew_all[rank].clone()
    dist.all_gather(list(ew_all.unbind(0)), mine, group=group)
    return ew_all


def loo_loglik_shared(ctx, points, raster, hgrid, rank: int, world: int, group=None):
    """Batched LogLikelihood of one study split over `world` ranks (this is
    rank `rank`): edge weights by point share + all-gather, partial sums over
    this rank's query share + all-reduce.  Returns (logL[nh], argmax,
    this rank's (edge evals, pair evals))."""
    import torch

    from . import kde

    hs = np.ascontiguousarray(hgrid, np.float32)
    ew_all = None
    ev_e = 0
    if raster is not None:
        c = share_chunk(points.n, world)
        ew_all = torch.empty((world, len(hs), c), dtype=torch.float32, device="cuda")
        ev_e = kde.loo_share_edge_weights(ctx, points, raster, hs, rank, world, ew_all, count=True)
        ctx.synchronize()  # the chunk is read by the collective on torch's stream
        gather_edge_chunks(ew_all, rank, group)
        torch.cuda.current_stream().synchronize()
    part, ev_p = kde.loo_share_loglik(ctx, points, hs, rank, world, ew_all)
    tot, am = allreduce_loglik(part, group)
    return tot, am, (ev_e, ev_p)
