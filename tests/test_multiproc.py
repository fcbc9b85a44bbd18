"""Multi-rank host logic on CPU (gloo, world size 2): the tile partition
covers every tile once with balanced work, and the one exchange of the LOO
search (an all-reduce of per-rank partial log likelihoods) reproduces the
single-process oracle sum and argmax."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mgpukde_tiled_b200 import shard


def test_tile_plan_and_assignment():
    tiles = shard.tile_plan(10_000, 10_000, 4096)
    assert len(tiles) == 9
    assert sum(nr * nc for (_, _, nr, nc) in tiles) == 10_000 * 10_000
    parts = shard.assign_tiles(tiles, 4)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(tiles)))
    assert shard.assign_tiles(tiles, 4) == parts  # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    import torch.distributed as dist

    import oracle_py as o
    from mgpukde_tiled_b200 import shard as sh
    from mgpukde_tiled_b200 import synth
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    x, y = synth.mixture_points(800, 3, 100.0, 4.0, 10.0, seed=5)
    hs = synth.log_h_grid(1.0, 10.0, 6)
    a, b = sh.query_range(len(x), rank, world)
    part = []
    for h in hs:
        _, loo, _ = o.loo_loglik(x, y, None, None, float(h))
        v = np.maximum(loo[a:b], float(np.float32(1e-14)))
        part.append(float(np.sum(np.log(v))))
    tot, am = sh.allreduce_loglik(part)
    # tile assignment is the same on every rank
    parts = sh.assign_tiles(sh.tile_plan(300, 500, 128), world)
    q.put((rank, tot.tolist(), am, parts))
    dist.destroy_process_group()


def test_two_rank_loo_allreduce():
    import oracle_py as o
    from mgpukde_tiled_b200 import synth
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    x, y = synth.mixture_points(800, 3, 100.0, 4.0, 10.0, seed=5)
    hs = synth.log_h_grid(1.0, 10.0, 6)
    ref = np.array([o.loo_loglik(x, y, None, None, float(h))[0] for h in hs])
    (r0, t0, a0, p0), (r1, t1, a1, p1) = sorted(res)
    np.testing.assert_allclose(t0, ref, rtol=1e-12)
    assert t0 == t1 and a0 == a1 == int(np.argmax(ref))
    assert p0 == p1


def _shared_worker(rank, world, port, q):
    """One rank of the split bandwidth selection and of the row split, with
    the FP64 oracle standing in for the device kernels: edge weights of this
    rank's point share into its chunk, the all-gather of the chunks, the
    partial leave-one-out sums of its query share, the all-reduce."""
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    import torch
    import torch.distributed as dist

    import oracle_py as o
    from mgpukde_tiled_b200 import shard as sh
    from mgpukde_tiled_b200 import synth
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    c = synth.bandwidth_select(scale=0.04, seed=2, nh=5)
    x, y, w = c["x"], c["y"], c["w"]
    n, hs = len(x), c["hgrid"]
    eg, em = o.grid(*c["edge_grid"].astuple()), c["edge_mask"]
    d2 = o.dist2_boundary(x, y, eg, o.mark_boundary(eg, em))
    ch = sh.share_chunk(n, world)
    p0, p1 = min(n, rank * ch), min(n, (rank + 1) * ch)
    ew_all = torch.zeros((world, len(hs), ch), dtype=torch.float32)
    for k, h in enumerate(hs):
        e, _ = o.edge_weights(x[p0:p1], y[p0:p1], float(h), d2[p0:p1], eg, em)
        ew_all[rank, k, :p1 - p0] = torch.from_numpy(e.astype(np.float32))
    sh.gather_edge_chunks(ew_all, rank)
    # chunk layout: e of point r * ch + j at h_k is ew_all[r, k, j]
    ew = ew_all.permute(1, 0, 2).reshape(len(hs), world * ch)[:, :n].numpy()
    a, b = sh.query_range(n, rank, world)
    part = []
    for k, h in enumerate(hs):
        _, loo, _ = o.loo_loglik(x, y, w, ew[k].astype(np.float64), float(h))
        part.append(float(np.sum(np.log(np.maximum(loo[a:b], float(np.float32(1e-14)))))))
    tot, am = sh.allreduce_loglik(part)
    # the row split of a density raster: every rank computes the same ranges
    d = synth.single_large(scale=0.05, seed=1)
    dg = d["density_grid"]
    mask = synth.rasterize_polygon(d["polygon"], dg)
    rows = sh.split_rows(dg.nrows, world, sh.row_costs(d["x"], d["y"], d["h"], dg, mask))
    q.put((rank, tot.tolist(), am, rows, ew_all.numpy().tolist()))
    dist.destroy_process_group()


def test_two_rank_shared_bandwidth_selection():
    """The split bandwidth selection of two gloo ranks (edge-weight chunks
    all-gathered, partial sums all-reduced) gives every rank the edge weights
    of all points and the single-process logL and argmax."""
    import oracle_py as o
    from mgpukde_tiled_b200 import shard as sh
    from mgpukde_tiled_b200 import synth
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shared_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    c = synth.bandwidth_select(scale=0.04, seed=2, nh=5)
    x, y, w = c["x"], c["y"], c["w"]
    eg, em = o.grid(*c["edge_grid"].astuple()), c["edge_mask"]
    d2 = o.dist2_boundary(x, y, eg, o.mark_boundary(eg, em))
    ref = np.array([o.loglik_at(x, y, w, d2, eg, em, float(h))[0] for h in c["hgrid"]])
    (_, t0, a0, rows0, ew0), (_, t1, a1, rows1, ew1) = res
    # both ranks hold the same gathered edge weights, the ones of every point
    assert ew0 == ew1
    ch = sh.share_chunk(len(x), 2)
    e_all = np.asarray(ew0, np.float32).transpose(1, 0, 2).reshape(len(c["hgrid"]), 2 * ch)[:, :len(x)]
    for k, h in enumerate(c["hgrid"]):
        e, _ = o.edge_weights(x, y, float(h), d2, eg, em)
        assert np.array_equal(e_all[k], e.astype(np.float32))
    # ew through float32 (as on the device): logL within 1e-7 relative
    np.testing.assert_allclose(t0, ref, rtol=1e-7)
    assert t0 == t1 and a0 == a1 == int(np.argmax(ref))
    # the row ranges are the same on both ranks and tile the raster
    assert rows0 == rows1
    assert rows0[0][0] == 0 and all(a + n == b for (a, n), (b, _) in zip(rows0, rows0[1:]))
    assert sum(n for _, n in rows0) == synth.single_large(scale=0.05, seed=1)["density_grid"].nrows


def test_row_halo_selection_keeps_every_contributing_point():
    """The densities of a range of rows from the points within 3h of those
    rows (the selection mgk_kde_raster_rows makes on the device) equal the
    rows of the whole-raster density."""
    import oracle_py as o
    from mgpukde_tiled_b200 import shard as sh
    from mgpukde_tiled_b200 import synth
    d = synth.single_large(scale=0.03, seed=4)
    dg = d["density_grid"]
    mask = synth.rasterize_polygon(d["polygon"], dg)
    x, y, w, h = d["x"], d["y"], d["w"], d["h"]
    full, ev_full = o.density(x, y, w, None, h, o.grid(*dg.astuple()), mask)
    ev_sum = 0
    for r0, nr in sh.split_rows(dg.nrows, 3):
        if nr == 0:
            continue
        y_top = float(np.float32(float(dg.yll) + (dg.nrows - 0.5 - r0) * float(dg.cs)))
        y_bot = float(np.float32(float(dg.yll) + (dg.nrows - 0.5 - (r0 + nr - 1)) * float(dg.cs)))
        reach = 3.0 * h * (1.0 + 1e-6) + 1e-6 * float(dg.cs)
        keep = (y.astype(np.float64) >= y_bot - reach) & (y.astype(np.float64) <= y_top + reach)
        part, ev = o.density(x[keep], y[keep], w[keep], None, h, o.grid(*dg.astuple()), mask,
                             window=(r0, 0, nr, dg.ncols))
        np.testing.assert_allclose(part, full[r0:r0 + nr], rtol=1e-13, atol=0)
        ev_sum += ev
    assert ev_sum == ev_full
