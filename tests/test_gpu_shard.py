"""The multi-GPU split of one study, on one GPU: the ranks' calls run one
after another on one context (no rank waits on another), and the host stands
in for the collectives (every rank's edge-weight chunk lands in one shared
buffer, which is what the all-gather produces; the partial log likelihoods
are summed).  Checked through the C ABI:

* mgk_points_select keeps exactly the points inside the rectangle, in input
  order;
* mgk_kde_raster_rows over the ranks' row ranges, stitched, equals
  mgk_kde_raster's raster (1e-6 relative) and the FP64 oracle's, and the
  ranks' density pair counts add up to the whole raster's;
* mgk_loo_share_edge_weights + mgk_loo_share_loglik over the parts give the
  logL of mgk_loo_loglik_batch (1e-12 relative; the FP64 sums are grouped
  differently), the same argmax, and the same pair counts in total.
"""
import numpy as np
import pytest

import oracle_py as o

torch = pytest.importorskip("torch")
import mgpukde_tiled_b200 as mk  # noqa: E402
from mgpukde_tiled_b200 import shard, synth  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mk.Context(0)
    yield c
    c.close()


def test_points_select_matches_host_filter(ctx):
    c = synth.single_large(scale=0.1, seed=3)
    x, y, w = c["x"], c["y"], c["w"]
    pts = mk.Points.upload(ctx, x, y, w)
    box = (200.0, 650.5, 300.25, 310.0)
    sel = pts.select(*box)
    keep = ((x.astype(np.float64) >= box[0]) & (x.astype(np.float64) <= box[1]) &
            (y.astype(np.float64) >= box[2]) & (y.astype(np.float64) <= box[3]))
    assert sel.n == int(keep.sum()) > 0
    from cuda.bindings import runtime as rt

    arr = sel.device_arrays()
    ctx.synchronize()
    got = {}
    for k in ("x", "y", "w"):
        a = np.empty(sel.n, np.float32)
        err, = rt.cudaMemcpy(a.ctypes.data, arr[k], 4 * sel.n, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert err == rt.cudaError_t.cudaSuccess
        got[k] = a
    assert np.array_equal(got["x"], x[keep]) and np.array_equal(got["y"], y[keep])
    assert np.array_equal(got["w"], w[keep])
    empty = pts.select(-5.0, -4.0, -5.0, -4.0)
    assert empty.n == 0
    for p in (empty, sel, pts):
        p.close()


def test_row_split_of_one_study_equals_the_whole(ctx):
    c = synth.single_large(scale=0.1, seed=5)
    dg, eg = mk.Grid.of(c["density_grid"]), mk.Grid.of(c["edge_grid"])
    mask = synth.rasterize_polygon(c["polygon"], c["density_grid"])
    x, y, w, h = c["x"], c["y"], c["w"], float(c["h"])
    whole, _, ev_whole = mk.kde_raster(ctx, x, y, w, h, dg, mask, eg, c["edge_mask"], count=True)
    rows = shard.split_rows(dg.nrows, 3, shard.row_costs(x, y, h, c["density_grid"], mask))
    stitched = np.full((dg.nrows, dg.ncols), np.nan, np.float32)
    for r0, nr in rows:
        if nr:
            stitched[r0:r0 + nr], _ = mk.kde_raster_rows(ctx, x, y, w, h, dg, r0, nr, mask[r0:r0 + nr], eg,
                                                         c["edge_mask"], count=True)
    valid = mask != dg.nodata
    assert np.array_equal(stitched[~valid], mask[~valid])
    rel = np.abs(stitched[valid].astype(np.float64) - whole[valid]) / np.abs(whole[valid].astype(np.float64))
    assert rel.max() <= 1e-6
    # against the FP64 oracle of the whole study
    og = o.grid(*c["edge_grid"].astuple())
    d2 = o.dist2_boundary(x, y, og, o.mark_boundary(og, c["edge_mask"]))
    ew, _ = o.edge_weights(x, y, h, d2, og, c["edge_mask"])
    ref, ev_den = o.density(x, y, w, ew, h, o.grid(*c["density_grid"].astuple()), mask)
    rel_o = np.abs(stitched[valid] - ref[valid]) / np.abs(ref[valid])
    assert rel_o.max() <= 1e-6
    # each rank's density pairs: the count of its rows (edge pairs of halo points repeat across ranks)
    pts = mk.Points.upload(ctx, x, y, w)
    em = mk.Raster.upload(ctx, eg, c["edge_mask"])
    mk.mark_boundary(ctx, em)
    mk.calc_dist2_boundary(ctx, pts, em)
    mk.edge_correction_weights(ctx, pts, em, h)
    idx = mk.Index(ctx, pts, h)
    dm = torch.from_numpy(mask).cuda()
    tot = 0
    for r0, nr in rows:
        if nr:
            out = torch.empty((nr, dg.ncols), dtype=torch.float32, device="cuda")
            tot += mk.density_tile(ctx, idx, dg, r0, 0, nr, dg.ncols, dm[r0:r0 + nr], out, count=True)
    assert tot == ev_den
    idx.close()
    em.close()
    pts.close()


def test_loo_shares_sum_to_the_batch(ctx):
    c = synth.bandwidth_select(scale=0.15, seed=2, nh=12)
    eg = mk.Grid.of(c["edge_grid"])
    pts = mk.Points.upload(ctx, c["x"], c["y"], c["w"])
    em = mk.Raster.upload(ctx, eg, c["edge_mask"])
    mk.mark_boundary(ctx, em)
    mk.calc_dist2_boundary(ctx, pts, em)
    hs = c["hgrid"]
    ref, best = mk.log_likelihood_batch(ctx, pts, em, hs)
    ev_edge_ref, ev_loo_ref = ctx.last_loo_evals
    world = 3
    ch = shard.share_chunk(pts.n, world)
    ew_all = torch.full((world, len(hs), ch), float("nan"), dtype=torch.float32, device="cuda")
    ev_e = sum(mk.loo_share_edge_weights(ctx, pts, em, hs, r, world, ew_all, count=True) for r in range(world))
    ctx.synchronize()
    parts = [mk.loo_share_loglik(ctx, pts, hs, r, world, ew_all) for r in range(world)]
    tot = np.sum([p for p, _ in parts], axis=0)
    assert np.all(np.abs(tot - ref) <= 1e-12 * np.abs(ref))
    assert int(np.argmax(tot)) == best
    assert ev_e == ev_edge_ref and sum(e for _, e in parts) == ev_loo_ref
    # without edge correction the shares need no exchange
    ref0, _ = mk.log_likelihood_batch(ctx, pts, None, hs)
    tot0 = np.sum([mk.loo_share_loglik(ctx, pts, hs, r, 2)[0] for r in range(2)], axis=0)
    assert np.all(np.abs(tot0 - ref0) <= 1e-12 * np.abs(ref0))
    em.close()
    pts.close()
