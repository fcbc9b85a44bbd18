"""Edge cases of the path through the C ABI, each against the FP64 oracle:
empty point sets, all-NoData masks, points outside the raster, bandwidths
far below a cell and wider than the raster, duplicate points (in the
density and in the leave-one-out sum), zero weights, one-cell and ragged
rasters and tiles.

Tolerances are those of the parity tests: 1e-6 relative on every valid
cell and edge weight (cells with no in-cutoff pair must be exactly 0),
NoData passed through, pair counts equal.
"""
import numpy as np
import pytest

import oracle_py as o

torch = pytest.importorskip("torch")
import mgpukde_tiled_b200 as mk  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-6
NODATA = -9999.0


@pytest.fixture(scope="module")
def ctx():
    c = mk.Context(0)
    yield c
    c.close()


def rel_err(got, ref):
    got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    return np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)


def check_raster(ctx, x, y, w, h, dg, dmask, eg=None, emask=None, tile=0):
    x, y, w = (np.asarray(a, np.float32) for a in (x, y, w))
    if eg is not None:
        d2 = o.dist2_boundary(x, y, eg, o.mark_boundary(eg, emask))
        ew, eev = o.edge_weights(x, y, h, d2, eg, emask)
    else:
        ew, eev = np.ones(len(x)), 0
    ref, rev = o.density(x, y, w, ew, h, dg, dmask)
    den, gew, gev = mk.kde_raster(ctx, x, y, w, h, mk.Grid.of(dg), dmask, mk.Grid.of(eg) if eg is not None else None,
                                  emask, tile=tile, return_ew=True, count=True)
    valid = np.ones(den.shape, bool) if dmask is None else dmask != dg.nodata
    if dmask is not None:
        assert np.array_equal(den[~valid], dmask[~valid])
    assert np.array_equal(den[valid] == 0, ref[valid] == 0)
    if valid.any():
        assert rel_err(den[valid], ref[valid]).max() <= RTOL
    if len(x):
        assert rel_err(gew, ew).max() <= RTOL
    assert gev == rev + eev
    return den, ref


def polygon_mask(n, cut=0.3):
    yy, xx = np.mgrid[0:n, 0:n]
    m = np.where((xx - n / 2) ** 2 + (yy - n / 2) ** 2 < (n * (0.5 - cut / 2)) ** 2, 1.0, NODATA)
    return m.astype(np.float32)


def rand_points(n, lo, hi, seed):
    r = np.random.default_rng(seed)
    return r.uniform(lo, hi, n).astype(np.float32), r.uniform(lo, hi, n).astype(np.float32)


def test_empty_point_set(ctx):
    dg = o.grid(64, 64, 0.0, 0.0, 1.0, NODATA)
    eg = o.grid(32, 32, 0.0, 0.0, 2.0, NODATA)
    e = np.zeros(0, np.float32)
    den, _ = check_raster(ctx, e, e, e, 2.0, dg, polygon_mask(64), eg, polygon_mask(32))
    assert np.all(den[polygon_mask(64) != NODATA] == 0)


def test_all_nodata_density_mask(ctx):
    dg = o.grid(48, 40, 0.0, 0.0, 1.0, NODATA)
    x, y = rand_points(300, 0, 48, 1)
    den, _ = check_raster(ctx, x, y, np.ones_like(x), 3.0, dg, np.full((40, 48), NODATA, np.float32))
    assert np.all(den == NODATA)


def test_all_nodata_edge_mask(ctx):
    """No valid edge cell: no boundary, every distance is the reference's
    initial maximum and every edge weight short-circuits to 1."""
    dg = o.grid(40, 40, 0.0, 0.0, 1.0, NODATA)
    eg = o.grid(20, 20, 0.0, 0.0, 2.0, NODATA)
    x, y = rand_points(200, 0, 40, 2)
    _, _ = check_raster(ctx, x, y, np.ones_like(x), 2.5, dg, polygon_mask(40), eg,
                        np.full((20, 20), NODATA, np.float32))
    pts = mk.Points.upload(ctx, x, y)
    em = mk.Raster.upload(ctx, mk.Grid.of(eg), np.full((20, 20), NODATA, np.float32))
    mk.calc_dist2_boundary(ctx, pts, em)
    got, _ = pts.download(dist2=True, ew=False)
    ref = o.dist2_boundary(x, y, eg, o.mark_boundary(eg, np.full((20, 20), NODATA, np.float32)))
    assert np.array_equal(got, ref)


def test_points_outside_the_raster(ctx):
    """Points beyond every edge: far ones add nothing, those within 3h of the
    raster add their partial discs; edge weights of points off the mask."""
    dg = o.grid(50, 50, 100.0, 200.0, 1.0, NODATA)
    eg = o.grid(25, 25, 100.0, 200.0, 2.0, NODATA)
    r = np.random.default_rng(3)
    x = np.concatenate([r.uniform(100, 150, 200), [95.0, 152.0, 99.5, 150.5, -1e4, 1e5, 125.0, 125.0]])
    y = np.concatenate([r.uniform(200, 250, 200), [225.0, 230.0, 199.0, 251.0, 225.0, 225.0, 190.0, 260.0]])
    check_raster(ctx, x, y, np.ones_like(x), 2.0, dg, polygon_mask(50), eg, polygon_mask(25))


@pytest.mark.parametrize("h", [0.05, 0.4, 200.0])
def test_bandwidth_far_below_a_cell_and_above_the_raster(ctx, h):
    dg = o.grid(37, 29, 0.0, 0.0, 1.0, NODATA)
    x, y = rand_points(150, 0, 29, 4)
    check_raster(ctx, x, y, np.ones_like(x), h, dg, polygon_mask(37)[:29, :37])


def test_duplicate_points_and_zero_weights(ctx):
    dg = o.grid(40, 40, 0.0, 0.0, 1.0, NODATA)
    x, y = rand_points(100, 0, 40, 5)
    x = np.concatenate([x, np.full(50, 20.25, np.float32)])
    y = np.concatenate([y, np.full(50, 19.75, np.float32)])
    w = np.ones_like(x)
    w[::3] = 0.0
    check_raster(ctx, x, y, w, 1.5, dg, polygon_mask(40))


def test_duplicate_points_in_the_leave_one_out_sum(ctx):
    """Only the point itself is left out: its copies at the same place stay in."""
    eg = o.grid(30, 30, 0.0, 0.0, 2.0, NODATA)
    em = polygon_mask(30, 0.1)
    x, y = rand_points(400, 5, 55, 6)
    x = np.concatenate([x, np.full(20, 30.0, np.float32), np.full(3, 31.5, np.float32)])
    y = np.concatenate([y, np.full(20, 30.0, np.float32), np.full(3, 28.0, np.float32)])
    w = np.ones_like(x)
    d2 = o.dist2_boundary(x, y, eg, o.mark_boundary(eg, em))
    hgrid = np.array([0.7, 1.5, 4.0, 9.0], np.float32)
    refs = [o.loglik_at(x, y, w, d2, eg, em, float(h)) for h in hgrid]
    ref = np.array([r[0] for r in refs])
    pts = mk.Points.upload(ctx, x, y, w)
    r = mk.Raster.upload(ctx, mk.Grid.of(eg), em)
    mk.calc_dist2_boundary(ctx, pts, r)
    got, am = mk.log_likelihood_batch(ctx, pts, r, hgrid)
    assert np.all(np.abs(got - ref) <= 1e-6 * np.abs(ref) + 1e-6)
    assert am == int(np.argmax(ref))
    assert sum(ctx.last_loo_evals) == sum(rr[1] for rr in refs)


@pytest.mark.parametrize("shape,tile", [((1, 1), 0), ((3, 5), 2), ((70, 9), 4), ((9, 300), 7)])
def test_one_cell_and_ragged_rasters(ctx, shape, tile):
    nr, nc = shape
    dg = o.grid(nc, nr, 10.0, 10.0, 0.5, NODATA)
    r = np.random.default_rng(7)
    x = r.uniform(10, 10 + 0.5 * nc, 80).astype(np.float32)
    y = r.uniform(10, 10 + 0.5 * nr, 80).astype(np.float32)
    m = np.ones(shape, np.float32)
    m.flat[::4] = NODATA
    if m.size == 1:
        m[:] = 1.0
    check_raster(ctx, x, y, np.ones_like(x), 0.8, dg, m, tile=tile)


def test_single_point(ctx):
    dg = o.grid(21, 21, 0.0, 0.0, 1.0, NODATA)
    den, ref = check_raster(ctx, [10.3], [10.6], [2.0], 2.0, dg, None)
    assert den.max() > 0 and np.count_nonzero(den) == np.count_nonzero(ref)


@pytest.mark.parametrize("ncols,nrows", [(1005, 700), (13, 600), (257, 1100)])
def test_band_path_mask_as_bits(ctx, ncols, nrows):
    """Full-width bands (no tile side) send the NoData mask as bits, packed on
    host threads: ragged widths (row padding to 128 columns), a short last
    band, NoData runs and scattered NoData cells."""
    dg = o.grid(ncols, nrows, 0.0, 0.0, 1.0, NODATA)
    r = np.random.default_rng(ncols + nrows)
    x = r.uniform(0, ncols, 1500).astype(np.float32)
    y = r.uniform(0, nrows, 1500).astype(np.float32)
    m = np.ones((nrows, ncols), np.float32)
    m[r.random((nrows, ncols)) < 0.1] = NODATA
    m[nrows // 3: nrows // 3 + 70, : ncols // 2] = NODATA
    check_raster(ctx, x, y, r.lognormal(0, 0.5, len(x)), 6.0, dg, m, tile=0)


def test_band_path_nan_nodata(ctx):
    """A NaN NoData value marks no cell as NoData (x != NaN holds for every
    x), in the packed bits as in the float kernels."""
    dg = o.grid(300, 600, 0.0, 0.0, 1.0, float("nan"))
    r = np.random.default_rng(11)
    x = r.uniform(0, 300, 800).astype(np.float32)
    y = r.uniform(0, 600, 800).astype(np.float32)
    m = np.ones((600, 300), np.float32)
    m[::7, ::3] = np.nan
    den, ref = check_raster(ctx, x, y, np.ones_like(x), 5.0, dg, m, tile=0)
    assert np.isfinite(den).all()
