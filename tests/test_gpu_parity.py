"""Parity of the CUDA path (through the C ABI) with the FP64 oracle.

Tolerances (stated by the product's accuracy target): density and edge
weights within 1e-6 relative of the FP64 oracle on every valid cell / point;
NoData cells, boundary flags, boundary distances, the edge-weight short-circuit,
in-cutoff pair counts and bandwidth argmax exactly equal.
"""
import numpy as np
import pytest

import oracle_py as o
from golden_cases import CASES, load, oracle_run

torch = pytest.importorskip("torch")
import mgpukde_tiled_b200 as mk  # noqa: E402
from mgpukde_tiled_b200 import synth  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-6


@pytest.fixture(scope="module")
def ctx():
    c = mk.Context(0)
    yield c
    c.close()


def rel_err(got, ref):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    return np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)


def run_components(ctx, d, h, count=True, hs=None):
    """boundary -> distance -> edge weights -> index -> one-tile density through the C ABI.
    hs: per-point bandwidths (default: the case's own, if any)."""
    x, y, w = d["x"], d["y"], d["w"]
    hs = d["hs"] if hs is None else hs
    eg, dg = mk.Grid.of(d["eg"]), mk.Grid.of(d["dg"])
    pts = mk.Points.upload(ctx, x, y, w, hs)
    res = {}
    if int(d["edge"]):
        em = mk.Raster.upload(ctx, eg, d["edge_mask"])
        res["nb"] = mk.mark_boundary(ctx, em)
        res["boundary"] = em.boundary()
        mk.calc_dist2_boundary(ctx, pts, em)
        res["edge_evals"] = mk.edge_correction_weights(ctx, pts, em, h if hs is None else 0.0, count=True)
        res["dist2"], res["ew"] = pts.download(dist2=True, ew=True)
    else:
        mk.unit_edge_weights(ctx, pts)
        res["ew"] = pts.download(ew=True)[1]
    idx = mk.Index(ctx, pts, h if hs is None else 0.0)
    dmask = torch.from_numpy(np.ascontiguousarray(d["density_mask"], np.float32)).cuda()
    out = torch.empty((dg.nrows, dg.ncols), dtype=torch.float32, device="cuda")
    res["density_evals"] = mk.density_tile(ctx, idx, dg, 0, 0, dg.nrows, dg.ncols, dmask, out, count=count)
    res["density"] = out.cpu().numpy()
    out64 = torch.empty_like(out)
    mk.density_tile(ctx, idx, dg, 0, 0, dg.nrows, dg.ncols, dmask, out64, fp64=True)
    res["density_fp64"] = out64.cpu().numpy()
    return res


@pytest.mark.parametrize("case", CASES)
def test_golden_case_components(ctx, case):
    d = load(case)
    ref = oracle_run(d)
    r = run_components(ctx, d, ref["h"], hs=ref.get("hs"))  # h_option 2: the oracle's adaptive h
    nd = d["density_mask"] == d["dg"].nodata
    assert np.array_equal(r["density"][nd], d["density_mask"][nd])
    assert rel_err(r["density"][~nd], ref["density"][~nd]).max() <= RTOL
    # FP64 form: FP64 sums of float-stored w*e, rounded to float once
    assert rel_err(r["density_fp64"][~nd], ref["density"][~nd]).max() <= 3e-7
    assert r["density_evals"] == ref["density_evals"]
    if int(d["edge"]):
        assert np.array_equal(r["boundary"], ref["boundary"])
        assert np.array_equal(r["dist2"], ref["dist2"])
        assert np.array_equal(r["ew"] == 1.0, ref["ew"] == 1.0)
        assert rel_err(r["ew"], ref["ew"]).max() <= RTOL
        assert r["edge_evals"] == ref["edge_evals"]


@pytest.mark.parametrize("case", ["c1_crop_h50", "c3_crop_h30"])
def test_large_coordinates_fixed_h(ctx, case):
    """The fixed-h kernels (one bandwidth for all points) at coordinates of
    about 1e4 and 4e4 units, with points on and within 1e-5 h of the 3h
    cutoff of cell centres; the fixtures' per-point h are all that h, so the
    oracle's answer is the same."""
    d = load(case)
    ref = oracle_run(d)
    h = float(d["h_pp"][0])
    assert np.all(d["h_pp"] == np.float32(h))
    r = run_components(ctx, dict(d, hs=None), h)
    nd = d["density_mask"] == d["dg"].nodata
    assert np.array_equal(r["density"][nd], d["density_mask"][nd])
    assert rel_err(r["density"][~nd], ref["density"][~nd]).max() <= RTOL
    assert r["density_evals"] == ref["density_evals"]
    assert np.array_equal(r["dist2"], ref["dist2"])
    assert np.array_equal(r["ew"] == 1.0, ref["ew"] == 1.0)
    assert rel_err(r["ew"], ref["ew"]).max() <= RTOL
    assert r["edge_evals"] == ref["edge_evals"]


@pytest.mark.parametrize("case", ["uniform_c0", "poly_fixed", "poly_varh"])
def test_golden_case_end_to_end(ctx, case):
    """mgk_kde_raster from host buffers, tiled into odd tile sizes."""
    d = load(case)
    ref = oracle_run(d)
    eg, dg = mk.Grid.of(d["eg"]), mk.Grid.of(d["dg"])
    den, ew, ev = mk.kde_raster(ctx, d["x"], d["y"], d["w"], ref["h"], dg, d["density_mask"], eg,
                                d["edge_mask"], h_pp=d["hs"], tile=37, return_ew=True, count=True)
    nd = d["density_mask"] == dg.nodata
    assert np.array_equal(den[nd], d["density_mask"][nd])
    assert rel_err(den[~nd], ref["density"][~nd]).max() <= RTOL
    assert rel_err(ew, ref["ew"]).max() <= RTOL
    assert ev == ref["density_evals"] + ref["edge_evals"]


def test_deterministic(ctx):
    d = load("poly_varh")
    ref = oracle_run(d)
    a = run_components(ctx, d, ref["h"], count=False)
    b = run_components(ctx, d, ref["h"], count=False)
    assert np.array_equal(a["density"].view(np.uint32), b["density"].view(np.uint32))
    assert np.array_equal(a["ew"].view(np.uint32), b["ew"].view(np.uint32))


def test_single_large_crop(ctx):
    """1/10-scale single-large workload (1e4 points, 1000^2 raster, h = 50,
    polygon mask), full raster against the oracle."""
    c = synth.single_large(scale=0.1, seed=1)
    dg = synth.Grid(**{k: getattr(c["density_grid"], k) for k in ("ncols", "nrows", "xll", "yll", "cs", "nodata")})
    dmask = synth.rasterize_polygon(c["polygon"], dg)
    og_e, og_d = o.grid(*c["edge_grid"].astuple()), o.grid(*dg.astuple())
    b = o.mark_boundary(og_e, c["edge_mask"])
    d2 = o.dist2_boundary(c["x"], c["y"], og_e, b)
    ew, eev = o.edge_weights(c["x"], c["y"], c["h"], d2, og_e, c["edge_mask"])
    ref, rev = o.density(c["x"], c["y"], c["w"], ew, c["h"], og_d, dmask)
    # 512^2 tiles, then the default full-width bands (256 rows: 4 bands through the copy pipeline)
    for tile in (512, 0):
        den, gew, gev = mk.kde_raster(ctx, c["x"], c["y"], c["w"], c["h"], mk.Grid.of(dg), dmask,
                                      mk.Grid.of(c["edge_grid"]), c["edge_mask"], tile=tile, return_ew=True,
                                      count=True)
        nd = dmask == dg.nodata
        assert np.array_equal(den[nd], dmask[nd])
        assert rel_err(den[~nd], ref[~nd]).max() <= RTOL
        assert rel_err(gew, ew).max() <= RTOL
        assert gev == rev + eev


def test_raster_band_schedules_agree(ctx, monkeypatch):
    """The whole-raster path's full-width bands (a 1500^2 raster: six bands)
    give bitwise the same raster whether the bands alternate over two
    streams, each waiting for the previous band's last CTA to start, or run
    on one stream (the schedule taken without stream memory operations),
    with and without the pair count."""
    c = synth.single_large(scale=0.15, seed=3)
    dg = mk.Grid.of(c["density_grid"])
    dmask = synth.rasterize_polygon(c["polygon"], c["density_grid"])
    args = (ctx, c["x"], c["y"], c["w"], c["h"], dg, dmask, mk.Grid.of(c["edge_grid"]), c["edge_mask"])
    for count in (False, True):
        monkeypatch.delenv("MGK_RASTER_ONE_STREAM", raising=False)
        two, _, ev2 = mk.kde_raster(*args, count=count)
        monkeypatch.setenv("MGK_RASTER_ONE_STREAM", "1")
        one, _, ev1 = mk.kde_raster(*args, count=count)
        assert np.array_equal(two.view(np.uint32), one.view(np.uint32))
        assert ev1 == ev2
    monkeypatch.delenv("MGK_RASTER_ONE_STREAM", raising=False)


def test_boundary_distance_exact_large(ctx):
    """Binned candidate-list search vs the oracle's brute force, bit for bit,
    on a 1000 x 1000 polygon mask with points inside, near the boundary and
    outside the mask extent."""
    c = synth.single_large(scale=0.4, seed=5)
    x = np.concatenate([c["x"][:60000], np.array([-300.0, 4500.0, -50.0, 2000.0, 3999.0], np.float32)])
    y = np.concatenate([c["y"][:60000], np.array([2000.0, -10.0, -70.0, 4321.0, 0.5], np.float32)])
    og = o.grid(*c["edge_grid"].astuple())
    b = o.mark_boundary(og, c["edge_mask"])
    ref = o.dist2_boundary(x, y, og, b)
    pts = mk.Points.upload(ctx, x, y)
    em = mk.Raster.upload(ctx, mk.Grid.of(c["edge_grid"]), c["edge_mask"])
    mk.calc_dist2_boundary(ctx, pts, em)
    got, _ = pts.download(dist2=True, ew=False)
    assert np.array_equal(got, ref)


def test_loo_batch_matches_oracle(ctx):
    d = load("loo_h1")
    x, y, w = d["x"], d["y"], d["w"]
    eg = d["eg"]
    b = o.mark_boundary(eg, d["edge_mask"])
    d2 = o.dist2_boundary(x, y, eg, b)
    hgrid = synth.log_h_grid(2.0, 20.0, 16)
    refs = [o.loglik_at(x, y, w, d2, eg, d["edge_mask"], float(h)) for h in hgrid]
    ref = np.array([r[0] for r in refs])
    pts = mk.Points.upload(ctx, x, y, w)
    em = mk.Raster.upload(ctx, mk.Grid.of(eg), d["edge_mask"])
    mk.calc_dist2_boundary(ctx, pts, em)
    got, am = mk.log_likelihood_batch(ctx, pts, em, hgrid)
    assert np.all(np.abs(got - ref) <= 1e-6 * np.abs(ref) + 1e-6)
    assert am == int(np.argmax(ref))
    assert sum(ctx.last_loo_evals) == sum(r[1] for r in refs)
    again, _ = mk.log_likelihood_batch(ctx, pts, em, hgrid)
    assert np.array_equal(got.view(np.uint64), again.view(np.uint64))
    hopt, it = mk.mle_fixed_bandwidth(ctx, pts, em, o.rule_of_thumb(x, y, w))
    assert abs(hopt - float(d["ref_hopt"])) <= 5e-6 * hopt + 5e-6


def test_errors_leave_device_usable(ctx):
    p = mk.Points.upload(ctx, np.zeros(3, np.float32), np.zeros(3, np.float32))
    with pytest.raises(mk.MgkError) as e:
        mk.Index(ctx, p, -1.0)  # no per-point bandwidths
    assert e.value.status == -1
    p.close()
    small = mk.Context(0, hbm_budget=1 << 20)
    with pytest.raises(mk.MgkError) as e:
        mk.Points.upload(small, np.zeros(1 << 20, np.float32), np.zeros(1 << 20, np.float32))
    assert e.value.status == -3
    small.close()
    # the device still works
    d = load("uniform_h0_noedge")
    ref = oracle_run(d)
    r = run_components(ctx, d, ref["h"], hs=ref.get("hs"))  # h_option 2: the oracle's adaptive h
    nd = d["density_mask"] == d["dg"].nodata
    assert rel_err(r["density"][~nd], ref["density"][~nd]).max() <= RTOL


def test_bandwidth_select_grid_matches_oracle(ctx):
    """1/10-scale batched bandwidth selection (2,000 mixture points in 500^2,
    polygon edge mask at cell 4, 16 log-spaced h in [5, 500]): logL per h,
    the argmax and the edge + pair eval counts against the oracle."""
    c = synth.bandwidth_select(scale=0.1, seed=2, nh=16)
    x, y, w = c["x"], c["y"], c["w"]
    eg = o.grid(*c["edge_grid"].astuple())
    b = o.mark_boundary(eg, c["edge_mask"])
    d2 = o.dist2_boundary(x, y, eg, b)
    refs = [o.loglik_at(x, y, w, d2, eg, c["edge_mask"], float(h)) for h in c["hgrid"]]
    ref = np.array([r[0] for r in refs])
    pts = mk.Points.upload(ctx, x, y, w)
    em = mk.Raster.upload(ctx, mk.Grid.of(c["edge_grid"]), c["edge_mask"])
    mk.calc_dist2_boundary(ctx, pts, em)
    got, am = mk.log_likelihood_batch(ctx, pts, em, c["hgrid"])
    assert np.all(np.abs(got - ref) <= 1e-6 * np.abs(ref) + 1e-6)
    assert am == int(np.argmax(ref))
    assert sum(ctx.last_loo_evals) == sum(r[1] for r in refs)


def test_loo_without_edge_correction(ctx):
    d = load("loo_h1")
    x, y, w = d["x"], d["y"], d["w"]
    hgrid = synth.log_h_grid(2.0, 20.0, 8)
    ref = np.array([o.loo_loglik(x, y, w, None, float(h))[0] for h in hgrid])
    pts = mk.Points.upload(ctx, x, y, w)
    got, am = mk.log_likelihood_batch(ctx, pts, None, hgrid)
    assert np.all(np.abs(got - ref) <= 1e-6 * np.abs(ref) + 1e-6)
    assert am == int(np.argmax(ref))
