"""Adaptive bandwidths (h_option 2) through the C ABI against the FP64 oracle.

The likelihood LogLikelihood(h, alpha) of kde_cuda_kdtr_tiled.cu:3553-3650
(pilot density with itself, geometric-mean bandwidths, edge weights at the
per-point h, leave-one-out density with each source point's h) and the
Hooke-Jeeves search of hooke_jeeves / hj_likelihood (:3677-3785).

Tolerances: logL within 1e-8 relative of the oracle (FP32 pair sums with
Kahan compensation and an unbiased exp2, FP64 logarithms); the search visits
the same (h, alpha) points, so its optimum and iteration count are equal;
per-point bandwidths within 4e-7 relative (a float ulp, from the FP32 pilot
densities); the density raster at those bandwidths within 3e-6 relative
(K_h moves up to 7x the relative change of h).
"""
import numpy as np
import pytest

import oracle_py as o
from golden_cases import load

torch = pytest.importorskip("torch")
import mgpukde_tiled_b200 as mk  # noqa: E402
from mgpukde_tiled_b200 import synth  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mk.Context(0)
    yield c
    c.close()


def rel(got, ref):
    got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    return np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)


def setup(ctx, d):
    pts = mk.Points.upload(ctx, d["x"], d["y"], d["w"])
    em, d2 = None, None
    if int(d["edge"]):
        em = mk.Raster.upload(ctx, mk.Grid.of(d["eg"]), d["edge_mask"])
        mk.mark_boundary(ctx, em)
        mk.calc_dist2_boundary(ctx, pts, em)
        d2 = pts.download(dist2=True, ew=False)[0]
    return pts, em, d2


def mixture_case(n=20000, seed=3):
    """Seeded clustered points in a 2,000 x 2,000 square with a disc-shaped
    edge mask at cell 10 (200 x 200)."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(300, 1700, (12, 2))
    k = rng.integers(0, 12, n)
    xy = c[k] + rng.normal(0, 120, (n, 2))
    xy = np.clip(xy, 1, 1999).astype(np.float32)
    eg = o.grid(200, 200, 0.0, 0.0, 10.0, -9999.0)
    yy, xx = np.mgrid[0:200, 0:200]
    cx, cy = (xx + 0.5) * 10, 2000 - (yy + 0.5) * 10
    em = np.where((cx - 1000) ** 2 + (cy - 1000) ** 2 < 980 ** 2, 1.0, -9999.0).astype(np.float32)
    dg = o.grid(100, 100, 0.0, 0.0, 20.0, -9999.0)
    return dict(x=xy[:, 0].copy(), y=xy[:, 1].copy(), w=rng.uniform(0.5, 2, n).astype(np.float32), edge=1,
                eg=eg, edge_mask=em, dg=dg, density_mask=np.ones((100, 100), np.float32))


@pytest.mark.parametrize("case", ["redwood_h2", "poly_h2", "uniform_h0_noedge", "mixture_20k"])
def test_loglik_adaptive_matches_oracle(ctx, case):
    d = mixture_case() if case == "mixture_20k" else load(case)
    x, y, w = d["x"], d["y"], d["w"]
    h0 = o.rule_of_thumb(x, y, w)
    pts, em, d2 = setup(ctx, d)
    mask = d["edge_mask"] if int(d["edge"]) else None
    eg = d["eg"] if mask is not None else None
    for h, a in ((h0, -0.5), (0.7 * h0, -0.2), (1.4 * h0, -0.8)):
        ref, _ = o.loglik_adaptive(x, y, w, d2, eg, mask, h, a)
        got = mk.loglik_adaptive(ctx, pts, em, h, a)
        assert abs(got - ref) <= 1e-8 * abs(ref), (h, a, got, ref)
        # eval counts of the same steps in the oracle: edge-mask cells at h and
        # at hs, pilot pairs (self included) and leave-one-out pairs
        if mask is not None:
            ew1, e1 = o.edge_weights(x, y, h, d2, eg, mask)
        else:
            ew1, e1 = np.ones(len(x)), 0
        den0, p0 = o.point_density(x, y, w, ew1, h, self_term=True)
        hs = o.adaptive_bandwidths(den0, h, a)
        if mask is not None:
            ew2, e2 = o.edge_weights(x, y, 0.0, d2, eg, mask, hs=hs)
        else:
            ew2, e2 = np.ones(len(x)), 0
        _, p1 = o.point_density(x, y, w, ew2, 0.0, hs=hs, self_term=False)
        edge_ev, pair_ev = ctx.last_loo_evals
        # the device's hs may differ from the oracle's by one float ulp, which
        # can move a pair or a cell lying exactly at a cutoff
        assert abs(edge_ev - (e1 + e2)) <= 1e-6 * (e1 + e2)
        assert abs(pair_ev - (p0 + p1)) <= 1e-6 * (p0 + p1)
        assert ctx.last_loo_ms > 0.0


@pytest.mark.parametrize("case", ["redwood_h2", "poly_h2"])
def test_adaptive_search_matches_oracle(ctx, case):
    d = load(case)
    x, y, w = d["x"], d["y"], d["w"]
    h0 = o.rule_of_thumb(x, y, w)
    pts, em, d2 = setup(ctx, d)
    rh, ra, rl, rhs, rit = o.adaptive_search(x, y, w, d2, d["eg"], d["edge_mask"], h0)
    h, a, lm, it, hs = mk.adaptive_bandwidths(ctx, pts, em, h0)
    assert (h, a, it) == (rh, ra, rit)
    assert abs(np.float32(lm) - np.float32(rl)) <= 1e-6 * abs(rl)
    assert rel(hs, rhs).max() <= 4e-7
    # density at the per-point bandwidths left in the points object
    mk.edge_correction_weights(ctx, pts, em, 0.0)
    ew = pts.download(ew=True)[1]
    ref_ew, _ = o.edge_weights(x, y, 0.0, d2, d["eg"], d["edge_mask"], hs=rhs)
    assert rel(ew, ref_ew).max() <= 3e-6
    idx = mk.Index(ctx, pts, 0.0)
    dg = mk.Grid.of(d["dg"])
    dmask = torch.from_numpy(np.ascontiguousarray(d["density_mask"], np.float32)).cuda()
    out = torch.empty((dg.nrows, dg.ncols), dtype=torch.float32, device="cuda")
    mk.density_tile(ctx, idx, dg, 0, 0, dg.nrows, dg.ncols, dmask, out)
    ref_den, _ = o.density(x, y, w, ref_ew, 0.0, d["dg"], d["density_mask"], hs=rhs)
    nd = d["density_mask"] == d["dg"].nodata
    den = out.cpu().numpy()
    assert np.array_equal(den[nd], d["density_mask"][nd])
    assert rel(den[~nd], ref_den[~nd]).max() <= 3e-6


def test_adaptive_wrapped_points_keep_caller_h(ctx):
    """Points wrapping caller device arrays: the search writes its bandwidths
    into a buffer of its own, never into the caller's h array."""
    d = load("poly_h2")
    x = torch.from_numpy(d["x"]).cuda()
    y = torch.from_numpy(d["y"]).cuda()
    hcaller = torch.full_like(x, 7.0)
    pts = mk.Points.wrap(ctx, x, y, None, hcaller)
    h0 = o.rule_of_thumb(d["x"], d["y"])
    _, _, _, _, hs = mk.adaptive_bandwidths(ctx, pts, None, h0)
    torch.cuda.synchronize()
    assert torch.all(hcaller == 7.0)
    assert np.isfinite(hs).all() and (hs > 0).all()


def test_adaptive_deterministic(ctx):
    d = load("poly_h2")
    runs = []
    for _ in range(2):
        pts, em, _ = setup(ctx, d)
        runs.append(mk.adaptive_bandwidths(ctx, pts, em, 6.0))
    assert runs[0][:4] == runs[1][:4]
    assert np.array_equal(runs[0][4].view(np.uint32), runs[1][4].view(np.uint32))


def test_adaptive_rejects_bad_arguments(ctx):
    d = load("poly_h2")
    pts = mk.Points.upload(ctx, d["x"], d["y"])
    em = mk.Raster.upload(ctx, mk.Grid.of(d["eg"]), d["edge_mask"])
    mk.mark_boundary(ctx, em)
    with pytest.raises(mk.MgkError):
        mk.adaptive_bandwidths(ctx, pts, None, -1.0)
    with pytest.raises(mk.MgkError):  # edge correction needs the boundary distances first
        mk.loglik_adaptive(ctx, pts, em, 5.0, -0.5)
    assert synth is not None
