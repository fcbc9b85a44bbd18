"""mgk_boundary_dist_within: boundary distances exact up to a reach.

Points whose nearest boundary cell lies within the reach get the brute-force
FP64 minimum bit for bit, the others a value above reach^2; the edge weights
computed from them are bitwise those of the exact distances whenever the
reach covers 3h, and every call that reads the distances refuses a reach
below 3h for its bandwidths (MGK_ERR_INVALID) instead of misreading them."""
import numpy as np
import pytest

import oracle_py as o

torch = pytest.importorskip("torch")
import mgpukde_tiled_b200 as mk  # noqa: E402
from mgpukde_tiled_b200 import synth  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mk.Context(0)
    yield c
    c.close()


def _case():
    c = synth.single_large(scale=0.2, seed=9)  # 40,000 points, 2,000^2 domain, edge mask 500^2 at cell 4
    og = o.grid(*c["edge_grid"].astuple())
    ref = o.dist2_boundary(c["x"], c["y"], og, o.mark_boundary(og, c["edge_mask"]))
    return c, ref


@pytest.mark.parametrize("reach", [37.5, 150.0, 600.0])
def test_distances_exact_within_the_reach(ctx, reach):
    c, ref = _case()
    pts = mk.Points.upload(ctx, c["x"], c["y"], c["w"])
    em = mk.Raster.upload(ctx, mk.Grid.of(c["edge_grid"]), c["edge_mask"])
    mk.calc_dist2_boundary(ctx, pts, em, reach=reach)
    d2, _ = pts.download(dist2=True, ew=False)
    near = ref <= reach * reach
    assert near.sum() > 100 and (~near).sum() > 100
    assert np.array_equal(d2[near], ref[near])
    assert np.all(d2[~near] > reach * reach)
    em.close()
    pts.close()


def test_edge_weights_and_likelihood_unchanged_by_a_reach_of_3h(ctx):
    c, _ = _case()
    h = float(c["h"])
    eg = mk.Grid.of(c["edge_grid"])
    full = mk.Points.upload(ctx, c["x"], c["y"], c["w"])
    capped = mk.Points.upload(ctx, c["x"], c["y"], c["w"])
    em = mk.Raster.upload(ctx, eg, c["edge_mask"])
    em_cap = mk.Raster.upload(ctx, eg, c["edge_mask"])  # its candidate lists are built for the reach
    mk.calc_dist2_boundary(ctx, full, em)
    mk.calc_dist2_boundary(ctx, capped, em_cap, reach=3.0 * h * (1.0 + 1e-6))
    e_full = mk.edge_correction_weights(ctx, full, em, h, count=True)
    e_cap = mk.edge_correction_weights(ctx, capped, em_cap, h, count=True)
    _, w_full = full.download(ew=True)
    _, w_cap = capped.download(ew=True)
    assert e_full == e_cap and np.array_equal(w_full.view(np.uint32), w_cap.view(np.uint32))
    hs = np.array([20.0, 35.0, 50.0], np.float32)
    l_full, b_full = mk.log_likelihood_batch(ctx, full, em, hs)
    l_cap, b_cap = mk.log_likelihood_batch(ctx, capped, em_cap, hs)
    assert np.array_equal(l_full, l_cap) and b_full == b_cap
    em_cap.close()
    em.close()
    capped.close()
    full.close()


def test_a_reach_below_3h_is_refused(ctx):
    c, _ = _case()
    h = float(c["h"])
    pts = mk.Points.upload(ctx, c["x"], c["y"], c["w"])
    em = mk.Raster.upload(ctx, mk.Grid.of(c["edge_grid"]), c["edge_mask"])
    mk.calc_dist2_boundary(ctx, pts, em, reach=2.5 * h)
    for call in (lambda: mk.edge_correction_weights(ctx, pts, em, h),
                 lambda: mk.log_likelihood_batch(ctx, pts, em, np.array([h], np.float32)),
                 lambda: mk.loglik_adaptive(ctx, pts, em, h, -0.5)):
        with pytest.raises(mk.MgkError) as e:
            call()
        assert e.value.status == -1
    # a smaller bandwidth is covered
    mk.edge_correction_weights(ctx, pts, em, 0.8 * h)
    # per-point bandwidths: the largest one decides
    hp = np.full(len(c["x"]), 0.5 * h, np.float32)
    hp[7] = h
    pp = mk.Points.upload(ctx, c["x"], c["y"], c["w"], hp)
    mk.calc_dist2_boundary(ctx, pp, em, reach=2.5 * h)
    with pytest.raises(mk.MgkError):
        mk.edge_correction_weights(ctx, pp, em, 0.0)
    mk.calc_dist2_boundary(ctx, pp, em, reach=3.0 * h * (1.0 + 1e-6))
    mk.edge_correction_weights(ctx, pp, em, 0.0)
    for p in (pp, pts):
        p.close()
    em.close()
