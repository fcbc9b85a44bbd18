"""Several tiles per launch and the serving loop on the GPU.

Each result must be bitwise the same alone and in a mix (the tiles of a
batch are planned independently), and match the FP64 oracle within 1e-6
relative with exact NoData passthrough and exact eval counts.
"""
import numpy as np
import pytest

import oracle_py as o
from golden_cases import load, oracle_run

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


def _job(ctx, case):
    d = load(case)
    ref = oracle_run(d)
    pts = mk.Points.upload(ctx, d["x"], d["y"], d["w"], d["hs"])
    if int(d["edge"]):
        em = mk.Raster.upload(ctx, mk.Grid.of(d["eg"]), d["edge_mask"])
        mk.calc_dist2_boundary(ctx, pts, em)
        mk.edge_correction_weights(ctx, pts, em, ref["h"] if d["hs"] is None else 0.0)
    else:
        mk.unit_edge_weights(ctx, pts)
    idx = mk.Index(ctx, pts, ref["h"] if d["hs"] is None else 0.0)
    dg = mk.Grid.of(d["dg"])
    mask = torch.from_numpy(np.ascontiguousarray(d["density_mask"], np.float32)).cuda()
    return d, ref, pts, idx, dg, mask


def test_density_tiles_equal_alone_and_batched(ctx):
    cases = ["poly_fixed", "uniform_c0", "poly_varh", "redwood_h0"]
    built = [_job(ctx, c) for c in cases]
    alone, alone_ev = [], []
    for d, ref, pts, idx, dg, mask in built:
        out = torch.empty((dg.nrows, dg.ncols), dtype=torch.float32, device="cuda")
        alone_ev.append(mk.density_tile(ctx, idx, dg, 0, 0, dg.nrows, dg.ncols, mask, out, count=True))
        alone.append(out.cpu().numpy())
    outs = [torch.empty((b[4].nrows, b[4].ncols), dtype=torch.float32, device="cuda") for b in built]
    jobs = [(idx, dg, 0, 0, dg.nrows, dg.ncols, mask, out) for (d, ref, pts, idx, dg, mask), out in zip(built, outs)]
    ev = mk.density_tiles(ctx, jobs, count=True)
    for k, ((d, ref, pts, idx, dg, mask), out) in enumerate(zip(built, outs)):
        got = out.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), alone[k].view(np.uint32))
        assert ev[k] == alone_ev[k] == ref["density_evals"]
        nd = d["density_mask"] == d["dg"].nodata
        assert rel_err(got[~nd], ref["density"][~nd]).max() <= RTOL


def _requests(n_req, seed):
    """Small synthetic requests: mixture points, square rasters of 128-700
    cells, h in [2, 12] cells, half with a polygon edge mask, some with a
    polygon density mask."""
    r = np.random.default_rng(seed)
    out = []
    for k in range(n_req):
        side = int(r.integers(128, 700))
        n = int(r.integers(1000, 20000))
        x, y = synth.mixture_points(n, 5, float(side), 5.0, 60.0, seed * 100 + k)
        w = synth.lognormal_weights(n, seed * 100 + k + 50)
        g = synth.Grid(side, side, 0.0, 0.0, 1.0)
        h = float(r.uniform(2.0, 12.0))
        poly = synth.star_polygon(float(side), seed * 100 + k + 70)
        mask = synth.rasterize_polygon(poly, g) if k % 3 == 0 else None
        edge = k % 2 == 0
        eg = synth.Grid(side // 4, side // 4, 0.0, 0.0, 4.0)
        out.append(dict(x=x, y=y, w=w, h=h, grid=g, mask=mask, edge_grid=eg if edge else None,
                        edge_mask=synth.rasterize_polygon(poly, eg) if edge else None))
    return out


def _submit(srv, q):
    return srv.submit(q["x"], q["y"], q["w"], q["h"], mk.Grid.of(q["grid"]), q["mask"],
                      mk.Grid.of(q["edge_grid"]) if q["edge_grid"] is not None else None, q["edge_mask"])


def test_serving_mix_equals_alone_and_oracle():
    reqs = _requests(6, seed=3)
    with mk.Server(0, tile=256, max_active=4) as srv:
        alone = []
        for q in reqs:
            out, res = srv.wait(_submit(srv, q))
            alone.append((out.copy(), res))
        tickets = [_submit(srv, q) for q in reqs]
        mixed = [srv.wait(t) for t in tickets]
        st = srv.stats()
    assert st["max_batch"] >= 2  # the mix really shared launches
    for (a, ra), (b, rb) in zip(alone, mixed):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        assert ra["evals"] == rb["evals"]
    # one request with edge correction and a density mask against the oracle
    q = reqs[0]
    g = o.grid(*q["grid"].astuple())
    eg = o.grid(*q["edge_grid"].astuple())
    b = o.mark_boundary(eg, q["edge_mask"])
    d2 = o.dist2_boundary(q["x"], q["y"], eg, b)
    ew, eev = o.edge_weights(q["x"], q["y"], np.float32(q["h"]), d2, eg, q["edge_mask"])
    ref, rev = o.density(q["x"], q["y"], q["w"], ew, np.float32(q["h"]), g, q["mask"])
    got = alone[0][0]
    nd = q["mask"] == q["grid"].nodata
    assert np.array_equal(got[nd], q["mask"][nd])
    assert rel_err(got[~nd], ref[~nd]).max() <= RTOL
    assert alone[0][1]["evals"] == rev + eev


def test_serving_admission_under_a_small_budget():
    reqs = _requests(4, seed=5)
    with mk.Server(0, hbm_budget=600 << 20, tile=256, max_active=4) as srv:
        tickets = [_submit(srv, q) for q in reqs]
        res = [srv.wait(t) for t in tickets]
        st = srv.stats()
    assert st["completed"] == 4 and st["active"] == 0 and st["queued"] == 0
    assert all(r[1]["evals"] > 0 for r in res)


def test_serving_rejects_bad_requests():
    with mk.Server(0, tile=256, max_active=2) as srv:
        with pytest.raises(mk.MgkError):
            srv.submit(np.zeros(3), np.zeros(3), None, -1.0, mk.Grid(10, 10, 0.0, 0.0, 1.0))
