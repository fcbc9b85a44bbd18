"""Autotuner: measured settings are applied and cached, a second call with a
matching workload reads the cache, and results under the tuned settings
still match the oracle."""
import numpy as np
import pytest

from golden_cases import load, oracle_run

torch = pytest.importorskip("torch")
import mgpukde_tiled_b200 as mk  # noqa: E402
from mgpukde_tiled_b200 import synth  # noqa: E402

pytestmark = pytest.mark.gpu


def test_autotune_caches_and_keeps_parity(tmp_path):
    ctx = mk.Context(0)
    c = synth.single_large(scale=0.1, seed=1)  # 10,000 points, 1000^2 raster, h = 50
    pts = mk.Points.upload(ctx, c["x"], c["y"], c["w"])
    cache = str(tmp_path / "tune.txt")
    t1 = mk.autotune(ctx, pts, c["h"], mk.Grid.of(c["density_grid"]), cache)
    assert t1["bin_factor"] in (0.5, 0.75, 1.0, 1.25) and not t1["from_cache"]
    assert mk.get_tuning(ctx)["bin_factor"] == t1["bin_factor"]
    t2 = mk.autotune(ctx, pts, c["h"], mk.Grid.of(c["density_grid"]), cache)
    assert t2["from_cache"] and t2["bin_factor"] == t1["bin_factor"]
    # a golden case computed under a non-default bin factor and split
    mk.set_tuning(ctx, bin_factor=0.5, split_waves=32)
    d = load("poly_fixed")
    ref = oracle_run(d)
    hfix = ref["h"] if d["hs"] is None else 0.0  # this case carries per-point bandwidths
    p2 = mk.Points.upload(ctx, d["x"], d["y"], d["w"], d["hs"])
    em = mk.Raster.upload(ctx, mk.Grid.of(d["eg"]), d["edge_mask"])
    mk.calc_dist2_boundary(ctx, p2, em)
    mk.edge_correction_weights(ctx, p2, em, hfix)
    idx = mk.Index(ctx, p2, hfix)
    dg = mk.Grid.of(d["dg"])
    mask = torch.from_numpy(np.ascontiguousarray(d["density_mask"], np.float32)).cuda()
    out = torch.empty((dg.nrows, dg.ncols), dtype=torch.float32, device="cuda")
    ev = mk.density_tile(ctx, idx, dg, 0, 0, dg.nrows, dg.ncols, mask, out, count=True)
    got = out.cpu().numpy()
    nd = d["density_mask"] == d["dg"].nodata
    rel = np.abs(got[~nd].astype(np.float64) - ref["density"][~nd]) / np.maximum(np.abs(ref["density"][~nd]), 1e-300)
    assert rel.max() <= 1e-6 and ev == ref["density_evals"]
    ctx.close()
