"""Out-of-core tile pipeline on the GPU: tiles streamed to a host sink match
the oracle, two runs are bitwise equal, and a run stopped by a failing sink
resumes from its completed tiles to the same raster bit for bit."""
import numpy as np
import pytest

import oracle_py as o

torch = pytest.importorskip("torch")
import mgpukde_tiled_b200 as mk  # noqa: E402
from mgpukde_tiled_b200 import synth  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-6


@pytest.fixture(scope="module")
def setup():
    ctx = mk.Context(0)
    c = synth.out_of_core(scale=0.02, seed=3)  # 8,000 points, 800 x 800 raster, h = 30
    dg = mk.Grid.of(c["density_grid"])
    mask = synth.rasterize_polygon(c["polygon"], c["density_grid"])
    pts = mk.Points.upload(ctx, c["x"], c["y"], c["w"])
    em = mk.Raster.upload(ctx, mk.Grid.of(c["edge_grid"]), c["edge_mask"])
    mk.calc_dist2_boundary(ctx, pts, em)
    mk.edge_correction_weights(ctx, pts, em, c["h"])
    idx = mk.Index(ctx, pts, c["h"])
    yield ctx, c, dg, mask, pts, idx
    ctx.close()


def run(ctx, idx, dg, mask, tile, done=None, fail_after=None):
    out = np.full((dg.nrows, dg.ncols), np.nan, np.float32)
    seen = []

    def sink(t, r0, c0, a):
        if fail_after is not None and len(seen) >= fail_after:
            return False
        out[r0:r0 + a.shape[0], c0:c0 + a.shape[1]] = a
        seen.append(t)
        return True

    ev = mk.density_stream(ctx, idx, dg, tile, sink, mask=mask, done=done, count=True)
    return out, seen, ev


def test_stream_matches_oracle_and_is_deterministic(setup):
    ctx, c, dg, mask, pts, idx = setup
    out, seen, ev = run(ctx, idx, dg, mask, 192)
    ntiles = ((dg.nrows + 191) // 192) * ((dg.ncols + 191) // 192)
    assert seen == list(range(ntiles))
    og_e = o.grid(*c["edge_grid"].astuple())
    b = o.mark_boundary(og_e, c["edge_mask"])
    d2 = o.dist2_boundary(c["x"], c["y"], og_e, b)
    ew, _ = o.edge_weights(c["x"], c["y"], c["h"], d2, og_e, c["edge_mask"])
    ref, rev = o.density(c["x"], c["y"], c["w"], ew, c["h"], o.grid(*c["density_grid"].astuple()), mask)
    nd = mask == dg.nodata
    assert np.array_equal(out[nd], mask[nd])
    rel = np.abs(out[~nd].astype(np.float64) - ref[~nd]) / np.maximum(np.abs(ref[~nd]), 1e-300)
    assert rel.max() <= RTOL
    assert ev == rev
    again, _, _ = run(ctx, idx, dg, mask, 192)
    assert np.array_equal(out.view(np.uint32), again.view(np.uint32))


def test_stream_resume_after_a_failed_sink(setup):
    ctx, c, dg, mask, pts, idx = setup
    full, _, _ = run(ctx, idx, dg, mask, 256)
    with pytest.raises(mk.MgkError) as e:
        run(ctx, idx, dg, mask, 256, fail_after=3)
    assert e.value.status == -6  # MGK_ERR_IO
    # the interrupted run: record what the sink completed, then resume
    out = np.full((dg.nrows, dg.ncols), np.nan, np.float32)
    done_tiles = []

    def sink_stop(t, r0, c0, a):
        if len(done_tiles) >= 3:
            return False
        out[r0:r0 + a.shape[0], c0:c0 + a.shape[1]] = a
        done_tiles.append(t)
        return True

    with pytest.raises(mk.MgkError):
        mk.density_stream(ctx, idx, dg, 256, sink_stop, mask=mask)
    ntiles = ((dg.nrows + 255) // 256) * ((dg.ncols + 255) // 256)
    done = np.zeros(ntiles, bool)
    done[done_tiles] = True

    def sink_rest(t, r0, c0, a):
        assert not done[t]
        out[r0:r0 + a.shape[0], c0:c0 + a.shape[1]] = a
        return True

    mk.density_stream(ctx, idx, dg, 256, sink_rest, mask=mask, done=done)
    assert np.array_equal(out.view(np.uint32), full.view(np.uint32))
    # the device is still usable
    again, _, _ = run(ctx, idx, dg, mask, 256)
    assert np.array_equal(again.view(np.uint32), full.view(np.uint32))


def test_stream_copy_sink_fills_a_host_array(setup):
    ctx, c, dg, mask, pts, idx = setup
    ref, _, _ = run(ctx, idx, dg, mask, 192)
    host = np.full((dg.nrows, dg.ncols), np.nan, np.float32)
    mk.density_stream(ctx, idx, dg, 192, host, mask=mask)
    assert np.array_equal(host.view(np.uint32), ref.view(np.uint32))


def test_stream_copy_sink_into_page_locked_memory(setup):
    ctx, c, dg, mask, pts, idx = setup
    ref, _, _ = run(ctx, idx, dg, mask, 192)
    host = torch.full((dg.nrows, dg.ncols), float("nan"), dtype=torch.float32, pin_memory=True).numpy()
    mk.density_stream(ctx, idx, dg, 192, host, mask=mask)
    assert np.array_equal(host.view(np.uint32), ref.view(np.uint32))
