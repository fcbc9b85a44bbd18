"""mgk_density_tile_noalloc: the density entry point that allocates nothing.

Callers that cannot let a library allocate device memory while they run (an
application that reserves all GPU memory for its own allocator, or a running
latency-critical loop in which cudaMalloc/cudaFree are not allowed) use this
variant; its scratch is one fixed device array inside the library.  This file
sorts last so that a run stopping at its first failure has already run every
other test.  Through the C ABI it checks, on two calls in a row:

* the densities against the FP64 oracle and against mgk_density_tile, both
  within the parity tolerance (1e-6 relative), with NoData passed through;
* that heavy blocks were split into several work items, i.e. that the FP64
  partial sums in the fixed scratch and their merge kernel were exercised
  (the call launches the merge kernel only when some block was split);

and that a tile beyond the fixed scratch is refused with a clear error.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle_py as o  # noqa: E402

import mgpukde_tiled_b200 as mk  # noqa: E402
from mgpukde_tiled_b200 import synth  # noqa: E402
from mgpukde_tiled_b200._native import MgkGrid, lib  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-6


def _noalloc(ctx, idx, grid, row0, col0, nr, nc, d_mask, d_out):
    g = grid.c()
    return lib().mgk_density_tile_noalloc(ctx.handle, idx._h, C.byref(g), int(row0), int(col0), int(nr), int(nc),
                                          C.c_void_p(d_mask.data_ptr()) if d_mask is not None else None,
                                          C.c_void_p(d_out.data_ptr()))


def _clustered_case():
    """20,000 weighted points in one tight cluster (sigma 30 cells, h = 10)
    over a 300 x 400 raster under a polygon mask; the tile is the 256 x 256
    window at row 20, column 10, whose four central 64 x 128 blocks each
    see about 14,000 of the points as candidates, against a work-item size
    of 2,048 candidates at this size, so they are split across work items."""
    rng = np.random.default_rng(11)
    n = 20000
    x = (140.0 + 30.0 * rng.standard_normal(n)).astype(np.float32)
    y = (150.0 + 30.0 * rng.standard_normal(n)).astype(np.float32)
    w = rng.lognormal(0.0, 0.5, n).astype(np.float32)
    sg = synth.Grid(400, 300, np.float32(0.0), np.float32(0.0), 1.0, -9999.0)
    poly = synth.star_polygon(400.0, 12)
    mask = synth.rasterize_polygon(poly, sg)
    return x, y, w, sg, mask, (20, 10, 256, 256), 10.0


def test_noalloc_matches_oracle_and_splits_blocks():
    x, y, w, sg, mask, (r0, c0, nr, nc), h = _clustered_case()
    ref, _ = o.density(x, y, w, np.ones(len(x)), h, o.grid(*sg.astuple()), mask, window=(r0, c0, nr, nc))
    tmask = np.ascontiguousarray(mask[r0:r0 + nr, c0:c0 + nc])
    valid = tmask != sg.nodata
    assert valid.sum() > 1000 and (~valid).sum() > 0
    dg = mk.Grid.of(sg)
    with mk.Context(0) as ctx:
        pts = mk.Points.upload(ctx, x, y, w)
        mk.unit_edge_weights(ctx, pts)
        idx = mk.Index(ctx, pts, h)
        d_mask = torch.from_numpy(tmask).cuda()
        alloc = torch.empty((nr, nc), dtype=torch.float32, device="cuda")
        mk.density_tile(ctx, idx, dg, r0, c0, nr, nc, d_mask, alloc)
        alloc_h = alloc.cpu().numpy().astype(np.float64)  # cells far from the cluster are exactly 0
        for call in range(2):
            out = torch.full((nr, nc), 12345.0, dtype=torch.float32, device="cuda")
            l0 = ctx.kernel_launches
            assert _noalloc(ctx, idx, dg, r0, c0, nr, nc, d_mask, out) == 0, lib().mgk_ctx_last_error(ctx.handle)
            # block counts + density + merge of the split blocks' partials
            assert ctx.kernel_launches - l0 == 3, "no block was split: the scratch partials went unused"
            got = out.cpu().numpy().astype(np.float64)
            assert np.array_equal(got[~valid], tmask[~valid])
            rel = np.abs(got[valid] - ref[valid]) / np.maximum(np.abs(ref[valid]), 1e-300)
            assert rel.max() <= RTOL, ("oracle", call, rel.max())
            rel_a = np.abs(got[valid] - alloc_h[valid]) / np.maximum(np.abs(alloc_h[valid]), 1e-300)
            assert rel_a.max() <= RTOL, ("mgk_density_tile", call, rel_a.max())
        idx.close()
        pts.close()


def test_noalloc_refuses_a_tile_beyond_its_scratch():
    c = synth.single_large(scale=0.05, seed=7)
    with mk.Context(0) as ctx:
        pts = mk.Points.upload(ctx, c["x"], c["y"], c["w"])
        mk.unit_edge_weights(ctx, pts)
        idx = mk.Index(ctx, pts, float(c["h"]))
        out = torch.empty((16, 16), dtype=torch.float32, device="cuda")
        big = MgkGrid(5000, 5000, 0.0, 0.0, 1.0, -9999.0)
        st = lib().mgk_density_tile_noalloc(ctx.handle, idx._h, C.byref(big), 0, 0, 4200, 4200, None,
                                            C.c_void_p(out.data_ptr()))
        assert st == -1 and b"4096" in lib().mgk_ctx_last_error(ctx.handle)
        # the device stays usable: a small tile still computes
        small = torch.empty((64, 64), dtype=torch.float32, device="cuda")
        assert _noalloc(ctx, idx, mk.Grid.of(c["density_grid"]), 0, 0, 64, 64, None, small) == 0
        idx.close()
        pts.close()
