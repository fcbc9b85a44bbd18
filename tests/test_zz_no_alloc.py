"""mgk_density_tile_noalloc: the density entry point that allocates nothing.

Callers that cannot let a library allocate device memory while they run (an
application that reserves all GPU memory for its own allocator, or a running
latency-critical loop in which cudaMalloc/cudaFree are not allowed) use this
variant; its scratch is one fixed device array inside the library.  This file
sorts last so that a run stopping at its first failure has already run every
other test.  It checks, through the C ABI, that two calls in a row give the
same densities as mgk_density_tile within the parity tolerance (1e-6
relative), that NoData cells pass through, and that a tile beyond the fixed
scratch is refused with a clear error.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import mgpukde_tiled_b200 as mk  # noqa: E402
from mgpukde_tiled_b200 import synth  # noqa: E402
from mgpukde_tiled_b200._native import MgkGrid, lib  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-6


def _noalloc(ctx, idx, grid, row0, col0, nr, nc, d_mask, d_out):
    g = grid.c()
    st = lib().mgk_density_tile_noalloc(ctx.handle, idx._h, C.byref(g), int(row0), int(col0), int(nr), int(nc),
                                        C.c_void_p(d_mask.data_ptr()) if d_mask is not None else None,
                                        C.c_void_p(d_out.data_ptr()))
    return st


def test_noalloc_matches_allocating_entry_point():
    # dense clustered points so that heavy blocks are split (the scratch partials are used)
    c = synth.single_large(scale=0.25, seed=7)
    dg = mk.Grid.of(c["density_grid"])
    mask = synth.rasterize_polygon(c["polygon"], c["density_grid"])
    with mk.Context(0) as ctx:
        pts = mk.Points.upload(ctx, c["x"], c["y"], c["w"])
        mk.unit_edge_weights(ctx, pts)
        idx = mk.Index(ctx, pts, float(c["h"]))
        d_mask = torch.from_numpy(mask).cuda()
        ref = torch.empty((dg.nrows, dg.ncols), dtype=torch.float32, device="cuda")
        mk.density_tile(ctx, idx, dg, 0, 0, dg.nrows, dg.ncols, d_mask, ref)
        ref_h = ref.cpu().numpy()
        valid = mask != dg.nodata
        for call in range(2):
            out = torch.full((dg.nrows, dg.ncols), 12345.0, dtype=torch.float32, device="cuda")
            assert _noalloc(ctx, idx, dg, 0, 0, dg.nrows, dg.ncols, d_mask, out) == 0, \
                lib().mgk_ctx_last_error(ctx.handle)
            got = out.cpu().numpy()
            assert np.array_equal(got[~valid], mask[~valid])
            rel = np.abs(got[valid] - ref_h[valid]) / np.maximum(np.abs(ref_h[valid]), 1e-300)
            assert rel.max() <= RTOL, (call, rel.max())
        # a tile beyond the fixed scratch is refused, and the device stays usable
        big = MgkGrid(5000, 5000, 0.0, 0.0, 1.0, -9999.0)
        st = lib().mgk_density_tile_noalloc(ctx.handle, idx._h, C.byref(big), 0, 0, 4200, 4200, None,
                                            C.c_void_p(out.data_ptr()))
        assert st == -1 and b"4096" in lib().mgk_ctx_last_error(ctx.handle)
        idx.close()
        pts.close()
