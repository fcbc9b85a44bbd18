"""Python host API over the C ABI (include/mgk.h).

Names follow the reference's operations (kde_cuda_kdtr_tiled.cu): MarkBoundary,
CalcDist2Boundary, EdgeCorrectionWeightsExact, the tiled density loop,
LogLikelihood / MLE_FixedBandWidth and the rule-of-thumb bandwidth.  Device
buffers are passed as torch CUDA tensors (or raw device pointers as ints);
host buffers as numpy arrays.  Every call goes to libmgk.so; a failure raises
MgkError with the library's message.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._native import TILE_SINK, TILE_SOURCE, MgkCopyTarget, MgkError, MgkGrid, MgkTileJob, MgkTuning, lib


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, int):
        return C.c_void_p(a)
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(C.c_void_p)
    raise TypeError(f"cannot pass {type(a)}")


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


@dataclass
class Grid:
    """Raster geometry (AsciiRaster fields): row 0 is the top row."""

    ncols: int
    nrows: int
    xll: float
    yll: float
    cs: float
    nodata: float = -9999.0

    def c(self) -> MgkGrid:
        return MgkGrid(int(self.ncols), int(self.nrows), float(self.xll), float(self.yll),
                       float(self.cs), float(self.nodata))

    @classmethod
    def of(cls, g) -> "Grid":
        return cls(int(g.ncols), int(g.nrows), float(g.xll), float(g.yll), float(g.cs), float(g.nodata))


class Context:
    """A device, a CUDA stream and an HBM budget (mgk_ctx)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, stream=None):
        self._h = C.c_void_p()
        st = lib().mgk_ctx_create(int(device), int(hbm_budget), C.byref(self._h))
        if st != 0:
            raise MgkError(st, "mgk_ctx_create failed")
        if stream is not None:
            self.set_stream(stream)

    def check(self, st):
        if st != 0:
            raise MgkError(st, lib().mgk_ctx_last_error(self._h).decode())

    def set_stream(self, stream):
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        self.check(lib().mgk_ctx_set_stream(self._h, C.c_void_p(s)))

    def synchronize(self):
        self.check(lib().mgk_ctx_synchronize(self._h))

    @property
    def bytes_in_use(self) -> int:
        return int(lib().mgk_ctx_bytes_in_use(self._h))

    @property
    def kernel_launches(self) -> int:
        return int(lib().mgk_ctx_kernel_launches(self._h))

    @property
    def last_density_ms(self) -> float:
        return float(lib().mgk_ctx_last_density_ms(self._h))

    @property
    def last_loo_ms(self) -> float:
        return float(lib().mgk_ctx_last_loo_ms(self._h))

    @property
    def last_loo_evals(self):
        """(edge-mask cells, point pairs) in the cutoff in the last LOO batch run."""
        e, l = C.c_int64(), C.c_int64()
        lib().mgk_ctx_last_loo_evals(self._h, C.byref(e), C.byref(l))
        return int(e.value), int(l.value)

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().mgk_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Points:
    """Device-resident SamplePoints (+ per-point h, boundary distance, edge weight)."""

    def __init__(self, ctx: Context, handle, n: int, keep=()):
        self.ctx, self._h, self.n, self._keep = ctx, handle, n, keep

    @classmethod
    def upload(cls, ctx: Context, x, y, w=None, h=None) -> "Points":
        x, y, w, h = _f32(x), _f32(y), _f32(w), _f32(h)
        out = C.c_void_p()
        ctx.check(lib().mgk_points_upload(ctx.handle, len(x), _ptr(x), _ptr(y), _ptr(w), _ptr(h), C.byref(out)))
        return cls(ctx, out, len(x))

    @classmethod
    def wrap(cls, ctx: Context, x, y, w=None, h=None) -> "Points":
        """Over device arrays (torch CUDA float32 tensors); they must outlive the handle."""
        out = C.c_void_p()
        n = int(x.numel()) if hasattr(x, "numel") else len(x)
        ctx.check(lib().mgk_points_wrap(ctx.handle, n, _ptr(x), _ptr(y), _ptr(w), _ptr(h), C.byref(out)))
        return cls(ctx, out, n, keep=(x, y, w, h))

    def select(self, xlo=-np.inf, xhi=np.inf, ylo=-np.inf, yhi=np.inf) -> "Points":
        """The points inside [xlo, xhi] x [ylo, yhi] (input order) as a new
        device point set (mgk_points_select: a rank's halo points)."""
        big = np.finfo(np.float64).max
        out = C.c_void_p()
        self.ctx.check(lib().mgk_points_select(self.ctx.handle, self._h, max(float(xlo), -big), min(float(xhi), big),
                                               max(float(ylo), -big), min(float(yhi), big), C.byref(out)))
        return Points(self.ctx, out, int(lib().mgk_points_size(out)))

    def device_arrays(self):
        ps = [C.c_void_p() for _ in range(6)]
        self.ctx.check(lib().mgk_points_device_arrays(self._h, *[C.byref(p) for p in ps]))
        return dict(zip(("x", "y", "w", "h", "dist2", "ew"), (p.value for p in ps)))

    def download(self, dist2=False, ew=True):
        d = np.zeros(self.n, np.float64) if dist2 else None
        e = np.zeros(self.n, np.float32) if ew else None
        self.ctx.check(lib().mgk_points_download(self._h, _ptr(d), _ptr(e)))
        return d, e

    def close(self):
        # objects are destroyed before their context (the context owns the memory pool)
        if self._h and self.ctx.handle:
            lib().mgk_points_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Raster:
    """Device-resident mask raster (AsciiRaster)."""

    def __init__(self, ctx, handle, grid, keep=None):
        self.ctx, self._h, self.grid, self._keep = ctx, handle, grid, keep

    @classmethod
    def upload(cls, ctx: Context, grid: Grid, mask) -> "Raster":
        m = _f32(mask).reshape(-1)
        g = grid.c()
        out = C.c_void_p()
        ctx.check(lib().mgk_raster_upload(ctx.handle, C.byref(g), _ptr(m), C.byref(out)))
        return cls(ctx, out, grid)

    @classmethod
    def wrap(cls, ctx: Context, grid: Grid, d_mask) -> "Raster":
        g = grid.c()
        out = C.c_void_p()
        ctx.check(lib().mgk_raster_wrap(ctx.handle, C.byref(g), _ptr(d_mask), C.byref(out)))
        return cls(ctx, out, grid, keep=d_mask)

    def boundary(self) -> np.ndarray:
        out = np.zeros((self.grid.nrows, self.grid.ncols), np.uint8)
        self.ctx.check(lib().mgk_raster_boundary_download(self._h, _ptr(out)))
        return out

    def close(self):
        if self._h and self.ctx.handle:
            lib().mgk_raster_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Index:
    """Cell-binned point index (replaces the k-d tree)."""

    def __init__(self, ctx: Context, points: Points, h: float, bin_size: float = 0.0):
        self.ctx = ctx
        self._h = C.c_void_p()
        ctx.check(lib().mgk_index_build(ctx.handle, points._h, float(h), float(bin_size), C.byref(self._h)))

    def close(self):
        if self._h and self.ctx.handle:
            lib().mgk_index_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mark_boundary(ctx: Context, raster: Raster) -> int:
    """MarkBoundary: returns the number of boundary cells."""
    nb = C.c_int64()
    ctx.check(lib().mgk_mark_boundary(ctx.handle, raster._h, C.byref(nb)))
    return nb.value


def calc_dist2_boundary(ctx: Context, points: Points, raster: Raster, reach=None) -> None:
    """CalcDist2Boundary: exact FP64 squared distance of each point to the
    boundary.  reach: exact only for points within that distance of the
    boundary (the others get a value above reach^2); 3 h_max is all the edge
    weights and likelihoods need (mgk_boundary_dist_within)."""
    if reach is None:
        ctx.check(lib().mgk_boundary_dist(ctx.handle, points._h, raster._h))
    else:
        ctx.check(lib().mgk_boundary_dist_within(ctx.handle, points._h, raster._h, float(reach)))


def edge_correction_weights(ctx: Context, points: Points, raster: Raster, h: float, count=False):
    """EdgeCorrectionWeightsExact / CalcEdgeCorrectionWeights (h <= 0: per-point h)."""
    ev = C.c_int64()
    ctx.check(lib().mgk_edge_weights(ctx.handle, points._h, raster._h, float(h), C.byref(ev) if count else None))
    return ev.value if count else None


def unit_edge_weights(ctx: Context, points: Points) -> None:
    ctx.check(lib().mgk_edge_weights_unit(ctx.handle, points._h))


def density_tile(ctx: Context, index: Index, grid: Grid, row0, col0, nr, nc, d_mask, d_out,
                 count=False, fp64=False):
    """Density of one tile into d_out (device, nr*nc float32)."""
    g = grid.c()
    ev = C.c_int64()
    f = lib().mgk_density_tile_fp64 if fp64 else lib().mgk_density_tile
    ctx.check(f(ctx.handle, index._h, C.byref(g), int(row0), int(col0), int(nr), int(nc), _ptr(d_mask),
                _ptr(d_out), C.byref(ev) if count else None))
    return ev.value if count else None


def density_tiles(ctx: Context, jobs, count=False):
    """Several tiles in one launch.  jobs: sequence of (index, grid, row0,
    col0, nr, nc, d_mask, d_out) tuples; returns per-job eval counts when
    count is set."""
    arr = (MgkTileJob * max(len(jobs), 1))()
    for k, (index, grid, row0, col0, nr, nc, d_mask, d_out) in enumerate(jobs):
        arr[k] = MgkTileJob(index._h, grid.c(), int(row0), int(col0), int(nr), int(nc), _ptr(d_mask), _ptr(d_out))
    ev = (C.c_int64 * max(len(jobs), 1))()
    ctx.check(lib().mgk_density_tiles(ctx.handle, len(jobs), arr, ev if count else None))
    return [int(ev[k]) for k in range(len(jobs))] if count else None


def density_stream(ctx: Context, index: Index, grid: Grid, tile: int, sink, mask=None, done=None, count=False):
    """Out-of-core density: sink(tile_id, row0, col0, tile_array) receives
    every finished tile (a float32 nrows x ncols view, valid during the call;
    return False to stop), or sink is a whole host float32 array that the
    library's own copy sink fills; mask is None, a full host array, or
    mask(tile_id, row0, col0, nrows, ncols) -> array.  done: optional bool
    per tile (row-major tile order) to skip.  Returns the eval count when
    count is set."""
    def src_cb(user, t, r0, c0, nr, nc, buf):
        try:
            m = mask[r0:r0 + nr, c0:c0 + nc] if isinstance(mask, np.ndarray) else mask(t, r0, c0, nr, nc)
            dst = np.ctypeslib.as_array(buf, shape=(nr * nc,)).reshape(nr, nc)
            dst[...] = m
            return 0
        except Exception:  # noqa: BLE001 - reported to the library as a failed read
            return 1

    def sink_cb(user, t, r0, c0, nr, nc, buf):
        try:
            arr = np.ctypeslib.as_array(buf, shape=(nr * nc,)).reshape(nr, nc)
            return 0 if sink(int(t), int(r0), int(c0), arr) is not False else 1
        except Exception:  # noqa: BLE001 - reported to the library as a failed write
            return 1

    src = TILE_SOURCE(src_cb) if mask is not None else TILE_SOURCE()
    target = None
    if isinstance(sink, np.ndarray):
        if sink.dtype != np.float32 or not sink.flags.c_contiguous or sink.shape != (grid.nrows, grid.ncols):
            raise ValueError("sink array must be a C-contiguous float32 nrows x ncols array")
        target = MgkCopyTarget(sink.ctypes.data, grid.ncols)
        snk = C.cast(lib().mgk_copy_sink, TILE_SINK)
    else:
        snk = TILE_SINK(sink_cb)
    g = grid.c()
    d = None if done is None else np.ascontiguousarray(done, dtype=np.uint8)
    ev = C.c_int64()
    ctx.check(lib().mgk_density_stream(ctx.handle, index._h, C.byref(g), int(tile), src, None, snk,
                                       C.cast(C.pointer(target), C.c_void_p) if target is not None else None, _ptr(d),
                                       C.byref(ev) if count else None))
    return ev.value if count else None


def _tuning_dict(t):
    return {"bin_factor": float(t.bin_factor), "split_waves": int(t.split_waves), "tile_side": int(t.tile_side),
            "density_ms": float(t.density_ms), "from_cache": bool(t.from_cache)}


def autotune(ctx: Context, points: Points, h: float, grid: Grid, cache_file: str | None = None) -> dict:
    """Measures and applies the index bin factor and the streamed tile side
    for this workload (cached in cache_file when given)."""
    t = MgkTuning()
    g = grid.c()
    ctx.check(lib().mgk_autotune(ctx.handle, points._h, float(h), C.byref(g),
                                 cache_file.encode() if cache_file else None, C.byref(t)))
    return _tuning_dict(t)


def get_tuning(ctx: Context) -> dict:
    t = MgkTuning()
    ctx.check(lib().mgk_ctx_get_tuning(ctx.handle, C.byref(t)))
    return _tuning_dict(t)


def set_tuning(ctx: Context, bin_factor=0.5, split_waves=4, tile_side=0):
    t = MgkTuning(float(bin_factor), int(split_waves), int(tile_side), 0.0, 0)
    ctx.check(lib().mgk_ctx_set_tuning(ctx.handle, C.byref(t)))


def log_likelihood_batch(ctx: Context, points: Points, raster: Raster | None, hgrid):
    """LogLikelihood over a grid of fixed bandwidths; returns (logL[nh], argmax)."""
    hs = _f32(hgrid)
    out = np.zeros(len(hs), np.float64)
    am = C.c_int()
    ctx.check(lib().mgk_loo_loglik_batch(ctx.handle, points._h, raster._h if raster else None, _ptr(hs),
                                         len(hs), _ptr(out), C.byref(am)))
    return out, am.value


def loo_share_edge_weights(ctx: Context, points: Points, raster: Raster, hgrid, part: int, nparts: int, d_ew_all,
                           count=False):
    """Multi-GPU bandwidth selection, step 1 on rank `part` of `nparts`: the
    edge weights of this rank's points for every h into its chunk of d_ew_all
    (device float32, nparts * nh * ceil(n / nparts)); returns the eval count
    when count is set."""
    hs = _f32(hgrid)
    ev = C.c_int64()
    ctx.check(lib().mgk_loo_share_edge_weights(ctx.handle, points._h, raster._h, _ptr(hs), len(hs), int(part),
                                               int(nparts), _ptr(d_ew_all), C.byref(ev) if count else None))
    return ev.value if count else None


def loo_share_loglik(ctx: Context, points: Points, hgrid, part: int, nparts: int, d_ew_all=None):
    """Multi-GPU bandwidth selection, step 2 on rank `part` of `nparts`: the
    FP64 partial log likelihoods (nh) of this rank's share of the queries, and
    its pair count; summed over ranks they are logL."""
    hs = _f32(hgrid)
    out = np.zeros(len(hs), np.float64)
    ev = C.c_int64()
    ctx.check(lib().mgk_loo_share_loglik(ctx.handle, points._h, _ptr(hs), len(hs), int(part), int(nparts),
                                         _ptr(d_ew_all), _ptr(out), C.byref(ev)))
    return out, ev.value


def mle_fixed_bandwidth(ctx: Context, points: Points, raster: Raster | None, h0: float):
    """MLE_FixedBandWidth (golden section); returns (h_opt, iterations)."""
    h = C.c_float()
    it = C.c_int()
    ctx.check(lib().mgk_mle_fixed_bandwidth(ctx.handle, points._h, raster._h if raster else None, float(h0),
                                            C.byref(h), C.byref(it)))
    return h.value, it.value


def loglik_adaptive(ctx: Context, points: Points, raster: Raster | None, h: float, alpha: float) -> float:
    """LogLikelihood(h, alpha) with adaptive bandwidths (h_option 2)."""
    v = C.c_double()
    ctx.check(lib().mgk_loglik_adaptive(ctx.handle, points._h, raster._h if raster else None, float(h),
                                        float(alpha), C.byref(v)))
    return v.value


def adaptive_bandwidths(ctx: Context, points: Points, raster: Raster | None, h0: float):
    """h_option 2: Hooke-Jeeves over (h, alpha); returns (h, alpha, lmax, iterations, hs[n])."""
    h, a, lm, it = C.c_float(), C.c_float(), C.c_double(), C.c_int()
    hs = np.empty(points.n, np.float32)
    ctx.check(lib().mgk_adaptive_bandwidths(ctx.handle, points._h, raster._h if raster else None, float(h0),
                                            C.byref(h), C.byref(a), C.byref(lm), C.byref(it), _ptr(hs)))
    return h.value, a.value, lm.value, it.value, hs


def rule_of_thumb(x, y, w=None) -> float:
    x, y, w = _f32(x), _f32(y), _f32(w)
    return float(lib().mgk_rule_of_thumb(len(x), _ptr(x), _ptr(y), _ptr(w)))


def kde_raster(ctx: Context, x, y, w, h, dens_grid: Grid, dens_mask=None, edge_grid: Grid | None = None,
               edge_mask=None, h_pp=None, tile=0, out=None, return_ew=False, count=False):
    """The whole path from host buffers; returns (density[nrows, ncols], edge weights|None, evals|None).
    count: also count the in-cutoff pairs (the counting kernels run somewhat slower)."""
    x, y, w, h_pp = _f32(x), _f32(y), _f32(w), _f32(h_pp)
    dm = None if dens_mask is None else _f32(dens_mask).reshape(-1)
    em = None if edge_mask is None else _f32(edge_mask).reshape(-1)
    if out is None:
        out = np.empty((dens_grid.nrows, dens_grid.ncols), np.float32)
    ew = np.empty(len(x), np.float32) if return_ew else None
    dg = dens_grid.c()
    eg = edge_grid.c() if edge_grid is not None else MgkGrid()
    ev = C.c_int64()
    ctx.check(lib().mgk_kde_raster(ctx.handle, len(x), _ptr(x), _ptr(y), _ptr(w), _ptr(h_pp),
                                   float(h if h is not None else 0.0), int(edge_grid is not None),
                                   C.byref(eg), _ptr(em), C.byref(dg), _ptr(dm), int(tile), _ptr(out), _ptr(ew),
                                   C.byref(ev) if count else None))
    return out, ew, (ev.value if count else None)


def kde_raster_rows(ctx: Context, x, y, w, h, dens_grid: Grid, row0: int, nrows: int, dens_mask_rows=None,
                    edge_grid: Grid | None = None, edge_mask=None, h_pp=None, tile=0, out=None, count=False):
    """Rows [row0, row0 + nrows) of the whole path from host buffers (one
    rank's share of a study split by rows); returns (density[nrows, ncols],
    evals|None).  dens_mask_rows: the rows' part of the density mask."""
    x, y, w, h_pp = _f32(x), _f32(y), _f32(w), _f32(h_pp)
    dm = None if dens_mask_rows is None else _f32(dens_mask_rows).reshape(-1)
    em = None if edge_mask is None else _f32(edge_mask).reshape(-1)
    if out is None:
        out = np.empty((nrows, dens_grid.ncols), np.float32)
    dg = dens_grid.c()
    eg = edge_grid.c() if edge_grid is not None else MgkGrid()
    ev = C.c_int64()
    ctx.check(lib().mgk_kde_raster_rows(ctx.handle, len(x), _ptr(x), _ptr(y), _ptr(w), _ptr(h_pp),
                                        float(h if h is not None else 0.0), int(edge_grid is not None),
                                        C.byref(eg), _ptr(em), C.byref(dg), int(row0), int(nrows), _ptr(dm),
                                        int(tile), _ptr(out), C.byref(ev) if count else None))
    return out, (ev.value if count else None)
