"""Loader and ctypes signatures of libmgk.so (include/mgk.h).

The library is built in-tree (python -m mgpukde_tiled_b200.build).  There is
no fallback: if it is missing or cannot be loaded, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libmgk.so")

MGK_OK = 0
STATUS = {0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "HBM budget exceeded",
          -4: "no suitable CUDA device", -5: "device wait timed out", -6: "I/O error"}

# Every symbol include/mgk.h declares.
EXPORTS = [
    "mgk_ctx_create", "mgk_ctx_destroy", "mgk_ctx_set_stream", "mgk_ctx_synchronize",
    "mgk_ctx_last_error", "mgk_ctx_bytes_in_use", "mgk_status_string",
    "mgk_ctx_kernel_launches", "mgk_ctx_last_density_ms", "mgk_ctx_last_loo_ms", "mgk_ctx_last_loo_evals",
    "mgk_points_upload", "mgk_points_wrap", "mgk_points_destroy", "mgk_points_device_arrays",
    "mgk_points_download", "mgk_raster_upload", "mgk_raster_wrap", "mgk_raster_destroy",
    "mgk_mark_boundary", "mgk_raster_boundary_download", "mgk_boundary_dist",
    "mgk_edge_weights", "mgk_edge_weights_unit", "mgk_index_build", "mgk_index_destroy",
    "mgk_density_tile", "mgk_density_tile_fp64", "mgk_density_tile_noalloc", "mgk_density_tiles", "mgk_loo_loglik_batch",
    "mgk_mle_fixed_bandwidth", "mgk_rule_of_thumb", "mgk_kde_raster",
    "mgk_serve_create", "mgk_serve_submit", "mgk_serve_poll", "mgk_serve_wait", "mgk_serve_stats",
    "mgk_serve_destroy", "mgk_density_stream", "mgk_copy_sink", "mgk_ctx_get_tuning", "mgk_ctx_set_tuning",
    "mgk_autotune", "mgk_loglik_adaptive", "mgk_adaptive_bandwidths",
    "mgk_boundary_dist_within", "mgk_points_select", "mgk_points_size", "mgk_kde_raster_rows", "mgk_loo_share_edge_weights", "mgk_loo_share_loglik",
]


class MgkGrid(C.Structure):
    _fields_ = [("ncols", C.c_int64), ("nrows", C.c_int64), ("xll", C.c_float),
                ("yll", C.c_float), ("cs", C.c_float), ("nodata", C.c_float)]


class MgkTileJob(C.Structure):
    _fields_ = [("index", C.c_void_p), ("grid", MgkGrid), ("row0", C.c_int64), ("col0", C.c_int64),
                ("nrows", C.c_int64), ("ncols", C.c_int64), ("d_mask", C.c_void_p), ("d_out", C.c_void_p)]


class MgkRequest(C.Structure):
    _fields_ = [("n", C.c_int64), ("x", C.c_void_p), ("y", C.c_void_p), ("w", C.c_void_p), ("h", C.c_float),
                ("grid", MgkGrid), ("mask", C.c_void_p), ("edge", C.c_int), ("edge_grid", MgkGrid),
                ("edge_mask", C.c_void_p), ("out", C.c_void_p)]


class MgkResult(C.Structure):
    _fields_ = [("status", C.c_int), ("evals", C.c_int64), ("queue_ms", C.c_double), ("run_ms", C.c_double),
                ("total_ms", C.c_double)]


class MgkServeInfo(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("ticks", "tiles", "max_batch", "completed", "queued", "active",
                                          "reserved_bytes", "device_bytes")]


TILE_SOURCE = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                          C.POINTER(C.c_float))
TILE_SINK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                        C.POINTER(C.c_float))


class MgkCopyTarget(C.Structure):
    _fields_ = [("base", C.c_void_p), ("ncols", C.c_int64)]


class MgkTuning(C.Structure):
    _fields_ = [("bin_factor", C.c_float), ("split_waves", C.c_int32), ("tile_side", C.c_int64),
                ("density_ms", C.c_float), ("from_cache", C.c_int32)]


class MgkError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"mgk status {status} ({STATUS.get(status, '?')}): {msg}")
        self.status = status


_lib = None


def lib():
    """Loads libmgk.so; raises if it is absent (there is no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m mgpukde_tiled_b200.build`")
    L = C.CDLL(LIB_PATH)
    P, I64, I = C.c_void_p, C.c_int64, C.c_int
    PP = C.POINTER(C.c_void_p)
    G = C.POINTER(MgkGrid)
    sig = {
        "mgk_ctx_create": (I, [I, C.c_uint64, PP]),
        "mgk_ctx_destroy": (I, [P]),
        "mgk_ctx_set_stream": (I, [P, P]),
        "mgk_ctx_synchronize": (I, [P]),
        "mgk_ctx_last_error": (C.c_char_p, [P]),
        "mgk_ctx_bytes_in_use": (C.c_uint64, [P]),
        "mgk_status_string": (C.c_char_p, [I]),
        "mgk_ctx_kernel_launches": (C.c_uint64, [P]),
        "mgk_ctx_last_density_ms": (C.c_float, [P]),
        "mgk_ctx_last_loo_ms": (C.c_float, [P]),
        "mgk_ctx_last_loo_evals": (C.c_int, [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "mgk_points_upload": (I, [P, I64, P, P, P, P, PP]),
        "mgk_points_wrap": (I, [P, I64, P, P, P, P, PP]),
        "mgk_points_destroy": (I, [P]),
        "mgk_points_device_arrays": (I, [P, PP, PP, PP, PP, PP, PP]),
        "mgk_points_download": (I, [P, P, P]),
        "mgk_raster_upload": (I, [P, G, P, PP]),
        "mgk_raster_wrap": (I, [P, G, P, PP]),
        "mgk_raster_destroy": (I, [P]),
        "mgk_mark_boundary": (I, [P, P, C.POINTER(I64)]),
        "mgk_raster_boundary_download": (I, [P, P]),
        "mgk_boundary_dist": (I, [P, P, P]),
        "mgk_edge_weights": (I, [P, P, P, C.c_float, C.POINTER(I64)]),
        "mgk_edge_weights_unit": (I, [P, P]),
        "mgk_index_build": (I, [P, P, C.c_float, C.c_float, PP]),
        "mgk_index_destroy": (I, [P]),
        "mgk_density_tile": (I, [P, P, G, I64, I64, I64, I64, P, P, C.POINTER(I64)]),
        "mgk_density_tile_fp64": (I, [P, P, G, I64, I64, I64, I64, P, P, C.POINTER(I64)]),
        "mgk_density_tile_noalloc": (I, [P, P, G, I64, I64, I64, I64, P, P]),
        "mgk_density_tiles": (I, [P, I, C.POINTER(MgkTileJob), C.POINTER(I64)]),
        "mgk_loo_loglik_batch": (I, [P, P, P, P, I, P, C.POINTER(I)]),
        "mgk_serve_create": (I, [I, C.c_uint64, I64, I, C.POINTER(P)]),
        "mgk_serve_submit": (I, [P, C.POINTER(MgkRequest), C.POINTER(C.c_uint64)]),
        "mgk_serve_poll": (I, [P, C.c_uint64, C.POINTER(I), C.POINTER(MgkResult)]),
        "mgk_serve_wait": (I, [P, C.c_uint64, C.c_double, C.POINTER(MgkResult)]),
        "mgk_serve_stats": (I, [P, C.POINTER(MgkServeInfo)]),
        "mgk_serve_destroy": (I, [P]),
        "mgk_density_stream": (I, [P, P, G, I64, TILE_SOURCE, P, TILE_SINK, P, P, C.POINTER(I64)]),
        "mgk_copy_sink": (I, [P, I64, I64, I64, I64, I64, C.POINTER(C.c_float)]),
        "mgk_ctx_get_tuning": (I, [P, C.POINTER(MgkTuning)]),
        "mgk_ctx_set_tuning": (I, [P, C.POINTER(MgkTuning)]),
        "mgk_autotune": (I, [P, P, C.c_float, G, C.c_char_p, C.POINTER(MgkTuning)]),
        "mgk_mle_fixed_bandwidth": (I, [P, P, P, C.c_float, C.POINTER(C.c_float), C.POINTER(I)]),
        "mgk_loglik_adaptive": (I, [P, P, P, C.c_float, C.c_float, C.POINTER(C.c_double)]),
        "mgk_adaptive_bandwidths": (I, [P, P, P, C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                        C.POINTER(C.c_double), C.POINTER(I), P]),
        "mgk_rule_of_thumb": (C.c_float, [I64, P, P, P]),
        "mgk_kde_raster": (I, [P, I64, P, P, P, P, C.c_float, I, G, P, G, P, I64, P, P, C.POINTER(I64)]),
        "mgk_points_select": (I, [P, P, C.c_double, C.c_double, C.c_double, C.c_double, PP]),
        "mgk_points_size": (I64, [P]),
        "mgk_boundary_dist_within": (I, [P, P, P, C.c_double]),
        "mgk_kde_raster_rows": (I, [P, I64, P, P, P, P, C.c_float, I, G, P, G, I64, I64, P, I64, P,
                                    C.POINTER(I64)]),
        "mgk_loo_share_edge_weights": (I, [P, P, P, P, I, I, I, P, C.POINTER(I64)]),
        "mgk_loo_share_loglik": (I, [P, P, P, I, I, I, P, P, C.POINTER(I64)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L
