"""B200-native (sm_100a) tiled fixed-bandwidth Gaussian KDE.

The hot path of mGPUKDE_tiled — density on a masked raster computed tile by
tile, exact edge correction, leave-one-out bandwidth selection — as CUDA
kernels behind a C ABI (include/mgk.h, libmgk.so).  This package is the
Python host side over that ABI; the C++ host driver with the reference's
command line is `_lib/mgkde_tiled`.
"""
from ._native import EXPORTS, LIB_PATH, MgkError, MgkGrid, lib  # noqa: F401
from .kde import (Context, Grid, Index, Points, Raster, autotune, calc_dist2_boundary, density_tile,  # noqa: F401
                  get_tuning, set_tuning,
                  density_stream, density_tiles, edge_correction_weights, kde_raster, log_likelihood_batch, mark_boundary,
                  mle_fixed_bandwidth, rule_of_thumb, unit_edge_weights, loglik_adaptive, adaptive_bandwidths,
                  kde_raster_rows, loo_share_edge_weights, loo_share_loglik)
from .serve import Server  # noqa: F401

__all__ = [
    "Context", "Grid", "Index", "Points", "Raster", "MgkError", "Server", "calc_dist2_boundary", "density_tile",
    "density_stream", "density_tiles", "autotune", "get_tuning", "set_tuning",
    "edge_correction_weights", "kde_raster", "log_likelihood_batch", "mark_boundary",
    "mle_fixed_bandwidth", "rule_of_thumb", "unit_edge_weights", "loglik_adaptive", "adaptive_bandwidths", "lib",
    "kde_raster_rows", "loo_share_edge_weights", "loo_share_loglik",
]
