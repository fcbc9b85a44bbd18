"""ctypes front end of the FP64 oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class OrcGrid(C.Structure):
    _fields_ = [("ncols", C.c_int64), ("nrows", C.c_int64), ("xll", C.c_float),
                ("yll", C.c_float), ("cs", C.c_float), ("nodata", C.c_float)]


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.c_void_p
        L.orc_rule_of_thumb.restype = C.c_float
        L.orc_rule_of_thumb.argtypes = [C.c_int64, P, P, P]
        L.orc_h2.restype = C.c_double
        L.orc_h2.argtypes = [C.c_float]
        L.orc_mark_boundary.argtypes = [C.POINTER(OrcGrid), P, P]
        L.orc_dist2_boundary.argtypes = [C.c_int64, P, P, C.POINTER(OrcGrid), P, P]
        L.orc_sort_order.argtypes = [C.c_int64, P, P]
        L.orc_edge_weights.argtypes = [C.c_int64, P, P, P, C.c_float, P, C.POINTER(OrcGrid), P, P, P]
        L.orc_density.argtypes = [C.c_int64, P, P, P, P, P, C.c_float, C.POINTER(OrcGrid), P,
                                  C.c_int64, C.c_int64, C.c_int64, C.c_int64, P, P, C.c_int]
        L.orc_loo_loglik.restype = C.c_double
        L.orc_loo_loglik.argtypes = [C.c_int64, P, P, P, P, C.c_float, P, P]
        L.orc_loglik_at.restype = C.c_double
        L.orc_loglik_at.argtypes = [C.c_int64, P, P, P, P, C.POINTER(OrcGrid), P, C.c_float, P]
        L.orc_mle_fixed_bandwidth.restype = C.c_float
        L.orc_mle_fixed_bandwidth.argtypes = [C.c_int64, P, P, P, P, C.POINTER(OrcGrid), P, C.c_float,
                                              C.POINTER(C.c_int)]
        L.orc_point_density.argtypes = [C.c_int64, P, P, P, P, P, C.c_float, C.c_int, P, P]
        L.orc_adaptive_bandwidths.argtypes = [C.c_int64, P, C.c_float, C.c_float, P]
        L.orc_loglik_adaptive.restype = C.c_double
        L.orc_loglik_adaptive.argtypes = [C.c_int64, P, P, P, P, C.POINTER(OrcGrid), P, C.c_float, C.c_float, P]
        L.orc_adaptive_search.argtypes = [C.c_int64, P, P, P, P, C.POINTER(OrcGrid), P, C.c_float, P, P,
                                          C.POINTER(C.c_int)]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_threads.restype = C.c_int
        _lib = L
    return _lib


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def grid(ncols, nrows, xll, yll, cs, nodata=-9999.0) -> OrcGrid:
    return OrcGrid(int(ncols), int(nrows), float(xll), float(yll), float(cs), float(nodata))


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def threads() -> int:
    return lib().orc_get_threads()


def h2(h: float) -> float:
    return lib().orc_h2(h)


def rule_of_thumb(x, y, w=None) -> float:
    x, y, w = _f32(x), _f32(y), _f32(w)
    return float(lib().orc_rule_of_thumb(len(x), _p(x), _p(y), _p(w)))


def mark_boundary(g: OrcGrid, mask) -> np.ndarray:
    mask = _f32(mask).reshape(-1)
    out = np.zeros(mask.shape, np.uint8)
    lib().orc_mark_boundary(C.byref(g), _p(mask), _p(out))
    return out.reshape(g.nrows, g.ncols)


def dist2_boundary(x, y, g: OrcGrid, boundary) -> np.ndarray:
    x, y = _f32(x), _f32(y)
    b = np.ascontiguousarray(boundary, dtype=np.uint8).reshape(-1)
    out = np.zeros(len(x), np.float64)
    lib().orc_dist2_boundary(len(x), _p(x), _p(y), C.byref(g), _p(b), _p(out))
    return out


def sort_order(dist2) -> np.ndarray:
    d = _f64(dist2)
    out = np.zeros(len(d), np.int64)
    lib().orc_sort_order(len(d), _p(d), _p(out))
    return out


def edge_weights(x, y, h, dist2, g: OrcGrid, mask, hs=None):
    x, y, hs, d = _f32(x), _f32(y), _f32(hs), _f64(dist2)
    mask = _f32(mask).reshape(-1)
    out = np.zeros(len(x), np.float64)
    ev = C.c_int64(0)
    lib().orc_edge_weights(len(x), _p(x), _p(y), _p(hs), float(h), _p(d), C.byref(g), _p(mask),
                           _p(out), C.byref(ev))
    return out, ev.value


def density(x, y, w, ew, h, g: OrcGrid, mask=None, window=None, hs=None, brute=False):
    """Density on a window (r0, c0, nr, nc) of grid g (whole grid by default)."""
    x, y, w, ew, hs = _f32(x), _f32(y), _f32(w), _f64(ew), _f32(hs)
    m = None if mask is None else _f32(mask).reshape(-1)
    r0, c0, nr, nc = window if window is not None else (0, 0, g.nrows, g.ncols)
    out = np.zeros((nr, nc), np.float64)
    ev = C.c_int64(0)
    lib().orc_density(len(x), _p(x), _p(y), _p(w), _p(ew), _p(hs), float(h), C.byref(g), _p(m),
                      r0, c0, nr, nc, _p(out), C.byref(ev), int(bool(brute)))
    return out, ev.value


def loo_loglik(x, y, w, ew, h):
    x, y, w, ew = _f32(x), _f32(y), _f32(w), _f64(ew)
    loo = np.zeros(len(x), np.float64)
    ev = C.c_int64(0)
    ll = lib().orc_loo_loglik(len(x), _p(x), _p(y), _p(w), _p(ew), float(h), _p(loo), C.byref(ev))
    return float(ll), loo, ev.value


def loglik_at(x, y, w, dist2, g: OrcGrid, mask, h):
    x, y, w, d = _f32(x), _f32(y), _f32(w), _f64(dist2)
    m = _f32(mask).reshape(-1)
    ev = C.c_int64(0)
    ll = lib().orc_loglik_at(len(x), _p(x), _p(y), _p(w), _p(d), C.byref(g), _p(m), float(h), C.byref(ev))
    return float(ll), ev.value


def mle_fixed_bandwidth(x, y, w, dist2, g: OrcGrid, mask, h0):
    x, y, w, d = _f32(x), _f32(y), _f32(w), _f64(dist2)
    m = _f32(mask).reshape(-1)
    it = C.c_int(0)
    h = lib().orc_mle_fixed_bandwidth(len(x), _p(x), _p(y), _p(w), _p(d), C.byref(g), _p(m),
                                      float(h0), C.byref(it))
    return float(h), it.value


def point_density(x, y, w, ew, h, hs=None, self_term=True):
    x, y, w, ew, hs = _f32(x), _f32(y), _f32(w), _f64(ew), _f32(hs)
    out = np.zeros(len(x), np.float64)
    ev = C.c_int64(0)
    lib().orc_point_density(len(x), _p(x), _p(y), _p(w), _p(ew), _p(hs), float(h), int(bool(self_term)),
                            _p(out), C.byref(ev))
    return out, ev.value


def adaptive_bandwidths(den0, h, alpha):
    den0 = _f64(den0)
    hs = np.zeros(len(den0), np.float32)
    lib().orc_adaptive_bandwidths(len(den0), _p(den0), float(h), float(alpha), _p(hs))
    return hs


def loglik_adaptive(x, y, w, dist2, g, mask, h, alpha):
    x, y, w, d = _f32(x), _f32(y), _f32(w), _f64(dist2)
    m = None if mask is None else _f32(mask).reshape(-1)
    hs = np.zeros(len(x), np.float32)
    ll = lib().orc_loglik_adaptive(len(x), _p(x), _p(y), _p(w), _p(d), C.byref(g) if g is not None else None,
                                   _p(m), float(h), float(alpha), _p(hs))
    return float(ll), hs


def adaptive_search(x, y, w, dist2, g, mask, h0):
    """Hooke-Jeeves over (h, alpha) and the final per-point bandwidths;
    returns (h_opt, alpha_opt, Lmax, hs, iterations)."""
    x, y, w, d = _f32(x), _f32(y), _f32(w), _f64(dist2)
    m = None if mask is None else _f32(mask).reshape(-1)
    out3 = np.zeros(3, np.float32)
    hs = np.zeros(len(x), np.float32)
    it = C.c_int(0)
    lib().orc_adaptive_search(len(x), _p(x), _p(y), _p(w), _p(d), C.byref(g) if g is not None else None, _p(m),
                              float(h0), _p(out3), _p(hs), C.byref(it))
    return float(out3[0]), float(out3[1]), float(out3[2]), hs, it.value
