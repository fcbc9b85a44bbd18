"""Python side of the serving loop (mgk_serve_* in the C ABI).

A Server owns a preparation thread and a worker thread, each with a device
context (requests are uploaded and indexed on the first while the second
runs the ticks); submit() queues a whole
fixed-h KDE request and returns a Ticket; wait() blocks until the request's
raster is in its host output array.  The arrays handed to submit() are kept
alive by the ticket until the request completes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._native import MgkError, MgkRequest, MgkResult, MgkServeInfo, lib
from .kde import Grid


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _host_raster(nrows, ncols):
    """A page-locked host raster when torch can provide one (device-to-host
    copies into it run at full link speed), else an ordinary array."""
    try:
        import torch
        return torch.empty((nrows, ncols), dtype=torch.float32, pin_memory=True).numpy()
    except Exception:  # noqa: BLE001 - no CUDA host allocator: pageable memory works too
        return np.empty((nrows, ncols), np.float32)


class Ticket:
    def __init__(self, tid, out, keep):
        self.id = tid
        self.out = out
        self._keep = keep


class Server:
    def __init__(self, device: int = 0, hbm_budget: int = 0, tile: int = 2048, max_active: int = 8):
        self._h = C.c_void_p()
        st = lib().mgk_serve_create(int(device), int(hbm_budget), int(tile), int(max_active), C.byref(self._h))
        if st != 0:
            raise MgkError(st, "mgk_serve_create failed")

    def submit(self, x, y, w, h: float, grid: Grid, mask=None, edge_grid: Grid | None = None, edge_mask=None,
               out=None) -> Ticket:
        x, y, w, mask, edge_mask = _f32(x), _f32(y), _f32(w), _f32(mask), _f32(edge_mask)
        if out is None:
            out = _host_raster(grid.nrows, grid.ncols)
        edge = edge_mask is not None
        req = MgkRequest(len(x), _p(x), _p(y), _p(w), float(h), grid.c(), _p(mask), int(edge),
                         edge_grid.c() if edge else Grid(1, 1, 0.0, 0.0, 1.0).c(), _p(edge_mask), _p(out))
        t = C.c_uint64()
        st = lib().mgk_serve_submit(self._h, C.byref(req), C.byref(t))
        if st != 0:
            raise MgkError(st, "mgk_serve_submit rejected the request")
        return Ticket(t.value, out, (x, y, w, mask, edge_mask))

    def wait(self, ticket: Ticket, timeout: float = 600.0):
        r = MgkResult()
        st = lib().mgk_serve_wait(self._h, ticket.id, float(timeout), C.byref(r))
        if st != 0:
            raise MgkError(st, "request failed or timed out")
        ticket._keep = None
        return ticket.out, {"evals": r.evals, "queue_ms": r.queue_ms, "run_ms": r.run_ms, "total_ms": r.total_ms}

    def poll(self, ticket: Ticket):
        done = C.c_int()
        r = MgkResult()
        st = lib().mgk_serve_poll(self._h, ticket.id, C.byref(done), C.byref(r))
        if st != 0:
            raise MgkError(st, "unknown ticket")
        if not done.value:
            return None
        if r.status != 0:
            raise MgkError(r.status, "request failed")
        ticket._keep = None
        return ticket.out, {"evals": r.evals, "queue_ms": r.queue_ms, "run_ms": r.run_ms, "total_ms": r.total_ms}

    def stats(self) -> dict:
        s = MgkServeInfo()
        lib().mgk_serve_stats(self._h, C.byref(s))
        return {k: int(getattr(s, k)) for k, _ in MgkServeInfo._fields_}

    def close(self):
        if self._h:
            lib().mgk_serve_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
