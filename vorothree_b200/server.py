"""Serving tessellations with continuous batching (vd_server_* C ABI).

Worker slots keep resident device buffers; requests are admitted FIFO by an
HBM budget as soon as a slot frees, and concurrent requests overlap on the
GPU.  A request's result equals a standalone Tessellation's.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from ._lib import VD_ESTATE, VD_PREC_FP64, VD_PREC_MIXED, VoronoidError, load
from .batch import _walls
from .tessellation import BoundingBox, Wall


class TessellationServer:
    def __init__(self, slots: int = 4, hbm_budget_bytes: int = 32 << 30, precision: str = "fp64"):
        self._L = load()
        h = C.c_void_p()
        rc = self._L.vd_server_create(int(slots), int(hbm_budget_bytes),
                                      {"fp64": VD_PREC_FP64, "mixed": VD_PREC_MIXED}[precision], C.byref(h))
        if rc != 0:
            raise VoronoidError(rc, self._L.vd_server_last_error(None).decode())
        self._h = h

    def _chk(self, rc):
        if rc != 0:
            msg = self._L.vd_server_last_error(self._h)
            raise VoronoidError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.vd_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, bounds: BoundingBox, grid: Sequence[int], generators, walls: Sequence[Wall] = ()) -> int:
        mn = np.asarray(bounds.min, np.float64)
        mx = np.asarray(bounds.max, np.float64)
        pts = np.ascontiguousarray(np.asarray(generators, np.float64).reshape(-1))
        wd = _walls(walls)
        t = C.c_uint64()
        d = C.POINTER(C.c_double)
        self._chk(self._L.vd_server_submit(self._h, mn.ctypes.data_as(d), mx.ctypes.data_as(d), int(grid[0]),
                                           int(grid[1]), int(grid[2]), C.cast(wd.arr, C.c_void_p), len(walls),
                                           pts.ctypes.data_as(d), pts.size // 3, C.byref(t)))
        return t.value

    def submit_text(self, bounds: BoundingBox, grid: Sequence[int], text, walls: Sequence[Wall] = ()) -> int:
        """submit() with the generators in the read_generators text format
        (``id x y z`` per line; str or UTF-8 bytes), parsed by the library."""
        mn = np.asarray(bounds.min, np.float64)
        mx = np.asarray(bounds.max, np.float64)
        data = text.encode("utf-8") if isinstance(text, str) else bytes(text)
        wd = _walls(walls)
        t = C.c_uint64()
        d = C.POINTER(C.c_double)
        self._chk(self._L.vd_server_submit_text(self._h, mn.ctypes.data_as(d), mx.ctypes.data_as(d), int(grid[0]),
                                                int(grid[1]), int(grid[2]), C.cast(wd.arr, C.c_void_p), len(walls),
                                                data, len(data), C.byref(t)))
        return t.value

    def wait(self, ticket: int):
        """(n_cells, latency_seconds) once the request is done."""
        n = C.c_size_t()
        lat = C.c_double()
        self._chk(self._L.vd_server_wait(self._h, C.c_uint64(ticket), C.byref(n), C.byref(lat)))
        return n.value, lat.value

    def take(self, ticket: int):
        """(volume[n], centroid[n,3], n_faces[n]); releases the request."""
        n, _ = self.wait(ticket)
        vol = np.zeros(n, np.float64)
        cen = np.zeros((n, 3), np.float64)
        nf = np.zeros(n, np.int32)
        self._chk(self._L.vd_server_take(self._h, C.c_uint64(ticket), C.c_void_p(vol.ctypes.data),
                                         C.c_void_p(cen.ctypes.data), C.c_void_p(nf.ctypes.data)))
        return vol, cen, nf

    def set_face_results(self, on: bool = True):
        """Requests submitted afterwards also return each cell's neighbour ids
        and face areas (take_faces)."""
        self._chk(self._L.vd_server_set_face_results(self._h, 1 if on else 0))

    def take_faces(self, ticket: int):
        """(volume, centroid, n_faces, offsets[n+1], neighbour ids, face areas)
        of a request submitted with face results; releases the request."""
        n, _ = self.wait(ticket)
        tot = C.c_int64()
        self._chk(self._L.vd_server_total_faces(self._h, C.c_uint64(ticket), C.byref(tot)))
        vol = np.zeros(n, np.float64)
        cen = np.zeros((n, 3), np.float64)
        nf = np.zeros(n, np.int32)
        off = np.zeros(n + 1, np.int64)
        ids = np.zeros(max(tot.value, 1), np.int32)
        ar = np.zeros(max(tot.value, 1), np.float64)
        vp = C.c_void_p
        self._chk(self._L.vd_server_take_faces(self._h, C.c_uint64(ticket), vp(vol.ctypes.data), vp(cen.ctypes.data),
                                               vp(nf.ctypes.data), vp(off.ctypes.data), vp(ids.ctypes.data),
                                               vp(ar.ctypes.data)))
        return vol, cen, nf, off, ids[:tot.value], ar[:tot.value]

    def cancel(self, ticket: int) -> bool:
        """Drop a request still in the queue (True); False when it has already
        started (it runs to completion)."""
        rc = self._L.vd_server_cancel(self._h, C.c_uint64(ticket))
        if rc == VD_ESTATE:
            return False
        self._chk(rc)
        return True

    def set_merging(self, max_members: int = 64, max_request: int = 65536, max_group: int = 1 << 20):
        """Merging of small requests (off by default): a slot
        that starts a request without face results of at most max_request
        generators also takes the run of such requests behind it in the queue
        (up to max_members, max_group generators in all, within the HBM budget)
        and computes them as one batch; max_members <= 1 turns it off."""
        self._chk(self._L.vd_server_set_merging(self._h, int(max_members), int(max_request), int(max_group)))

    def merge_stats(self) -> dict:
        """Merged batches run and the requests they served since reset_stats."""
        g = C.c_uint64()
        m = C.c_uint64()
        self._chk(self._L.vd_server_merge_stats(self._h, C.byref(g), C.byref(m)))
        return {"groups": g.value, "merged_requests": m.value}

    def concurrency(self) -> dict:
        """Requests on the GPU now, and the most at once since reset_stats."""
        run = C.c_int()
        peak = C.c_int()
        self._chk(self._L.vd_server_concurrency(self._h, C.byref(run), C.byref(peak)))
        return {"running": run.value, "peak_running": peak.value}

    def stats(self) -> dict:
        done = C.c_uint64()
        cells = C.c_uint64()
        p50 = C.c_double()
        p99 = C.c_double()
        peak = C.c_size_t()
        self._chk(self._L.vd_server_stats(self._h, C.byref(done), C.byref(cells), C.byref(p50), C.byref(p99),
                                          C.byref(peak)))
        return {"completed": done.value, "cells": cells.value, "p50_s": p50.value, "p99_s": p99.value,
                "peak_bytes": peak.value}

    def reset_stats(self):
        self._chk(self._L.vd_server_reset_stats(self._h))
