"""Many independent tessellations computed together (vd_batch_* C ABI).

Each member is a reference Tessellation (bounds, Algorithm3DGrid
resolution, walls of any kind, generators); the batch runs every member's
binning and clipping in shared persistent launches and keeps Lloyd steps on
the device.  Results per member equal what a standalone Tessellation with
the same inputs returns.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence

import numpy as np

from ._lib import FAST_LAYOUTS, VD_PREC_FP64, VD_PREC_MIXED, VoronoidError, load
from .tessellation import (BoundingBox, ConeGeometry, CylinderGeometry, PlaneGeometry, SphereGeometry,
                           TorusGeometry, Wall)


class _WallDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("id", C.c_int), ("a", C.c_double * 3), ("n", C.c_double * 3),
                ("r", C.c_double), ("r2", C.c_double), ("points", C.c_void_p), ("normals", C.c_void_p),
                ("nplanes", C.c_int)]


class _Walls:
    """vd_wall_desc array for a batch member or a request; keeps the
    polyhedron plane arrays it points at alive while it lives."""

    def __init__(self, walls: Sequence[Wall]):
        self.arr = (_WallDesc * max(len(walls), 1))()
        self.keep = []
        for k, w in enumerate(walls):
            g = w.geometry
            d = self.arr[k]
            d.id = w.id()
            if isinstance(g, PlaneGeometry):
                d.kind = 0
                d.a[:] = list(g.point)
                d.n[:] = list(g.normal)
            elif isinstance(g, SphereGeometry):
                d.kind = 1
                d.a[:] = list(g.center)
                d.r = g.radius
            elif isinstance(g, CylinderGeometry):
                d.kind = 2
                d.a[:] = list(g.center)
                d.n[:] = list(g.axis)
                d.r = g.radius
            elif isinstance(g, ConeGeometry):
                d.kind = 3
                d.a[:] = list(g.tip)
                d.n[:] = list(g.axis)
                d.r = g.angle
            elif isinstance(g, TorusGeometry):
                d.kind = 4
                d.a[:] = list(g.center)
                d.n[:] = list(g.axis)
                d.r = g.major_radius
                d.r2 = g.minor_radius
            else:
                d.kind = 5
                p = np.ascontiguousarray(g.points, np.float64)
                n = np.ascontiguousarray(g.normals, np.float64)
                self.keep += [p, n]
                d.points = p.ctypes.data
                d.normals = n.ctypes.data
                d.nplanes = len(p)


def _walls(walls: Sequence[Wall]) -> _Walls:
    return _Walls(walls)


class TessellationBatch:
    def __init__(self):
        self._L = load()
        h = C.c_void_p()
        self._chk(self._L.vd_batch_create(C.byref(h)), None)
        self._h = h
        self._n = 0

    def _chk(self, rc, h=...):
        if rc != 0:
            msg = self._L.vd_batch_last_error(self._h if h is ... else h)
            raise VoronoidError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.vd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, bounds: BoundingBox, grid: Sequence[int], generators, walls: Sequence[Wall] = ()) -> int:
        mn = np.asarray(bounds.min, np.float64)
        mx = np.asarray(bounds.max, np.float64)
        pts = np.ascontiguousarray(np.asarray(generators, np.float64).reshape(-1))
        n = pts.size // 3
        idx = C.c_int()
        wd = _walls(walls)
        d = C.POINTER(C.c_double)
        self._chk(self._L.vd_batch_add(self._h, mn.ctypes.data_as(d), mx.ctypes.data_as(d), int(grid[0]),
                                       int(grid[1]), int(grid[2]), C.cast(wd.arr, C.c_void_p), len(walls),
                                       pts.ctypes.data_as(d), n, C.byref(idx)))
        self._n += 1
        return idx.value

    def set_precision(self, precision: str):
        self._chk(self._L.vd_batch_set_precision(self._h, {"fp64": VD_PREC_FP64, "mixed": VD_PREC_MIXED}[precision]))

    def set_fast_layout(self, layout: str):
        """'slots' (default) or 'full': the first tier's polytope layout."""
        self._chk(self._L.vd_batch_set_fast_layout(self._h, FAST_LAYOUTS[layout]))

    def set_instrumentation(self, on: bool):
        self._chk(self._L.vd_batch_set_instrumentation(self._h, 1 if on else 0))

    def reset(self):
        """Drop the members so that the batch takes new ones (add, commit and
        calculate again); its device buffers are kept."""
        self._chk(self._L.vd_batch_reset(self._h))
        self._n = 0

    def commit(self):
        self._chk(self._L.vd_batch_commit(self._h))

    def calculate(self):
        self._chk(self._L.vd_batch_calculate(self._h))

    def lloyd(self, steps: int):
        self._chk(self._L.vd_batch_lloyd(self._h, int(steps)))

    def count_cells(self, index: int) -> int:
        n = C.c_size_t()
        self._chk(self._L.vd_batch_count_cells(self._h, int(index), C.byref(n)))
        return n.value

    def total_cells(self) -> int:
        n = C.c_size_t()
        self._chk(self._L.vd_batch_total_cells(self._h, C.byref(n)))
        return n.value

    def generators(self, index: int) -> np.ndarray:
        out = np.zeros(3 * self.count_cells(index), np.float64)
        self._chk(self._L.vd_batch_get_generators(self._h, int(index), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def summaries(self, index: int):
        n = self.count_cells(index)
        vol = np.zeros(n, np.float64)
        cen = np.zeros((n, 3), np.float64)
        nf = np.zeros(n, np.int32)
        self._chk(self._L.vd_batch_get_summaries(self._h, int(index), C.c_void_p(vol.ctypes.data),
                                                 C.c_void_p(cen.ctypes.data), C.c_void_p(nf.ctypes.data)))
        return vol, cen, nf

    def timing_ms(self) -> float:
        t = C.c_float()
        self._chk(self._L.vd_batch_timing(self._h, C.byref(t)))
        return t.value

    def counters(self) -> dict:
        out = (C.c_uint64 * 8)()
        self._chk(self._L.vd_batch_counters(self._h, out))
        names = ("candidates", "clips", "classified", "modifying", "intersections", "kept", "triangles", "offsets")
        return {k: int(v) for k, v in zip(names, out)}

    def stream(self) -> int:
        s = C.c_void_p()
        self._chk(self._L.vd_batch_stream(self._h, C.byref(s)))
        return s.value or 0
