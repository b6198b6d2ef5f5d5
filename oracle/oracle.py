"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a plain-C restatement of the reference crate ``voronoid``'s
3D path (see vd_oracle.c for the file:line map).  Tests, the smoke check and
the benchmark's CPU-baseline leg use it as the checker; the product package
``vorothree_b200`` never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libvd_oracle.so")
_lib = None

NCOUNTERS = 8
COUNTER_NAMES = ("candidates", "clips", "classified", "modifying",
                 "intersections", "kept", "triangles", "offsets")


def build() -> str:
    """Compile the oracle with its Makefile (system gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    d3 = C.POINTER(C.c_double)
    vp = C.c_void_p
    L.vdo_create.restype = vp
    L.vdo_create.argtypes = [d3, d3, C.c_int, C.c_int, C.c_int]
    L.vdo_create_truncated.restype = vp
    L.vdo_create_truncated.argtypes = [d3, d3, C.c_int, C.c_int, C.c_int, C.c_int]
    L.vdo_table_exhausted.restype = C.c_size_t
    L.vdo_table_exhausted.argtypes = [vp]
    L.vdo_destroy.argtypes = [vp]
    L.vdo_add_wall_plane.argtypes = [vp, d3, d3, C.c_int]
    L.vdo_add_wall_sphere.argtypes = [vp, d3, C.c_double, C.c_int]
    L.vdo_add_wall_cylinder.argtypes = [vp, d3, d3, C.c_double, C.c_int]
    L.vdo_add_wall_cone.argtypes = [vp, d3, d3, C.c_double, C.c_int]
    L.vdo_add_wall_torus.argtypes = [vp, d3, d3, C.c_double, C.c_double, C.c_int]
    L.vdo_add_wall_polyhedron.argtypes = [vp, d3, d3, C.c_int, C.c_int]
    L.vdo_regular_polyhedron.argtypes = [C.c_int, d3, C.c_double, d3, d3]
    L.vdo_calculate_sealed.argtypes = [vp, C.c_int]
    L.vdo_prune_boundaries.argtypes = [vp]
    for nm in ("seal_log", "prune_log", "prune_pos_log"):
        getattr(L, f"vdo_{nm}_len").restype = C.c_size_t
        getattr(L, f"vdo_{nm}_len").argtypes = [vp]
    L.vdo_get_seal_log.argtypes = [vp, C.POINTER(C.c_int32)]
    L.vdo_get_prune_log.argtypes = [vp, C.POINTER(C.c_int32)]
    L.vdo_get_prune_pos_log.argtypes = [vp, d3]
    L.vdo_clear_walls.argtypes = [vp]
    L.vdo_set_generators.restype = C.c_size_t
    L.vdo_set_generators.argtypes = [vp, d3, C.c_size_t]
    L.vdo_set_generator.restype = None
    L.vdo_set_generator.argtypes = [vp, C.c_size_t, d3]
    L.vdo_random_generators.restype = C.c_size_t
    L.vdo_random_generators.argtypes = [vp, C.c_size_t, C.c_uint64]
    L.vdo_wall_contains_at.restype = C.c_int
    L.vdo_wall_contains_at.argtypes = [vp, C.c_int, d3]
    L.vdo_wall_cut_at.restype = C.c_int
    L.vdo_wall_cut_at.argtypes = [vp, C.c_int, d3, d3, d3]
    L.vdo_get_bins.restype = None
    L.vdo_get_bins.argtypes = [vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
    L.vdo_calculate.argtypes = [vp, C.c_int]
    L.vdo_calculate_range.argtypes = [vp, C.c_size_t, C.c_size_t, C.c_int]
    L.vdo_relax.argtypes = [vp]
    L.vdo_count_generators.restype = C.c_size_t
    L.vdo_count_generators.argtypes = [vp]
    L.vdo_count_cells.restype = C.c_size_t
    L.vdo_count_cells.argtypes = [vp]
    L.vdo_get_generators.argtypes = [vp, d3]
    L.vdo_search_order_len.restype = C.c_size_t
    L.vdo_search_order_len.argtypes = [vp]
    L.vdo_get_search_order.argtypes = [vp, C.POINTER(C.c_int32), d3]
    L.vdo_bin_index.restype = C.c_size_t
    L.vdo_bin_index.argtypes = [vp, C.c_double, C.c_double, C.c_double]
    L.vdo_get_summaries.argtypes = [vp, d3, d3, C.POINTER(C.c_int32)]
    L.vdo_total_faces.restype = C.c_int64
    L.vdo_total_faces.argtypes = [vp]
    L.vdo_get_neighbors.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
    L.vdo_get_face_areas.argtypes = [vp, C.POINTER(C.c_int64), d3]
    L.vdo_get_counters.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.vdo_get_cell.restype = vp
    L.vdo_get_cell.argtypes = [vp, C.c_size_t]
    L.vdo_cell_new.restype = vp
    L.vdo_cell_new.argtypes = [C.c_size_t, d3, d3]
    L.vdo_cell_clone.restype = vp
    L.vdo_cell_clone.argtypes = [vp]
    L.vdo_cell_free.argtypes = [vp]
    L.vdo_cell_clip.restype = C.c_int
    L.vdo_cell_clip.argtypes = [vp, d3, d3, C.c_int]
    for f in ("vdo_cell_num_vertices", "vdo_cell_num_faces", "vdo_cell_num_face_indices"):
        getattr(L, f).restype = C.c_int
        getattr(L, f).argtypes = [vp]
    L.vdo_cell_export.argtypes = [vp, d3, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_int32)]
    L.vdo_cell_volume.restype = C.c_double
    L.vdo_cell_volume.argtypes = [vp]
    L.vdo_cell_centroid.argtypes = [vp, d3]
    L.vdo_cell_face_area.restype = C.c_double
    L.vdo_cell_face_area.argtypes = [vp, C.c_size_t]
    L.vdo_cell_max_radius_sq.restype = C.c_double
    L.vdo_cell_max_radius_sq.argtypes = [vp, d3]
    L.vdo_cell_id.restype = C.c_size_t
    L.vdo_cell_id.argtypes = [vp]
    _lib = L
    return L


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


class OracleCell:
    """Cell3DFaces restated (cell_3d_faces.rs): owned or borrowed polytope."""

    def __init__(self, handle, owned: bool, keep=None):
        self._h = handle
        self._owned = owned
        self._keep = keep

    @classmethod
    def new(cls, id_: int, bmin, bmax) -> "OracleCell":
        _, pmn = _d(bmin)
        mn, pmn = _d(bmin)
        mx, pmx = _d(bmax)
        return cls(lib().vdo_cell_new(id_, pmn, pmx), True)

    def __del__(self):
        if getattr(self, "_owned", False) and self._h:
            lib().vdo_cell_free(self._h)
            self._h = None

    def clone(self) -> "OracleCell":
        return OracleCell(lib().vdo_cell_clone(self._h), True)

    def clip(self, point, normal, neighbor_id: int) -> bool:
        p, pp = _d(point)
        n, pn = _d(normal)
        return bool(lib().vdo_cell_clip(self._h, pp, pn, int(neighbor_id)))

    def id(self) -> int:
        return int(lib().vdo_cell_id(self._h))

    def export(self):
        L = lib()
        nv = L.vdo_cell_num_vertices(self._h)
        nf = L.vdo_cell_num_faces(self._h)
        nh = L.vdo_cell_num_face_indices(self._h)
        v = np.zeros(3 * nv, np.float64)
        fc = np.zeros(nf, np.uint32)
        fi = np.zeros(nh, np.uint32)
        fn = np.zeros(nf, np.int32)
        L.vdo_cell_export(self._h, v.ctypes.data_as(C.POINTER(C.c_double)),
                          fc.ctypes.data_as(C.POINTER(C.c_uint32)),
                          fi.ctypes.data_as(C.POINTER(C.c_uint32)),
                          fn.ctypes.data_as(C.POINTER(C.c_int32)))
        return v, fc, fi, fn

    def vertices(self):
        return self.export()[0]

    def face_counts(self):
        return self.export()[1]

    def face_indices(self):
        return self.export()[2]

    def face_neighbors(self):
        return self.export()[3]

    def is_empty(self) -> bool:
        return lib().vdo_cell_num_vertices(self._h) == 0

    def volume(self) -> float:
        return float(lib().vdo_cell_volume(self._h))

    def centroid(self):
        out = np.zeros(3, np.float64)
        lib().vdo_cell_centroid(self._h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def face_area(self, k: int) -> float:
        return float(lib().vdo_cell_face_area(self._h, int(k)))

    def max_radius_sq(self, center) -> float:
        c, pc = _d(center)
        return float(lib().vdo_cell_max_radius_sq(self._h, pc))


def regular_polyhedron(faces: int, center, radius: float):
    """(points, normals) of ConvexPolyhedronGeometry::new_* with `faces` faces
    (4, 6, 8, 12 or 20), restated in C."""
    c, pc = _d(center)
    pts = np.zeros(60, np.float64)
    nrm = np.zeros(60, np.float64)
    m = lib().vdo_regular_polyhedron(int(faces), pc, float(radius), pts.ctypes.data_as(C.POINTER(C.c_double)),
                                     nrm.ctypes.data_as(C.POINTER(C.c_double)))
    if m < 0:
        raise ValueError(faces)
    return pts[:3 * m].reshape(-1, 3), nrm[:3 * m].reshape(-1, 3)


class OracleTessellation:
    """Tessellation<3, Cell3DFaces, Algorithm3DGrid> restated on the CPU."""

    def __init__(self, bmin, bmax, nx: int, ny: int, nz: int, order_k: int = 0):
        """order_k > 0 truncates the search order to offsets of at most
        order_k bins per axis (grids whose complete table does not fit in
        memory); calculate() then raises if a cell's walk ran off it."""
        mn, pmn = _d(bmin)
        mx, pmx = _d(bmax)
        self._h = lib().vdo_create_truncated(pmn, pmx, int(nx), int(ny), int(nz), int(order_k))
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        if not self._h:
            raise ValueError("invalid grid resolution")

    def __del__(self):
        if getattr(self, "_h", None):
            lib().vdo_destroy(self._h)
            self._h = None

    def add_wall_plane(self, point, normal, wall_id: int):
        p, pp = _d(point)
        n, pn = _d(normal)
        if lib().vdo_add_wall_plane(self._h, pp, pn, int(wall_id)) != 0:
            raise ValueError("Wall ID must be <= -1000")

    def add_wall_sphere(self, center, radius: float, wall_id: int):
        c, pc = _d(center)
        if lib().vdo_add_wall_sphere(self._h, pc, float(radius), int(wall_id)) != 0:
            raise ValueError("Wall ID must be <= -1000")

    def add_wall_cylinder(self, center, axis, radius: float, wall_id: int):
        c, pc = _d(center)
        a, pa = _d(axis)
        if lib().vdo_add_wall_cylinder(self._h, pc, pa, float(radius), int(wall_id)) != 0:
            raise ValueError("Wall ID must be <= -1000")

    def add_wall_cone(self, tip, axis, angle: float, wall_id: int):
        c, pc = _d(tip)
        a, pa = _d(axis)
        if lib().vdo_add_wall_cone(self._h, pc, pa, float(angle), int(wall_id)) != 0:
            raise ValueError("Wall ID must be <= -1000")

    def add_wall_torus(self, center, axis, major: float, minor: float, wall_id: int):
        c, pc = _d(center)
        a, pa = _d(axis)
        if lib().vdo_add_wall_torus(self._h, pc, pa, float(major), float(minor), int(wall_id)) != 0:
            raise ValueError("Wall ID must be <= -1000")

    def add_wall_polyhedron(self, points, normals, wall_id: int):
        p, pp = _d(np.asarray(points, np.float64).reshape(-1))
        n, pn = _d(np.asarray(normals, np.float64).reshape(-1))
        if lib().vdo_add_wall_polyhedron(self._h, pp, pn, p.size // 3, int(wall_id)) != 0:
            raise ValueError("bad polyhedron wall")

    def clear_walls(self):
        lib().vdo_clear_walls(self._h)

    def set_generators(self, xyz) -> int:
        a, pa = _d(np.asarray(xyz, np.float64).reshape(-1))
        return int(lib().vdo_set_generators(self._h, pa, a.size // 3))

    def set_generator(self, index: int, xyz):
        a, pa = _d(np.asarray(xyz, np.float64).reshape(3))
        lib().vdo_set_generator(self._h, int(index), pa)

    def calculate(self, nthreads: int = 0):
        lib().vdo_calculate(self._h, int(nthreads))
        self._check_table()

    def _check_table(self):
        n = int(lib().vdo_table_exhausted(self._h))
        if n:
            raise RuntimeError(f"{n} cells walked off the truncated search order: use a larger order_k")

    def calculate_range(self, begin: int, end: int, nthreads: int = 0):
        lib().vdo_calculate_range(self._h, int(begin), int(end), int(nthreads))

    def calculate_sealed(self, nthreads: int = 0):
        lib().vdo_calculate_sealed(self._h, int(nthreads))

    def prune_boundaries(self):
        lib().vdo_prune_boundaries(self._h)

    def seal_log(self):
        n = int(lib().vdo_seal_log_len(self._h))
        out = np.zeros(max(n, 1), np.int32)
        lib().vdo_get_seal_log(self._h, out.ctypes.data_as(C.POINTER(C.c_int32)))
        return out[:n]

    def prune_log(self):
        n = int(lib().vdo_prune_log_len(self._h))
        out = np.zeros(max(n, 1), np.int32)
        lib().vdo_get_prune_log(self._h, out.ctypes.data_as(C.POINTER(C.c_int32)))
        return out[:n]

    def prune_pos_log(self):
        n = int(lib().vdo_prune_pos_log_len(self._h))
        out = np.zeros(max(n, 1), np.float64)
        lib().vdo_get_prune_pos_log(self._h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out[:n]

    def relax(self):
        lib().vdo_relax(self._h)

    def count_generators(self) -> int:
        return int(lib().vdo_count_generators(self._h))

    def count_cells(self) -> int:
        return int(lib().vdo_count_cells(self._h))

    def generators(self):
        n = self.count_generators()
        out = np.zeros(3 * n, np.float64)
        lib().vdo_get_generators(self._h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def random_generators(self, count: int, seed: int) -> int:
        return int(lib().vdo_random_generators(self._h, int(count), int(seed)))

    def wall_contains(self, w: int, point) -> bool:
        a, pa = _d(np.asarray(point, np.float64).reshape(3))
        return bool(lib().vdo_wall_contains_at(self._h, int(w), pa))

    def wall_cut(self, w: int, generator):
        """[(point, normal), ...] wall w emits for the generator."""
        a, pa = _d(np.asarray(generator, np.float64).reshape(3))
        p = np.zeros(3 * 256, np.float64)
        n = np.zeros(3 * 256, np.float64)
        k = lib().vdo_wall_cut_at(self._h, int(w), pa, p.ctypes.data_as(C.POINTER(C.c_double)),
                                  n.ctypes.data_as(C.POINTER(C.c_double)))
        return [(p[3 * q:3 * q + 3].copy(), n[3 * q:3 * q + 3].copy()) for q in range(k)]

    def bins(self):
        """grid_bins as a list of id lists, in visit order."""
        start = np.zeros(self.nx * self.ny * self.nz + 1, np.uint64)
        mem = np.zeros(max(self.count_generators(), 1), np.uint64)
        lib().vdo_get_bins(self._h, start.ctypes.data_as(C.POINTER(C.c_size_t)),
                           mem.ctypes.data_as(C.POINTER(C.c_size_t)))
        return [mem[start[b]:start[b + 1]].tolist() for b in range(len(start) - 1)]

    def bin_index(self, x, y, z) -> int:
        return int(lib().vdo_bin_index(self._h, x, y, z))

    def search_order(self):
        n = int(lib().vdo_search_order_len(self._h))
        d = np.zeros(3 * n, np.int32)
        m = np.zeros(n, np.float64)
        lib().vdo_get_search_order(self._h, d.ctypes.data_as(C.POINTER(C.c_int32)),
                                   m.ctypes.data_as(C.POINTER(C.c_double)))
        return d.reshape(-1, 3), m

    def summaries(self):
        n = self.count_cells()
        vol = np.zeros(n, np.float64)
        cen = np.zeros(3 * n, np.float64)
        nf = np.zeros(n, np.int32)
        lib().vdo_get_summaries(self._h, vol.ctypes.data_as(C.POINTER(C.c_double)),
                                cen.ctypes.data_as(C.POINTER(C.c_double)),
                                nf.ctypes.data_as(C.POINTER(C.c_int32)))
        return vol, cen.reshape(-1, 3), nf

    def neighbors(self):
        n = self.count_cells()
        tot = int(lib().vdo_total_faces(self._h))
        off = np.zeros(n + 1, np.int64)
        ids = np.zeros(max(tot, 1), np.int32)
        lib().vdo_get_neighbors(self._h, off.ctypes.data_as(C.POINTER(C.c_int64)),
                                ids.ctypes.data_as(C.POINTER(C.c_int32)))
        return off, ids[:tot]

    def face_areas(self):
        n = self.count_cells()
        tot = int(lib().vdo_total_faces(self._h))
        off = np.zeros(n + 1, np.int64)
        ar = np.zeros(max(tot, 1), np.float64)
        lib().vdo_get_face_areas(self._h, off.ctypes.data_as(C.POINTER(C.c_int64)),
                                 ar.ctypes.data_as(C.POINTER(C.c_double)))
        return off, ar[:tot]

    def counters(self) -> dict:
        out = np.zeros(NCOUNTERS, np.uint64)
        lib().vdo_get_counters(self._h, out.ctypes.data_as(C.POINTER(C.c_uint64)))
        return {k: int(v) for k, v in zip(COUNTER_NAMES, out)}

    def get_cell(self, i: int) -> OracleCell:
        h = lib().vdo_get_cell(self._h, int(i))
        if not h:
            raise IndexError(i)
        return OracleCell(h, owned=False, keep=self)
