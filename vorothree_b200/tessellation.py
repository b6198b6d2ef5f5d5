"""Python mirror of the reference crate's 3D API, backed by the CUDA library.

Names, argument meanings and error behaviour follow the reference crate
``voronoid``:

* ``BoundingBox`` / ``box_side``         -- src/bounds/mod.rs:3-22
* ``Algorithm3DGrid``                   -- src/algorithm/algo_3d_grid.rs:10-95
* ``Wall``, ``WALL_ID_MAX``             -- src/wall/mod.rs:8-49 (id > -1000 is an error)
* ``PlaneGeometry``, ``SphereGeometry`` -- src/wall/wall_3d.rs:8-101
* ``CylinderGeometry``, ``ConeGeometry``, ``TorusGeometry``,
  ``ConvexPolyhedronGeometry``          -- src/wall/wall_3d.rs:107-365, 462-708
* ``Cell3DFaces``                       -- src/cell/cell_3d_faces.rs:22-270
* ``Tessellation``                      -- src/tessellation.rs:13-527

Every computation runs on the GPU through the C ABI; results come back as
numpy arrays.
"""
from __future__ import annotations

import ctypes as C
import os
import math
from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence

import numpy as np

from ._lib import FAST_LAYOUTS, VD_PREC_FP64, VD_PREC_MIXED, Tuning, check, load

WALL_ID_MAX = -1000


def box_side(axis: int, is_max: bool) -> int:
    """Id of a bounding-box face: x- -1, x+ -2, y- -3, y+ -4, z- -5, z+ -6."""
    return -1 - (axis * 2 + (1 if is_max else 0))


@dataclass
class BoundingBox:
    min: Sequence[float]
    max: Sequence[float]

    def __post_init__(self):
        self.min = [float(v) for v in self.min]
        self.max = [float(v) for v in self.max]


class Algorithm3DGrid:
    """Uniform bin grid with a shell-ordered neighbour walk (built on device)."""

    def __init__(self, nx: int, ny: int, nz: int, bounds: Optional[BoundingBox] = None):
        if nx <= 0 or ny <= 0 or nz <= 0:
            raise ValueError("grid resolution must be positive")
        self.grid_res_x, self.grid_res_y, self.grid_res_z = int(nx), int(ny), int(nz)
        self.bounds = bounds

    @classmethod
    def new(cls, nx: int, ny: int, nz: int, bounds: Optional[BoundingBox] = None) -> "Algorithm3DGrid":
        """Algorithm3DGrid::new (algo_3d_grid.rs:47-95)."""
        return cls(nx, ny, nz, bounds)

    def get_bin_index(self, x: float, y: float, z: float, bounds: Optional[BoundingBox] = None) -> int:
        """Algorithm3DGrid::get_bin_index (algo_3d_grid.rs:97-107): the bin
        of a point, x fastest, coordinates clamped into the grid."""
        b = bounds if bounds is not None else self.bounds
        if b is None:
            raise ValueError("get_bin_index needs the grid's bounds")
        L = load()
        mn = np.asarray(b.min, np.float64)
        mx = np.asarray(b.max, np.float64)
        p = np.asarray([x, y, z], np.float64)
        out = C.c_size_t()
        check(L.vd_grid_bin_index(_dp(mn), _dp(mx), self.grid_res_x, self.grid_res_y, self.grid_res_z, _dp(p),
                                  C.byref(out)))
        return out.value


class _WallQueries:
    """WallGeometry::contains / cut (wall_3d.rs) on the host, through the same
    functions the kernels use, so they agree with calculate() bit for bit."""

    def _desc(self):
        from .batch import _walls
        return _walls([Wall(WALL_ID_MAX, self)])

    def contains(self, point: Sequence[float]) -> bool:
        L = load()
        d = self._desc()
        p = np.asarray(point, np.float64).reshape(3)
        inside = C.c_int()
        check(L.vd_wall_contains(C.cast(d.arr, C.c_void_p), _dp(p), C.byref(inside)))
        return bool(inside.value)

    def cut(self, generator: Sequence[float], callback: Callable[[np.ndarray, np.ndarray], object]) -> None:
        """Calls callback(point, normal) for each plane the wall emits for
        `generator`, in order (normal pointing out of the valid region)."""
        L = load()
        d = self._desc()
        g = np.asarray(generator, np.float64).reshape(3)
        n = C.c_int()
        check(L.vd_wall_cut(C.cast(d.arr, C.c_void_p), _dp(g), None, None, 0, C.byref(n)))
        k = n.value
        pts = np.zeros(3 * max(k, 1), np.float64)
        nrm = np.zeros(3 * max(k, 1), np.float64)
        check(L.vd_wall_cut(C.cast(d.arr, C.c_void_p), _dp(g), _dp(pts), _dp(nrm), k, C.byref(n)))
        for q in range(k):
            callback(pts[3 * q:3 * q + 3].copy(), nrm[3 * q:3 * q + 3].copy())


class PlaneGeometry(_WallQueries):
    """Plane wall; ``normal`` points into the valid region and is normalised."""

    def __init__(self, point: Sequence[float], normal: Sequence[float]):
        self.point = [float(v) for v in point]
        self.normal = [float(v) for v in normal]

    def is_planar(self) -> bool:
        return True


class SphereGeometry(_WallQueries):
    """Spherical wall; the valid region is inside."""

    def __init__(self, center: Sequence[float], radius: float):
        self.center = [float(v) for v in center]
        self.radius = float(radius)

    def is_planar(self) -> bool:
        return False


class CylinderGeometry(_WallQueries):
    """Infinite cylinder wall (wall_3d.rs:107-174); the valid region is inside.
    ``axis`` is normalised on the device side as the reference's constructor does."""

    def __init__(self, center: Sequence[float], axis: Sequence[float], radius: float):
        self.center = [float(v) for v in center]
        self.axis = [float(v) for v in axis]
        self.radius = float(radius)

    def is_planar(self) -> bool:
        return False


class ConeGeometry(_WallQueries):
    """Infinite cone wall (wall_3d.rs:177-262): apex ``tip``, ``axis`` pointing
    into the cone, half-angle ``angle`` in radians; the valid region is inside."""

    def __init__(self, tip: Sequence[float], axis: Sequence[float], angle: float):
        self.tip = [float(v) for v in tip]
        self.axis = [float(v) for v in axis]
        self.angle = float(angle)

    def is_planar(self) -> bool:
        return False


class TorusGeometry(_WallQueries):
    """Torus wall (wall_3d.rs:265-365); the valid region is inside the tube."""

    def __init__(self, center: Sequence[float], axis: Sequence[float], major_radius: float,
                 minor_radius: float):
        self.center = [float(v) for v in center]
        self.axis = [float(v) for v in axis]
        self.major_radius = float(major_radius)
        self.minor_radius = float(minor_radius)

    def is_planar(self) -> bool:
        return False


class ConvexPolyhedronGeometry(_WallQueries):
    """Convex polyhedron wall (wall_3d.rs:462-708): the intersection of the
    half-spaces behind planes (point, normal pointing OUT of the valid
    region).  The ``new_*`` constructors build the regular solids exactly as
    the reference's do (same arithmetic, in IEEE double)."""

    def __init__(self, points, normals):
        p = np.asarray(points, np.float64).reshape(-1)
        n = np.asarray(normals, np.float64).reshape(-1)
        if p.size != n.size or p.size % 3 != 0:
            raise ValueError("Points and normals must have same length and be multiple of 3")
        self.points = p.reshape(-1, 3)
        self.normals = n.reshape(-1, 3)

    def is_planar(self) -> bool:
        return True

    @classmethod
    def _regular(cls, center, base, dist, normalise=True):
        pts, nrm = [], []
        for b in base:
            nx, ny, nz = float(b[0]), float(b[1]), float(b[2])
            if normalise:
                ln = math.sqrt(nx * nx + ny * ny + nz * nz)
                nx, ny, nz = nx / ln, ny / ln, nz / ln
            nrm.append([nx, ny, nz])
            pts.append([center[0] + nx * dist, center[1] + ny * dist, center[2] + nz * dist])
        return cls(pts, nrm)

    @classmethod
    def new_tetrahedron(cls, center, radius: float):
        base = [[-1.0, -1.0, -1.0], [-1.0, 1.0, 1.0], [1.0, -1.0, 1.0], [1.0, 1.0, -1.0]]
        return cls._regular([float(c) for c in center], base, radius / 3.0)

    @classmethod
    def new_hexahedron(cls, center, radius: float):
        base = [[1.0, 0.0, 0.0], [-1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, -1.0, 0.0], [0.0, 0.0, 1.0],
                [0.0, 0.0, -1.0]]
        return cls._regular([float(c) for c in center], base, radius / math.sqrt(3.0), normalise=False)

    @classmethod
    def new_octahedron(cls, center, radius: float):
        base = [[x, y, z] for x in (-1.0, 1.0) for y in (-1.0, 1.0) for z in (-1.0, 1.0)]
        return cls._regular([float(c) for c in center], base, radius / math.sqrt(3.0))

    @classmethod
    def new_dodecahedron(cls, center, radius: float):
        phi = (1.0 + math.sqrt(5.0)) / 2.0
        xi = math.sqrt((5.0 + 2.0 * math.sqrt(5.0)) / 15.0)
        base = [[0.0, phi, 1.0], [0.0, -phi, 1.0], [0.0, phi, -1.0], [0.0, -phi, -1.0],
                [1.0, 0.0, phi], [1.0, 0.0, -phi], [-1.0, 0.0, phi], [-1.0, 0.0, -phi],
                [phi, 1.0, 0.0], [phi, -1.0, 0.0], [-phi, 1.0, 0.0], [-phi, -1.0, 0.0]]
        return cls._regular([float(c) for c in center], base, radius * xi)

    @classmethod
    def new_icosahedron(cls, center, radius: float):
        phi = (1.0 + math.sqrt(5.0)) / 2.0
        xi = math.sqrt((5.0 + 2.0 * math.sqrt(5.0)) / 15.0)
        ip = 1.0 / phi
        base = [[x, y, z] for x in (-1.0, 1.0) for y in (-1.0, 1.0) for z in (-1.0, 1.0)]
        base += [[0.0, y * phi, z * ip] for y in (-1.0, 1.0) for z in (-1.0, 1.0)]
        base += [[x * ip, 0.0, z * phi] for x in (-1.0, 1.0) for z in (-1.0, 1.0)]
        base += [[x * phi, y * ip, 0.0] for x in (-1.0, 1.0) for y in (-1.0, 1.0)]
        return cls._regular([float(c) for c in center], base, radius * xi)


WALL_GEOMETRIES = (PlaneGeometry, SphereGeometry, CylinderGeometry, ConeGeometry, TorusGeometry,
                   ConvexPolyhedronGeometry)


class Wall:
    """A wall geometry with an id <= WALL_ID_MAX (the reference panics otherwise)."""

    def __init__(self, id: int, geometry):
        if id > WALL_ID_MAX:
            raise ValueError(f"Wall ID must be <= {WALL_ID_MAX}")
        if not isinstance(geometry, WALL_GEOMETRIES):
            raise TypeError("unsupported wall geometry")
        self._id = int(id)
        self.geometry = geometry

    def id(self) -> int:
        return self._id

    def is_planar(self) -> bool:
        return self.geometry.is_planar()

    @classmethod
    def new(cls, id: int, geometry) -> "Wall":
        """Wall::new (wall/mod.rs:24-32)."""
        return cls(id, geometry)

    def contains(self, point: Sequence[float]) -> bool:
        """Wall::contains (wall/mod.rs:38-40)."""
        return self.geometry.contains(point)

    def cut(self, generator: Sequence[float], callback) -> None:
        """Wall::cut (wall/mod.rs:42-44)."""
        self.geometry.cut(generator, callback)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _vp(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


class Cell3DFaces:
    """Cell3DFaces (cell_3d_faces.rs:22-270), the reference's 3D cell type.

    Two ways to get one:

    * ``Tessellation.get_cell(i)``: the computed cell i of a tessellation,
      with the volume, centroid and face areas the GPU computed for it;
    * ``Cell3DFaces.new(id, bounds)``: the box cell (cell_3d_faces.rs:37-74),
      held in device memory and clipped call by call like the reference's
      (``clip`` = Cell::clip / clip_with_scratch, cell_3d_faces.rs:288-503).

    A computed cell moves to the device on its first ``clip``.  Every clip and
    every measure runs on the GPU (the tessellation kernels' warp routines);
    the accessors return copies of the device polytope.
    """

    def __init__(self, id: int, vertices, face_counts, face_indices, face_neighbors,
                 volume: Optional[float] = None, centroid=None, face_areas=None):
        self._id = int(id)
        self._h = None
        self._L = None
        self._set(vertices, face_counts, face_indices, face_neighbors, volume, centroid, face_areas)

    def _set(self, vertices, face_counts, face_indices, face_neighbors, volume, centroid, face_areas):
        self._vertices = np.asarray(vertices, np.float64)
        self._face_counts = np.asarray(face_counts, np.uint32)
        self._face_indices = np.asarray(face_indices, np.uint32)
        self._face_neighbors = np.asarray(face_neighbors, np.int32)
        self._volume = None if volume is None else float(volume)
        self._centroid = None if centroid is None else np.asarray(centroid, np.float64)
        self._face_areas = None if face_areas is None else np.asarray(face_areas, np.float64)
        self._stale = False

    @classmethod
    def new(cls, id: int, bounds: BoundingBox) -> "Cell3DFaces":
        """Cell3DFaces::new(id, bounds): the box, on the device."""
        L = load()
        h = C.c_void_p()
        lo = np.asarray(bounds.min, np.float64)
        hi = np.asarray(bounds.max, np.float64)
        rc = L.vd_cell_create_box(int(id), _dp(lo), _dp(hi), C.byref(h))
        cls._cell_check(L, rc, None)
        c = cls.__new__(cls)
        c._id = int(id)
        c._set([], [], [], [], None, None, None)
        c._L = L
        c._h = h
        c._stale = True
        return c

    @staticmethod
    def _cell_check(L, rc, h):
        if rc != 0:
            from ._lib import VoronoidError
            msg = L.vd_cell_last_error(h)
            raise VoronoidError(rc, msg.decode() if msg else "")

    def _device(self):
        """The device handle, uploading this cell's polytope on first use."""
        if self._h is not None:
            return self._h
        L = load()
        h = C.c_void_p()
        v = np.ascontiguousarray(self._vertices, np.float64)
        fc = np.ascontiguousarray(self._face_counts, np.uint32)
        fi = np.ascontiguousarray(self._face_indices, np.uint32)
        fn = np.ascontiguousarray(self._face_neighbors, np.int32)
        rc = L.vd_cell_create(self._id, v.size // 3, fc.size, _vp(v), _vp(fc), _vp(fi), _vp(fn), C.byref(h))
        self._cell_check(L, rc, None)
        self._L, self._h = L, h
        return h

    def _sync(self):
        """Refresh the host copies from the device after a clip."""
        if not self._stale:
            return
        L, h = self._L, self._h
        nv, nf, nh = C.c_int32(), C.c_int32(), C.c_int32()
        self._cell_check(L, L.vd_cell_get(h, C.byref(nv), C.byref(nf), C.byref(nh), None, None, None, None), h)
        v = np.zeros(3 * max(nv.value, 1), np.float64)
        fc = np.zeros(max(nf.value, 1), np.uint32)
        fi = np.zeros(max(nh.value, 1), np.uint32)
        fn = np.zeros(max(nf.value, 1), np.int32)
        self._cell_check(L, L.vd_cell_get(h, C.byref(nv), C.byref(nf), C.byref(nh), _vp(v), _vp(fc), _vp(fi),
                                          _vp(fn)), h)
        vol = C.c_double()
        cen = np.zeros(3, np.float64)
        nfo = C.c_int32()
        ar = np.zeros(max(nf.value, 1), np.float64)
        self._cell_check(L, L.vd_cell_measure(h, C.byref(vol), _dp(cen), C.byref(nfo), _vp(ar), None), h)
        self._set(v[:3 * nv.value], fc[:nf.value], fi[:nh.value], fn[:nf.value], vol.value, cen, ar[:nf.value])

    def close(self):
        if self._h is not None:
            self._L.vd_cell_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- Cell trait (cell/mod.rs:8-43) ---------------------------------
    def clip(self, point: Sequence[float], normal: Sequence[float], neighbor_id: int,
             generator: Optional[Sequence[float]] = None):
        """Clip by the plane through `point` with `normal` (the kept side is
        (v - point).normal <= 1e-9); returns (modified, new max radius^2 from
        `generator`, 0 without one), like Cell::clip."""
        h = self._device()
        self._sync()
        p = np.asarray(point, np.float64)
        n = np.asarray(normal, np.float64)
        g = None if generator is None else np.asarray(generator, np.float64)
        mod = C.c_int()
        r2 = C.c_double()
        self._cell_check(self._L, self._L.vd_cell_clip(h, _dp(p), _dp(n), int(neighbor_id),
                                                       None if g is None else _dp(g), C.byref(mod),
                                                       C.byref(r2)), h)
        self._stale = True
        return bool(mod.value), r2.value

    def clip_with_scratch(self, point: Sequence[float], normal: Sequence[float], neighbor_id: int, scratch=None,
                          generator: Optional[Sequence[float]] = None):
        """Cell3DFaces::clip_with_scratch (cell_3d_faces.rs:288-503): clip();
        the scratch space lives on the device, so `scratch` is not used."""
        return self.clip(point, normal, neighbor_id, generator)

    def max_radius_sq(self, center: Sequence[float]) -> float:
        h = self._device()
        c = np.asarray(center, np.float64)
        out = C.c_double()
        self._cell_check(self._L, self._L.vd_cell_max_radius_sq(h, _dp(c), C.byref(out)), h)
        return out.value

    def _measured(self):
        if self._volume is None:
            self._device()
            self._stale = True
        self._sync()

    # ---- accessors (cell_3d_faces.rs:76-104, 255-269) -------------------
    def id(self) -> int:
        return self._id

    def vertices(self) -> np.ndarray:
        self._sync()
        return self._vertices.copy()

    def face_counts(self) -> np.ndarray:
        self._sync()
        return self._face_counts.copy()

    def face_indices(self) -> np.ndarray:
        self._sync()
        return self._face_indices.copy()

    def face_neighbors(self) -> np.ndarray:
        self._sync()
        return self._face_neighbors.copy()

    def neighbors(self) -> np.ndarray:
        self._sync()
        return self._face_neighbors

    def faces(self) -> List[List[int]]:
        self._sync()
        out, off = [], 0
        for c in self._face_counts:
            out.append([int(v) for v in self._face_indices[off:off + c]])
            off += int(c)
        return out

    def is_empty(self) -> bool:
        self._sync()
        return self._vertices.size == 0

    def shared_vertices(self, neighbor_a: int, neighbor_b: int) -> np.ndarray:
        """Cell::shared_vertices (cell_3d_faces.rs:537-565): the vertices on
        both the face(s) of neighbour a and those of neighbour b, flat xyz."""
        self._sync()
        a, b = [], []
        for f, face in enumerate(self.faces()):
            nb = int(self._face_neighbors[f])
            for lst, want in ((a, neighbor_a), (b, neighbor_b)):
                if nb == want:
                    lst.extend(v for v in face if v not in lst)
        keep = [v for v in a if v in b]
        return self._vertices.reshape(-1, 3)[keep].reshape(-1).copy()

    # ---- measures (cell_3d_faces.rs:106-254) ----------------------------
    def volume(self) -> float:
        self._measured()
        return self._volume

    def centroid(self) -> np.ndarray:
        self._measured()
        return self._centroid.copy()

    def face_area(self, face_index: int) -> float:
        self._measured()
        if face_index >= self._face_areas.size:
            return 0.0
        return float(self._face_areas[face_index])


def parse_generators(text) -> np.ndarray:
    """The reader of Tessellation::read_generators (tessellation.rs:153-171),
    host only: an (n, 3) array of the points in ``text`` (str or UTF-8 bytes),
    before any wall filter."""
    L = load()
    data = text.encode("utf-8") if isinstance(text, str) else bytes(text)
    n = C.c_size_t()
    check(L.vd_parse_generators(data, len(data), None, 0, C.byref(n)))
    out = np.zeros(3 * max(n.value, 1), np.float64)
    check(L.vd_parse_generators(data, len(data), _dp(out), n.value, C.byref(n)))
    return out[:3 * n.value].reshape(-1, 3)


class Tessellation:
    """Tessellation<3, Cell3DFaces, Algorithm3DGrid> on one GPU."""

    def __init__(self, bounds: BoundingBox, algorithm: Algorithm3DGrid):
        self.bounds = bounds
        self.algorithm = algorithm
        self.walls: List[Wall] = []
        self._L = load()
        h = C.c_void_p()
        mn = np.asarray(bounds.min, np.float64)
        mx = np.asarray(bounds.max, np.float64)
        check(self._L.vd_tess_create(_dp(mn), _dp(mx), algorithm.grid_res_x, algorithm.grid_res_y,
                                     algorithm.grid_res_z, C.byref(h)))
        self._h = h

    @classmethod
    def new(cls, bounds: BoundingBox, algorithm: Algorithm3DGrid) -> "Tessellation":
        """Tessellation::new (tessellation.rs:25-39)."""
        return cls(bounds, algorithm)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.vd_tess_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc: int):
        check(rc, self._h)

    # ---- configuration -------------------------------------------------
    def set_precision(self, precision: str):
        """'fp64' (default, bitwise the reference's arithmetic) or 'mixed'."""
        code = {"fp64": VD_PREC_FP64, "mixed": VD_PREC_MIXED}[precision]
        self._ck(self._L.vd_tess_set_precision(self._h, code))

    def set_tuning(self, tuning: dict):
        """Launch choices that change no result (the autotuner's): any of
        fast_layout ('slots' / 'full'), fast_blocks_per_sm (5, 6, 7),
        huge_direct_max, huge_blocks_max, huge_narrow_max, noop_run; keys left
        out keep their current value."""
        cur = self.get_tuning()
        cur.update(tuning)
        k = Tuning(FAST_LAYOUTS[cur["fast_layout"]], int(cur["fast_blocks_per_sm"]), int(cur["huge_direct_max"]),
                   int(cur["huge_blocks_max"]), int(cur["huge_narrow_max"]), int(cur["noop_run"]))
        self._ck(self._L.vd_tess_set_tuning(self._h, C.byref(k)))

    def get_tuning(self) -> dict:
        k = Tuning()
        self._ck(self._L.vd_tess_get_tuning(self._h, C.byref(k)))
        names = {v: n for n, v in FAST_LAYOUTS.items()}
        return {"fast_layout": names[k.fast_layout], "fast_blocks_per_sm": k.fast_blocks_per_sm,
                "huge_direct_max": k.huge_direct_max, "huge_blocks_max": k.huge_blocks_max,
                "huge_narrow_max": k.huge_narrow_max, "noop_run": k.noop_run}

    def set_fast_layout(self, layout: str):
        """'slots' (default: a clip rewrites only the faces it cuts) or 'full'
        (every face loop rewritten per clip): the first tier's polytope
        layout, a tuning choice with identical results."""
        self._ck(self._L.vd_tess_set_fast_layout(self._h, FAST_LAYOUTS[layout]))

    def add_wall(self, wall: Wall):
        g = wall.geometry
        L, h, wid = self._L, self._h, wall.id()
        if isinstance(g, PlaneGeometry):
            p = np.asarray(g.point, np.float64)
            n = np.asarray(g.normal, np.float64)
            self._ck(L.vd_tess_add_wall_plane(h, _dp(p), _dp(n), wid))
        elif isinstance(g, SphereGeometry):
            c = np.asarray(g.center, np.float64)
            self._ck(L.vd_tess_add_wall_sphere(h, _dp(c), g.radius, wid))
        elif isinstance(g, CylinderGeometry):
            c = np.asarray(g.center, np.float64)
            a = np.asarray(g.axis, np.float64)
            self._ck(L.vd_tess_add_wall_cylinder(h, _dp(c), _dp(a), g.radius, wid))
        elif isinstance(g, ConeGeometry):
            c = np.asarray(g.tip, np.float64)
            a = np.asarray(g.axis, np.float64)
            self._ck(L.vd_tess_add_wall_cone(h, _dp(c), _dp(a), g.angle, wid))
        elif isinstance(g, TorusGeometry):
            c = np.asarray(g.center, np.float64)
            a = np.asarray(g.axis, np.float64)
            self._ck(L.vd_tess_add_wall_torus(h, _dp(c), _dp(a), g.major_radius, g.minor_radius, wid))
        else:
            p = np.ascontiguousarray(g.points, np.float64)
            n = np.ascontiguousarray(g.normals, np.float64)
            self._ck(L.vd_tess_add_wall_polyhedron(h, _dp(p), _dp(n), len(p), wid))
        self.walls.append(wall)

    def clear_walls(self):
        self._ck(self._L.vd_tess_clear_walls(self._h))
        self.walls = []

    # ---- generators ----------------------------------------------------
    def set_generators(self, generators) -> int:
        a = np.ascontiguousarray(np.asarray(generators, np.float64).reshape(-1))
        n = a.size // 3
        a = a[:3 * n]
        kept = C.c_size_t()
        self._ck(self._L.vd_tess_set_generators(self._h, _dp(a), n, C.byref(kept)))
        return kept.value

    def set_generators_device(self, ptr: int, n: int) -> int:
        """Generators already in device memory (AoS doubles at ``ptr``)."""
        kept = C.c_size_t()
        self._ck(self._L.vd_tess_set_generators_device(self._h, C.c_void_p(ptr), int(n), C.byref(kept)))
        return kept.value

    def set_generator(self, index: int, generator: Sequence[float]):
        g = np.asarray(generator, np.float64)
        self._ck(self._L.vd_tess_set_generator(self._h, int(index), _dp(g)))

    def random_generators(self, count: int, seed: Optional[int] = None) -> int:
        """Tessellation::random_generators (tessellation.rs:96-121): `count`
        points uniform in the bounds and inside every wall (rejection, at most
        count * 1000 attempts), generated on the device.  The reference seeds
        from thread_rng; ``seed=None`` does the same with the OS's entropy,
        an integer seed makes the points reproducible.  Returns the number
        found."""
        if seed is None:
            seed = int.from_bytes(os.urandom(8), "little")
        found = C.c_size_t()
        self._ck(self._L.vd_tess_random_generators(self._h, int(count), int(seed) & (2**64 - 1),
                                                   C.byref(found)))
        return found.value

    def read_generators(self, text):
        """Tessellation::read_generators (tessellation.rs:153-171): one
        ``id x y z`` per line, the id ignored, a missing or unparsable
        coordinate 0.0 (parsed by the library's native reader)."""
        data = text.encode("utf-8") if isinstance(text, str) else bytes(text)
        kept = C.c_size_t()
        self._ck(self._L.vd_tess_read_generators(self._h, data, len(data), C.byref(kept)))
        return kept.value

    def import_generators(self, path: str):
        """Tessellation::import_generators (tessellation.rs:126-148)."""
        kept = C.c_size_t()
        self._ck(self._L.vd_tess_import_generators(self._h, os.fsencode(path), C.byref(kept)))
        return kept.value

    def count_generators(self) -> int:
        n = C.c_size_t()
        self._ck(self._L.vd_tess_count_generators(self._h, C.byref(n)))
        return n.value

    def generators(self) -> np.ndarray:
        out = np.zeros(3 * self.count_generators(), np.float64)
        self._ck(self._L.vd_tess_get_generators(self._h, _dp(out)))
        return out

    def get_generator(self, index: int) -> np.ndarray:
        return self.generators()[3 * index:3 * index + 3]

    # ---- the hot path --------------------------------------------------
    def calculate(self):
        self._ck(self._L.vd_tess_calculate(self._h))

    def calculate_range(self, begin: int, end: int):
        """calculate() for the cells with ids in [begin, end) only (one
        shard of a tessellation split across GPUs); the other cells read as
        empty.  ValueError unless 0 <= begin <= end <= count_generators()."""
        if begin < 0 or end < begin:
            raise ValueError(f"bad cell range [{begin}, {end})")
        self._ck(self._L.vd_tess_calculate_range(self._h, int(begin), int(end)))

    def calculate_strided(self, chunk: int, stride: int, phase: int, begin: int = 0, end: Optional[int] = None):
        """calculate() for the cells with ids in [begin, end) whose chunk index
        (id - begin) // chunk equals phase modulo stride (one GPU's share of an
        interleaved split); the other cells read as empty."""
        end = self.count_generators() if end is None else end
        if begin < 0 or end < begin or chunk < 1 or not 0 <= phase < stride:
            raise ValueError(f"bad strided range [{begin}, {end}) chunk={chunk} stride={stride} phase={phase}")
        self._ck(self._L.vd_tess_calculate_strided(self._h, int(begin), int(end), int(chunk), int(stride),
                                                   int(phase)))

    def calculate_sealed(self):
        """Tessellation::calculate_sealed (tessellation.rs:234-318)."""
        self._ck(self._L.vd_tess_calculate_sealed(self._h))

    def prune_boundaries(self):
        """Tessellation::prune_boundaries (tessellation.rs:323-385)."""
        self._ck(self._L.vd_tess_prune_boundaries(self._h))

    @property
    def seal_log(self) -> np.ndarray:
        """(cell, neighbour, wall id) triples, flat, as the reference's seal_log."""
        n = C.c_size_t()
        self._ck(self._L.vd_tess_seal_log(self._h, None, C.byref(n)))
        out = np.zeros(max(n.value, 1), np.int32)
        self._ck(self._L.vd_tess_seal_log(self._h, _vp(out), C.byref(n)))
        return out[:n.value]

    def _prune(self):
        ne, npos = C.c_size_t(), C.c_size_t()
        self._ck(self._L.vd_tess_prune_log(self._h, None, C.byref(ne), None, C.byref(npos)))
        e = np.zeros(max(ne.value, 1), np.int32)
        p = np.zeros(max(npos.value, 1), np.float64)
        self._ck(self._L.vd_tess_prune_log(self._h, _vp(e), C.byref(ne), _vp(p), C.byref(npos)))
        return e[:ne.value], p[:npos.value]

    @property
    def prune_log(self) -> np.ndarray:
        """(cell, neighbour, wall id, vertex count) quadruples, flat."""
        return self._prune()[0]

    @property
    def prune_pos_log(self) -> np.ndarray:
        """xyz of the logged shared vertices, flat."""
        return self._prune()[1]

    def relax(self):
        self._ck(self._L.vd_tess_relax(self._h))

    def count_cells(self) -> int:
        n = C.c_size_t()
        self._ck(self._L.vd_tess_count_cells(self._h, C.byref(n)))
        return n.value

    # ---- results -------------------------------------------------------
    def summaries(self):
        """(volume[n], centroid[n,3], n_faces[n]) of every cell."""
        n = self.count_cells()
        vol = np.zeros(n, np.float64)
        cen = np.zeros((n, 3), np.float64)
        nf = np.zeros(n, np.int32)
        self._ck(self._L.vd_tess_get_cell_summaries(self._h, _vp(vol), _vp(cen), _vp(nf)))
        return vol, cen, nf

    def total_faces(self) -> int:
        t = C.c_int64()
        self._ck(self._L.vd_tess_total_faces(self._h, C.byref(t)))
        return t.value

    def neighbors(self):
        """CSR (offsets[n+1], ids[total]) of every cell's face_neighbors."""
        n = self.count_cells()
        tot = self.total_faces()
        off = np.zeros(n + 1, np.int64)
        ids = np.zeros(max(tot, 1), np.int32)
        self._ck(self._L.vd_tess_get_neighbors(self._h, _vp(off), _vp(ids)))
        return off, ids[:tot]

    def face_areas(self):
        n = self.count_cells()
        tot = self.total_faces()
        off = np.zeros(n + 1, np.int64)
        ar = np.zeros(max(tot, 1), np.float64)
        self._ck(self._L.vd_tess_get_face_areas(self._h, _vp(off), _vp(ar)))
        return off, ar[:tot]

    def get_cell(self, index: int) -> Optional[Cell3DFaces]:
        if index < 0 or index >= self.count_cells():
            return None
        nv, nf, nh = C.c_int32(), C.c_int32(), C.c_int32()
        self._ck(self._L.vd_tess_get_cell(self._h, int(index), C.byref(nv), C.byref(nf), C.byref(nh),
                                          None, None, None, None))
        v = np.zeros(3 * max(nv.value, 1), np.float64)
        fc = np.zeros(max(nf.value, 1), np.uint32)
        fi = np.zeros(max(nh.value, 1), np.uint32)
        fn = np.zeros(max(nf.value, 1), np.int32)
        self._ck(self._L.vd_tess_get_cell(self._h, int(index), C.byref(nv), C.byref(nf), C.byref(nh),
                                          _vp(v), _vp(fc), _vp(fi), _vp(fn)))
        vol, cen, _ = self._summary_cache()
        off, ar = self._area_cache()
        return Cell3DFaces(index, v[:3 * nv.value], fc[:nf.value], fi[:nh.value], fn[:nf.value],
                           vol[index], cen[index], ar[off[index]:off[index + 1]])

    def _summary_cache(self):
        key = ("sum", id(self))
        if getattr(self, "_cache_key", None) != self._calc_stamp():
            self._cache = {}
            self._cache_key = self._calc_stamp()
        if key not in self._cache:
            self._cache[key] = self.summaries()
        return self._cache[key]

    def _area_cache(self):
        self._summary_cache()
        if "areas" not in self._cache:
            self._cache["areas"] = self.face_areas()
        return self._cache["areas"]

    def _calc_stamp(self):
        t = (C.c_float * 4)()
        self._ck(self._L.vd_tess_timings(self._h, t))
        return tuple(t) + (self.count_cells(),)

    def export_cells(self, begin: int = 0, end: Optional[int] = None) -> dict:
        """The polytopes of cells [begin, end) in one device pass, as CSR:
        ``v_off``, ``f_off``, ``h_off`` (offsets per cell), ``vertices``
        (flat xyz), ``face_counts``, ``face_indices`` (local to each cell) and
        ``face_neighbors`` -- each cell exactly as get_cell gives it."""
        n_all = self.count_cells()
        end = n_all if end is None else int(end)
        begin = int(begin)
        n = max(end - begin, 0)
        vo = np.zeros(n + 1, np.int64)
        fo = np.zeros(n + 1, np.int64)
        ho = np.zeros(n + 1, np.int64)
        i64 = C.POINTER(C.c_int64)
        self._ck(self._L.vd_tess_export_cells(self._h, begin, end, vo.ctypes.data_as(i64), fo.ctypes.data_as(i64),
                                              ho.ctypes.data_as(i64), None, None, None, None))
        v = np.zeros(3 * max(int(vo[-1]), 1), np.float64)
        fc = np.zeros(max(int(fo[-1]), 1), np.uint32)
        fi = np.zeros(max(int(ho[-1]), 1), np.uint32)
        fn = np.zeros(max(int(fo[-1]), 1), np.int32)
        self._ck(self._L.vd_tess_export_cells(self._h, begin, end, vo.ctypes.data_as(i64), fo.ctypes.data_as(i64),
                                              ho.ctypes.data_as(i64), _vp(v), _vp(fc), _vp(fi), _vp(fn)))
        return {"v_off": vo, "f_off": fo, "h_off": ho, "vertices": v[:3 * int(vo[-1])],
                "face_counts": fc[:int(fo[-1])], "face_indices": fi[:int(ho[-1])], "face_neighbors": fn[:int(fo[-1])]}

    def _iter_cells(self, chunk: int = 1 << 18):
        """Every cell as a Cell3DFaces, exported a range at a time."""
        n = self.count_cells()
        if n == 0:
            return
        vol, cen, _ = self._summary_cache()
        aoff, ar = self._area_cache()
        for b in range(0, n, chunk):
            e = min(n, b + chunk)
            x = self.export_cells(b, e)
            vo, fo, ho = x["v_off"], x["f_off"], x["h_off"]
            for k in range(e - b):
                i = b + k
                yield Cell3DFaces(i, x["vertices"][3 * vo[k]:3 * vo[k + 1]], x["face_counts"][fo[k]:fo[k + 1]],
                                  x["face_indices"][ho[k]:ho[k + 1]], x["face_neighbors"][fo[k]:fo[k + 1]],
                                  vol[i], cen[i], ar[aoff[i]:aoff[i + 1]])

    def cells(self) -> List[Cell3DFaces]:
        """Tessellation::cells (tessellation.rs:524-526)."""
        return list(self._iter_cells())

    def map(self, f: Callable[[Cell3DFaces], object]) -> list:
        """Tessellation::map (tessellation.rs:391-412): compute, then apply f."""
        self.calculate()
        return [f(c) for c in self._iter_cells()]

    # ---- instrumentation -------------------------------------------------
    def stream(self) -> int:
        s = C.c_void_p()
        self._ck(self._L.vd_tess_stream(self._h, C.byref(s)))
        return s.value or 0

    def timings(self) -> dict:
        t = (C.c_float * 4)()
        self._ck(self._L.vd_tess_timings(self._h, t))
        return {"bin_ms": t[0], "clip_ms": t[1], "fallback_ms": t[2], "total_ms": t[3]}

    def set_instrumentation(self, on: bool):
        """Count the algorithmic events (candidates, clips, ...) in calculate()."""
        self._ck(self._L.vd_tess_set_instrumentation(self._h, 1 if on else 0))

    def counters(self) -> dict:
        out = (C.c_uint64 * 8)()
        self._ck(self._L.vd_tess_counters(self._h, out))
        names = ("candidates", "clips", "classified", "modifying", "intersections", "kept",
                 "triangles", "offsets")
        return {k: int(v) for k, v in zip(names, out)}

    def fallback_counts(self) -> dict:
        out = (C.c_uint64 * 2)()
        self._ck(self._L.vd_tess_fallback_counts(self._h, out))
        return {"overflow": int(out[0]), "table": int(out[1])}
