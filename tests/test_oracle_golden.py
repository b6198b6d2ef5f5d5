"""CPU: the oracle against the reference's own known answers and its Voro++
golden vectors (the pins that make it a trustworthy checker)."""
import math

import numpy as np
import pytest

from common import golden, uniform

WALL = -1000


def test_cell_box_volume_centroid(oracle_mod):
    # cell_3d_faces.rs:576-583
    c = oracle_mod.OracleCell.new(0, [0, 0, 0], [1, 1, 1])
    assert abs(c.volume() - 1.0) < 1e-6
    assert abs(c.centroid()[0] - 0.5) < 1e-6


def test_cell_half_clip(oracle_mod):
    # cell_3d_faces.rs:585-593
    c = oracle_mod.OracleCell.new(0, [0, 0, 0], [1, 1, 1])
    c.clip([0.5, 0.5, 0.5], [1.0, 0.0, 0.0], 10)
    assert abs(c.volume() - 0.5) < 1e-6
    assert 10 in list(c.face_neighbors())


def test_cell_metrics(oracle_mod):
    # tests/integration.rs:3-20
    c = oracle_mod.OracleCell.new(0, [0, 0, 0], [10, 20, 30])
    assert abs(c.volume() - 6000.0) < 1e-6
    assert np.allclose(c.centroid(), [5, 10, 15], atol=1e-6)


def test_grid_indexing(oracle_mod):
    # algo_3d_grid.rs:209-219
    t = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 10, 10, 10)
    assert t.bin_index(0.5, 0.5, 0.5) == 0
    assert t.bin_index(1.5, 0.5, 0.5) == 1


def test_two_generators_total_volume(oracle_mod):
    # tests/integration.rs:22-46
    t = oracle_mod.OracleTessellation([0, 0, 0], [100, 100, 100], 10, 10, 10)
    t.set_generators([10, 10, 10, 90, 90, 90])
    t.calculate()
    vol, _, _ = t.summaries()
    assert t.count_cells() == 2
    assert abs(vol.sum() - 1e6) < 1e-3


def test_octet(oracle_mod):
    # tests/integration.rs:48-79
    t = oracle_mod.OracleTessellation([0, 0, 0], [100, 100, 100], 10, 10, 10)
    pts = [[x, y, z] for x in (25, 75) for y in (25, 75) for z in (25, 75)]
    t.set_generators(np.asarray(pts, float))
    t.calculate()
    vol, _, _ = t.summaries()
    assert np.all(np.abs(vol - 125000.0) < 1e-3)


def test_mapping_face_counts(oracle_mod):
    # tests/mapping.rs:3-35
    t = oracle_mod.OracleTessellation([0, 0, 0], [1, 1, 1], 4, 4, 4)
    pts = [[x, y, z] for x in (0.25, 0.75) for y in (0.25, 0.75) for z in (0.25, 0.75)]
    t.set_generators(np.asarray(pts, float))
    t.calculate()
    _, _, nf = t.summaries()
    assert list(nf) == [6] * 8


def test_two_cells_neighbors(oracle_mod):
    # tests/neighbors.rs:96-114
    t = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 1, 1, 1)
    t.set_generators([2.5, 5, 5, 7.5, 5, 5])
    t.calculate()
    off, ids = t.neighbors()
    assert 1 in ids[off[0]:off[1]] and 0 in ids[off[1]:off[2]]


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_reciprocity_random(oracle_mod, seed):
    # tests/neighbors.rs:117-136 with seeded inputs
    t = oracle_mod.OracleTessellation([0, 0, 0], [30, 30, 30], 5, 5, 5)
    t.set_generators(uniform(27, 0, 30, seed))
    t.calculate()
    off, ids = t.neighbors()
    for i in range(t.count_cells()):
        for j in ids[off[i]:off[i + 1]]:
            if j >= 0:
                assert i in ids[off[j]:off[j + 1]]


def test_sphere_wall_volume(oracle_mod):
    # tests/volumes.rs:5-59 (20^3 lattice, grid 5^3, sphere r=4 within 1%)
    n = 20
    step = 10.0 / n
    g = [[x * step + step / 2, y * step + step / 2, z * step + step / 2]
         for x in range(n) for y in range(n) for z in range(n)]
    t = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 5, 5, 5)
    t.set_generators(np.asarray(g))
    t.add_wall_sphere([5, 5, 5], 4.0, WALL)
    t.calculate()
    vol, _, _ = t.summaries()
    exp = 4.0 / 3.0 * math.pi * 4.0 ** 3
    assert abs(vol.sum() - exp) / exp < 0.01


def test_wall_id_check(oracle_mod):
    t = oracle_mod.OracleTessellation([0, 0, 0], [1, 1, 1], 2, 2, 2)
    with pytest.raises(ValueError):
        t.add_wall_sphere([0.5, 0.5, 0.5], 0.3, -999)


def test_voro_face_counts(oracle_mod):
    # reference tests/data/face_counts: box [-10,10]^3, grid 6^3, no wall
    g = golden("voro_face_counts.json")
    t = oracle_mod.OracleTessellation(g["bounds_min"], g["bounds_max"], *g["grid"])
    t.set_generators(np.asarray([r[1:] for r in g["generators"]]))
    t.calculate()
    _, _, nf = t.summaries()
    exp = np.asarray([g["face_counts"][str(r[0])] for r in g["generators"]])
    assert np.array_equal(nf, exp)


def test_voro_vertex_positions(oracle_mod):
    # reference tests/comparisons.rs:109-207 against its Voro++ output
    g = golden("voro_vertex_positions.json")
    t = oracle_mod.OracleTessellation(g["bounds_min"], g["bounds_max"], *g["grid"])
    w = g["walls"][0]
    t.add_wall_sphere(w["center"], w["radius"], w["id"])
    t.set_generators(np.asarray([r[1:] for r in g["generators"]]))
    t.calculate()
    for cid, exp in g["cells"].items():
        v = t.get_cell(int(cid)).vertices().reshape(-1, 3)
        exp = np.asarray(exp)
        assert len(v) == len(exp), cid
        for e in exp:
            assert np.any(np.all(np.abs(v - e) < 1e-4, axis=1)), (cid, e)


def test_search_order_stable_ties(oracle_mod):
    t = oracle_mod.OracleTessellation([0, 0, 0], [1, 1, 1], 3, 3, 3)
    d, m = t.search_order()
    assert len(m) == 7 ** 3 and np.all(np.diff(m) >= 0)
    # the 27 offsets with min_d2 == 0 come first, in z-outer / x-inner order
    first = d[:27]
    lin = (first[:, 2] + 3) * 49 + (first[:, 1] + 3) * 7 + (first[:, 0] + 3)
    assert np.all(np.diff(lin) > 0)


def test_volume_sum_uniform(oracle_mod):
    t = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 10, 10, 10)
    t.set_generators(uniform(1000, 0, 10, 0))
    t.calculate()
    vol, _, _ = t.summaries()
    assert abs(vol.sum() - 1000.0) < 1e-9 * 1000


def test_interior_neighbours_match_delaunay(oracle_mod):
    """Independent cross-check: for cells that touch no box face, the
    Voronoi neighbour set is the Delaunay neighbour set of the generators
    (scipy.spatial.Delaunay), for random general-position inputs."""
    import numpy as np
    from scipy.spatial import Delaunay
    rng = np.random.Generator(np.random.PCG64(90))
    pts = rng.uniform(0.0, 1.0, size=(3000, 3))
    t = oracle_mod.OracleTessellation([0, 0, 0], [1, 1, 1], 14, 14, 14)
    t.set_generators(pts)
    t.calculate(1)
    off, ids = t.neighbors()
    tri = Delaunay(pts)
    indptr, nb = tri.vertex_neighbor_vertices
    checked = 0
    for i in range(len(pts)):
        mine = ids[off[i]:off[i + 1]]
        if np.any(mine < 0):
            continue
        assert set(int(x) for x in mine) == set(int(x) for x in nb[indptr[i]:indptr[i + 1]]), i
        checked += 1
    assert checked > 1500


def _library_order(lo, hi, n, k):
    import ctypes as C
    from vorothree_b200 import _lib
    L = _lib.load()
    mn = np.asarray(lo, np.float64)
    mx = np.asarray(hi, np.float64)
    dp = C.POINTER(C.c_double)
    cnt = C.c_size_t()
    comp = C.c_int()
    bound = C.c_double()
    _lib.check(L.vd_search_order(mn.ctypes.data_as(dp), mx.ctypes.data_as(dp), *n, k, None, None, 0, C.byref(cnt),
                                 C.byref(comp), C.byref(bound)))
    d = np.zeros(3 * max(cnt.value, 1), np.int32)
    m = np.zeros(max(cnt.value, 1), np.float64)
    _lib.check(L.vd_search_order(mn.ctypes.data_as(dp), mx.ctypes.data_as(dp), *n, k,
                                 d.ctypes.data_as(C.POINTER(C.c_int32)), m.ctypes.data_as(dp), cnt.value,
                                 C.byref(cnt), C.byref(comp), C.byref(bound)))
    return d[:3 * cnt.value].reshape(-1, 3), m[:cnt.value], bool(comp.value), bound.value


@pytest.mark.parametrize("lo,hi,n", [([0, 0, 0], [1, 1, 1], (9, 9, 9)), ([0, 0, 0], [10, 10, 10], (12, 12, 12)),
                                     ([-3, 0, 2], [4, 2, 9], (7, 5, 11)), ([0, 0, 0], [1, 2, 3], (10, 20, 30))])
def test_search_order_matches_oracle(oracle_mod, lo, hi, n):
    """Algorithm3DGrid::new's order as the kernels get it (a counting sort by
    the integer key on cubic bins, a stable sort otherwise) equals the
    oracle's stable sort, complete and truncated."""
    o = oracle_mod.OracleTessellation(lo, hi, *n)
    od, om = o.search_order()
    d, m, comp, _ = _library_order(lo, hi, n, max(n))
    assert comp and np.array_equal(d, od) and np.array_equal(m, om)
    for k in (2, 4):
        d, m, comp, bound = _library_order(lo, hi, n, k)
        assert not comp
        keep = om < bound
        assert np.array_equal(d, od[keep]) and np.array_equal(m, om[keep])


def test_truncated_search_order_equals_complete(oracle_mod):
    """The oracle's truncated search order (for grids whose complete table
    does not fit in memory) keeps the complete table's order: with enough
    bins per axis every result and event counter is the complete table's,
    and a table too short for some cell raises instead of answering."""
    pts = uniform(20000, 0.0, 1.0, 5)
    full = oracle_mod.OracleTessellation([0, 0, 0], [1, 1, 1], 40, 40, 40)
    full.set_generators(pts)
    full.calculate()
    cut = oracle_mod.OracleTessellation([0, 0, 0], [1, 1, 1], 40, 40, 40, order_k=6)
    cut.set_generators(pts)
    cut.calculate()
    for a, b in zip(full.summaries(), cut.summaries()):
        assert np.array_equal(a, b)
    assert np.array_equal(full.neighbors()[1], cut.neighbors()[1])
    assert full.counters() == cut.counters()
    short = oracle_mod.OracleTessellation([0, 0, 0], [1, 1, 1], 40, 40, 40, order_k=2)
    short.set_generators(pts)
    with pytest.raises(RuntimeError):
        short.calculate()
