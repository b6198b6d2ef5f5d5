"""GPU parity: the CUDA path through the C ABI against the oracle.

The plain FP64 path performs the reference's arithmetic in the reference's
order, so every per-cell result is compared for exact (bitwise) equality:
volumes, centroids, face counts, neighbour ids in face order, face areas, the
full polytope of sampled cells, and the algorithmic event counters.
"""
import math

import numpy as np
import pytest

from common import blobs, csr_lists, golden, uniform

pytestmark = pytest.mark.gpu

WALL = -1000


def gpu_tess(bmin, bmax, grid, pts, walls=(), walls_first=False, precision="fp64"):
    import vorothree_b200 as v
    t = v.Tessellation(v.BoundingBox(bmin, bmax), v.Algorithm3DGrid(*grid))
    t.set_instrumentation(True)
    t.set_precision(precision)
    if walls_first:
        for w in walls:
            t.add_wall(w)
        t.set_generators(pts)
    else:
        t.set_generators(pts)
        for w in walls:
            t.add_wall(w)
    t.calculate()
    return t


def oracle_tess(oracle_mod, bmin, bmax, grid, pts, walls=(), walls_first=False):
    t = oracle_mod.OracleTessellation(bmin, bmax, *grid)

    def add(w):
        g = w.geometry
        if hasattr(g, "radius"):
            t.add_wall_sphere(g.center, g.radius, w.id())
        else:
            t.add_wall_plane(g.point, g.normal, w.id())
    if walls_first:
        for w in walls:
            add(w)
        t.set_generators(pts)
    else:
        t.set_generators(pts)
        for w in walls:
            add(w)
    t.calculate()
    return t


def assert_same(g, o, check_counters=True, sample_cells=8):
    assert g.count_generators() == o.count_generators()
    assert g.count_cells() == o.count_cells()
    assert np.array_equal(g.generators(), o.generators())
    gv, gc, gn = g.summaries()
    ov, oc, on = o.summaries()
    assert np.array_equal(gn, on), np.nonzero(gn != on)[0][:10]
    assert np.array_equal(gv, ov), np.nonzero(gv != ov)[0][:10]
    assert np.array_equal(gc, oc)
    goff, gids = g.neighbors()
    ooff, oids = o.neighbors()
    assert np.array_equal(goff, ooff)
    assert np.array_equal(gids, oids)
    _, gar = g.face_areas()
    _, oar = o.face_areas()
    assert np.array_equal(gar, oar)
    if check_counters and sum(g.fallback_counts().values()) == 0:
        assert g.counters() == o.counters()
    n = g.count_cells()
    for i in sorted(set(np.linspace(0, n - 1, min(n, sample_cells)).astype(int))):
        gcell = g.get_cell(int(i))
        ocell = o.get_cell(int(i))
        ov_, ofc, ofi, ofn = ocell.export()
        assert np.array_equal(gcell.vertices(), ov_)
        assert np.array_equal(gcell.face_counts(), ofc)
        assert np.array_equal(gcell.face_indices(), ofi)
        assert np.array_equal(gcell.face_neighbors(), ofn)


def test_known_answers():
    import vorothree_b200 as v
    t = gpu_tess([0, 0, 0], [100, 100, 100], (10, 10, 10), [10, 10, 10, 90, 90, 90])
    vol, _, _ = t.summaries()
    assert t.count_cells() == 2 and abs(vol.sum() - 1e6) < 1e-3
    pts = np.asarray([[x, y, z] for x in (25, 75) for y in (25, 75) for z in (25, 75)], float)
    t = gpu_tess([0, 0, 0], [100, 100, 100], (10, 10, 10), pts)
    vol, _, _ = t.summaries()
    assert np.all(np.abs(vol - 125000.0) < 1e-3)
    pts = np.asarray([[x, y, z] for x in (0.25, 0.75) for y in (0.25, 0.75) for z in (0.25, 0.75)])
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(4, 4, 4))
    t.set_generators(pts)
    assert t.map(lambda c: len(c.face_counts())) == [6] * 8
    t = gpu_tess([0, 0, 0], [10, 10, 10], (1, 1, 1), [2.5, 5, 5, 7.5, 5, 5])
    assert 1 in t.get_cell(0).face_neighbors() and 0 in t.get_cell(1).face_neighbors()


PRECISIONS = ["fp64", "mixed"]


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_config_a_bitwise(oracle_mod, seed, precision):
    pts = uniform(1000, 0.0, 10.0, seed)
    g = gpu_tess([0, 0, 0], [10, 10, 10], (10, 10, 10), pts, precision=precision)
    o = oracle_tess(oracle_mod, [0, 0, 0], [10, 10, 10], (10, 10, 10), pts)
    assert_same(g, o)
    vol, _, _ = g.summaries()
    assert abs(vol.sum() - 1000.0) < 1e-9 * 1000


def test_voro_golden_through_gpu():
    import vorothree_b200 as v
    gf = golden("voro_face_counts.json")
    t = gpu_tess(gf["bounds_min"], gf["bounds_max"], gf["grid"], np.asarray([r[1:] for r in gf["generators"]]))
    _, _, nf = t.summaries()
    exp = np.asarray([gf["face_counts"][str(r[0])] for r in gf["generators"]])
    assert np.array_equal(nf, exp)
    gv = golden("voro_vertex_positions.json")
    w = gv["walls"][0]
    t = gpu_tess(gv["bounds_min"], gv["bounds_max"], gv["grid"], np.asarray([r[1:] for r in gv["generators"]]),
                 walls=[v.Wall(w["id"], v.SphereGeometry(w["center"], w["radius"]))], walls_first=True)
    for cid, exp in gv["cells"].items():
        vv = t.get_cell(int(cid)).vertices().reshape(-1, 3)
        exp = np.asarray(exp)
        assert len(vv) == len(exp)
        for e in exp:
            assert np.any(np.all(np.abs(vv - e) < 1e-4, axis=1))


@pytest.mark.parametrize("precision", PRECISIONS)
def test_walls_bitwise(oracle_mod, precision):
    import vorothree_b200 as v
    pts = uniform(3000, 0.0, 30.0, 5)
    walls = [v.Wall(WALL, v.SphereGeometry([15, 15, 15], 12.0)),
             v.Wall(WALL - 1, v.PlaneGeometry([15, 15, 15], [1.0, 0.3, 0.0]))]
    g = gpu_tess([0, 0, 0], [30, 30, 30], (8, 8, 8), pts, walls, precision=precision)
    o = oracle_tess(oracle_mod, [0, 0, 0], [30, 30, 30], (8, 8, 8), pts, walls)
    assert_same(g, o)


def test_sphere_lattice_volume(oracle_mod):
    import vorothree_b200 as v
    n = 20
    step = 10.0 / n
    pts = np.asarray([[x * step + step / 2, y * step + step / 2, z * step + step / 2]
                      for x in range(n) for y in range(n) for z in range(n)])
    walls = [v.Wall(WALL, v.SphereGeometry([5, 5, 5], 4.0))]
    g = gpu_tess([0, 0, 0], [10, 10, 10], (5, 5, 5), pts, walls)
    o = oracle_tess(oracle_mod, [0, 0, 0], [10, 10, 10], (5, 5, 5), pts, walls)
    assert_same(g, o)
    vol, _, _ = g.summaries()
    exp = 4.0 / 3.0 * math.pi * 64.0
    assert abs(vol.sum() - exp) / exp < 0.01


@pytest.mark.parametrize("precision", PRECISIONS)
def test_blobs_bitwise(oracle_mod, precision):
    import vorothree_b200 as v
    pts = blobs(20000, 8, 0.01, 0.7, 11)
    walls = [v.Wall(WALL, v.SphereGeometry([0.5, 0.5, 0.5], 0.45))]
    g = gpu_tess([0, 0, 0], [1, 1, 1], (20, 20, 20), pts, walls, precision=precision)
    o = oracle_tess(oracle_mod, [0, 0, 0], [1, 1, 1], (20, 20, 20), pts, walls)
    assert_same(g, o)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_uniform_100k_bitwise(oracle_mod, precision):
    pts = uniform(100_000, 0.0, 1.0, 3)
    g = gpu_tess([0, 0, 0], [1, 1, 1], (46, 46, 46), pts, precision=precision)
    o = oracle_tess(oracle_mod, [0, 0, 0], [1, 1, 1], (46, 46, 46), pts)
    assert_same(g, o)


def test_edge_cases(oracle_mod):
    import vorothree_b200 as v
    # empty input
    t = gpu_tess([0, 0, 0], [1, 1, 1], (3, 3, 3), np.zeros((0, 3)))
    assert t.count_cells() == 0 and t.total_faces() == 0
    # single generator: the whole box
    t = gpu_tess([0, 0, 0], [2, 3, 4], (3, 3, 3), [0.5, 0.5, 0.5])
    vol, cen, nf = t.summaries()
    assert vol[0] == 24.0 and nf[0] == 6
    # duplicate generators and points outside the box (kept, as in the reference)
    pts = np.concatenate([uniform(200, 0, 1, 9), uniform(5, 0, 1, 9), [[1.5, 0.5, 0.5], [-0.2, 0.1, 0.3]]])
    g = gpu_tess([0, 0, 0], [1, 1, 1], (4, 4, 4), pts)
    o = oracle_tess(oracle_mod, [0, 0, 0], [1, 1, 1], (4, 4, 4), pts)
    assert_same(g, o)
    # a wall that removes everything
    walls = [v.Wall(WALL, v.SphereGeometry([5, 5, 5], 0.1))]
    t = gpu_tess([0, 0, 0], [1, 1, 1], (2, 2, 2), uniform(50, 0, 1, 1), walls)
    assert t.count_generators() == 0


def test_relax_bitwise(oracle_mod):
    import vorothree_b200 as v
    pts = uniform(2000, 0.0, 1.0, 4)
    walls = [v.Wall(WALL, v.SphereGeometry([0.5, 0.5, 0.5], 0.48))]
    g = gpu_tess([0, 0, 0], [1, 1, 1], (12, 12, 12), pts, walls)
    o = oracle_tess(oracle_mod, [0, 0, 0], [1, 1, 1], (12, 12, 12), pts, walls)
    for _ in range(3):
        g.relax()
        o.relax()
        g.calculate()
        o.calculate()
        assert_same(g, o, sample_cells=2)


def test_table_extension(oracle_mod):
    # a large grid (truncated search order) with few generators: cells must
    # walk far and the table is extended on demand
    pts = uniform(300, 0.0, 1.0, 6)
    g = gpu_tess([0, 0, 0], [1, 1, 1], (80, 80, 80), pts)
    o = oracle_tess(oracle_mod, [0, 0, 0], [1, 1, 1], (80, 80, 80), pts)
    assert g.fallback_counts()["table"] > 0
    assert_same(g, o, check_counters=False)


def test_set_generator_moves_bin(oracle_mod):
    import vorothree_b200 as v
    pts = uniform(500, 0.0, 1.0, 8)
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(5, 5, 5))
    t.set_generators(pts)
    t.set_generator(3, [0.91, 0.92, 0.93])
    t.calculate()
    assert np.allclose(t.get_generator(3), [0.91, 0.92, 0.93])
    vol, _, _ = t.summaries()
    assert abs(vol.sum() - 1.0) < 1e-9


def test_read_and_import_generators(oracle_mod, tmp_path):
    """Tessellation::read_generators / import_generators (tessellation.rs:126-171)
    through the C ABI: the same generators, and the same cells, as
    set_generators of the parsed points; a file that cannot be read is
    VD_EIO and text that is not UTF-8 VD_EINVAL, with nothing changed."""
    import vorothree_b200 as v
    from vorothree_b200._lib import VD_EINVAL, VD_EIO
    pts = uniform(1500, 0.0, 1.0, 40).tolist()
    text = "".join(f"{i} {x!r} {y!r} {z!r}\n" for i, (x, y, z) in enumerate(pts))
    text += "\n  \n9999 0.5\r\n7 0.25 bad 0.75 extra\n"
    path = tmp_path / "generators.txt"
    path.write_text(text)
    wall = v.Wall(-1000, v.SphereGeometry([0.5, 0.5, 0.5], 0.45))

    def fresh():
        t = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(9, 9, 9))
        t.set_instrumentation(True)
        t.add_wall(wall)
        return t
    a, b = fresh(), fresh()
    ka = a.read_generators(text)
    kb = b.import_generators(str(path))
    parsed = v.parse_generators(text)
    assert parsed.shape == (len(pts) + 2, 3)
    assert parsed[-2].tolist() == [0.5, 0.0, 0.0] and parsed[-1].tolist() == [0.25, 0.0, 0.75]
    o = oracle_tess(oracle_mod, [0, 0, 0], [1, 1, 1], (9, 9, 9), parsed, [wall], walls_first=True)
    assert ka == kb == o.count_generators()
    for t in (a, b):
        t.calculate()
        assert_same(t, o, sample_cells=3)
    before = a.generators()
    with pytest.raises(v.VoronoidError) as e:
        a.import_generators(str(tmp_path / "missing.txt"))
    assert e.value.code == VD_EIO
    with pytest.raises(v.VoronoidError) as e:
        a.read_generators(b"0 0.5 0.5 0.5\n1 0.4 \xff 0.4\n")
    assert e.value.code == VD_EINVAL
    assert np.array_equal(a.generators(), before)


@pytest.mark.parametrize("scale,offset", [(1000.0, 0.0), (1e-3, 0.0), (1.0, 5000.0)])
def test_mixed_equals_fp64_across_scales(scale, offset):
    """The FP32 classification's error bound must hold at every coordinate
    scale: mixed results equal the FP64 path bit for bit."""
    pts = uniform(20000, 0.0, 1.0, 12) * scale + offset
    lo, hi = [offset] * 3, [offset + scale] * 3
    a = gpu_tess(lo, hi, (27, 27, 27), pts)
    b = gpu_tess(lo, hi, (27, 27, 27), pts, precision="mixed")
    av, ac, an = a.summaries()
    bv, bc, bn = b.summaries()
    assert np.array_equal(an, bn) and np.array_equal(av, bv) and np.array_equal(ac, bc)
    assert np.array_equal(a.neighbors()[1], b.neighbors()[1])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_dense_blob_overflow_tiers(oracle_mod, precision):
    """A dense blob on a coarse grid: the reference's bin-order walk clips each
    cell with thousands of candidates and the intermediate polytopes outgrow
    the fast path; the medium and large-capacity passes must give the oracle's
    bits."""
    rng = np.random.Generator(np.random.PCG64(17))
    pts = np.concatenate([0.5 + rng.normal(0.0, 0.01, size=(2500, 3)), rng.uniform(0, 1, size=(300, 3))])
    g = gpu_tess([0, 0, 0], [1, 1, 1], (4, 4, 4), pts, precision=precision)
    o = oracle_tess(oracle_mod, [0, 0, 0], [1, 1, 1], (4, 4, 4), pts)
    assert g.fallback_counts()["overflow"] > 0
    assert_same(g, o, check_counters=False)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_calculate_range_shards(oracle_mod, precision):
    """calculate_range computes exactly the oracle's cells of the range and
    leaves the others empty; the shards of a split put together equal one
    full calculate()."""
    import vorothree_b200 as v
    from vorothree_b200.shard import cell_range
    pts = uniform(30000, 0.0, 1.0, 21)
    walls = [v.Wall(WALL, v.SphereGeometry([0.5, 0.5, 0.5], 0.47))]
    g = gpu_tess([0, 0, 0], [1, 1, 1], (24, 24, 24), pts, walls, precision=precision)
    full_v, full_c, full_n = g.summaries()
    full_off, full_ids = g.neighbors()
    n = g.count_generators()
    o = oracle_mod.OracleTessellation([0, 0, 0], [1, 1, 1], 24, 24, 24)
    o.set_generators(pts)
    o.add_wall_sphere([0.5, 0.5, 0.5], 0.47, WALL)
    world = 3
    got_v, got_c, got_n = np.zeros(n), np.zeros((n, 3)), np.zeros(n, np.int32)
    for rank in range(world):
        b, e = cell_range(n, rank, world)
        g.calculate_range(b, e)
        o.calculate_range(b, e)
        assert_same(g, o, sample_cells=4)
        gv, gc, gn = g.summaries()
        outside = np.ones(n, bool)
        outside[b:e] = False
        assert np.all(gv[outside] == 0) and np.all(gn[outside] == 0) and np.all(gc[outside] == 0)
        got_v[b:e], got_c[b:e], got_n[b:e] = gv[b:e], gc[b:e], gn[b:e]
    assert np.array_equal(got_v, full_v) and np.array_equal(got_c, full_c) and np.array_equal(got_n, full_n)
    # an empty range and the full range
    g.calculate_range(5, 5)
    assert g.summaries()[2].sum() == 0 and g.total_faces() == 0
    g.calculate_range(0, n)
    assert np.array_equal(g.neighbors()[1], full_ids)
    with pytest.raises(v.VoronoidError):
        g.calculate_range(0, n + 1)
    with pytest.raises(ValueError):
        g.calculate_range(4, 3)


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("jitter", [0.0, 1e-13, 1e-9, 1e-6])
def test_degenerate_lattices_bitwise(oracle_mod, jitter, precision):
    """Generators on (or within `jitter` of) a cubic lattice: bisector planes
    pass exactly through existing vertices, so vertices fall inside the 1e-9
    band, intersection vertices coincide and lid segments share endpoints --
    the degenerate cases of clip_with_scratch.  The GPU must still match the
    oracle bit for bit."""
    n = 9
    ax = (np.arange(n) + 0.5) / n
    pts = np.array([[x, y, z] for z in ax for y in ax for x in ax])
    if jitter:
        rng = np.random.Generator(np.random.PCG64(77))
        pts = pts + rng.uniform(-jitter, jitter, size=pts.shape)
    g = gpu_tess([0, 0, 0], [1, 1, 1], (5, 5, 5), pts, precision=precision)
    o = oracle_tess(oracle_mod, [0, 0, 0], [1, 1, 1], (5, 5, 5), pts)
    assert_same(g, o, sample_cells=16)
    vol, _, _ = g.summaries()
    if jitter != 1e-9:
        assert abs(vol.sum() - 1.0) < 1e-9
    else:
        # jitter at the scale of the reference's 1e-9 clip band: its
        # classification drops slivers, so the cells no longer fill the box
        # (the oracle loses the same volume; the bits match above)
        assert 0.99 < vol.sum() < 1.0


GEOMETRIES = {
    # one bin: every cell walks the whole input in the reference's order
    "one_bin": ([0, 0, 0], [1, 1, 1], (1, 1, 1), 300),
    # flat, anisotropic box and grid
    "slab": ([0, 0, 0], [100, 1, 0.01], (50, 3, 1), 3000),
    "needle": ([-5, -5, -5], [-4.99, -4.99, 5], (1, 1, 200), 2000),
    # large offset and tiny extent; large extent
    "offset": ([1e6, 1e6, 1e6], [1e6 + 1e-3, 1e6 + 1e-3, 1e6 + 1e-3], (10, 10, 10), 4000),
    "huge": ([-1e9, -1e9, -1e9], [1e9, 1e9, 1e9], (16, 16, 16), 4000),
    # more bins than generators, odd resolutions
    "sparse": ([0, 0, 0], [1, 2, 3], (37, 41, 43), 500),
}


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("name", list(GEOMETRIES))
def test_geometry_extremes_bitwise(oracle_mod, name, precision):
    """Boxes, grids and coordinate scales far from the unit cube, with some
    generators exactly on bin boundaries and on the box's max faces (where
    get_bin_index clamps to grid_limit, algo_3d_grid.rs:97-106)."""
    lo, hi, grid, n = GEOMETRIES[name]
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    rng = np.random.Generator(np.random.PCG64(91))
    pts = lo + rng.uniform(0, 1, size=(n, 3)) * (hi - lo)
    k = n // 10
    cells = np.asarray(grid, np.float64)
    pts[:k] = lo + np.floor(rng.uniform(0, 1, size=(k, 3)) * cells) / cells * (hi - lo)
    pts[k:k + 5] = hi
    pts[k + 5:k + 10, 0] = hi[0]
    g = gpu_tess(lo, hi, grid, pts, precision=precision)
    o = oracle_tess(oracle_mod, lo, hi, grid, pts)
    # no volume-sum check: the five generators stacked on the max corner
    # overlap (bisector of coincident points), and at a 1e6 offset the
    # reference's volume formula, on absolute coordinates, cancels
    # catastrophically -- the oracle shows both, and the device matches it
    assert_same(g, o, sample_cells=6)


def test_wall_limits():
    """At most 16 walls and 256 convex-polyhedron planes per tessellation
    (fixed tables in the kernels' parameters); one more is VD_EINVAL and
    leaves the walls as they were."""
    import vorothree_b200 as v
    from vorothree_b200._lib import VD_EINVAL
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(2, 2, 2))
    for k in range(16):
        t.add_wall(v.Wall(WALL - k, v.PlaneGeometry([0.5, 0.5, 0.5], [0, 0, 1])))
    with pytest.raises(v.VoronoidError) as e:
        t.add_wall(v.Wall(WALL - 16, v.PlaneGeometry([0.5, 0.5, 0.5], [0, 0, 1])))
    assert e.value.code == VD_EINVAL
    t.set_generators(uniform(100, 0, 1, 3))
    t.calculate()
    assert t.count_cells() == int((uniform(100, 0, 1, 3)[:, 2] >= 0.5).sum())
    t.clear_walls()
    big = v.ConvexPolyhedronGeometry([[0.5, 0.5, 0.5]] * 200, [[0, 0, 1]] * 200)
    t.add_wall(v.Wall(WALL, big))
    with pytest.raises(v.VoronoidError) as e:
        t.add_wall(v.Wall(WALL - 1, v.ConvexPolyhedronGeometry([[0.5, 0.5, 0.5]] * 57, [[0, 0, 1]] * 57)))
    assert e.value.code == VD_EINVAL


@pytest.mark.parametrize("precision", PRECISIONS)
def test_degenerate_duplicates_and_planes(oracle_mod, precision):
    """Repeated generators, generators on the box faces and on a wall plane."""
    import vorothree_b200 as v
    rng = np.random.Generator(np.random.PCG64(78))
    base = rng.uniform(0, 1, size=(400, 3))
    on_faces = base[:60].copy()
    on_faces[:20, 0] = 0.0
    on_faces[20:40, 1] = 1.0
    on_faces[40:, 2] = 0.5
    pts = np.concatenate([base, base[:50], on_faces])
    walls = [v.Wall(WALL, v.PlaneGeometry([0.5, 0.5, 0.5], [0, 0, 1]))]
    g = gpu_tess([0, 0, 0], [1, 1, 1], (6, 6, 6), pts, walls, precision=precision)
    o = oracle_tess(oracle_mod, [0, 0, 0], [1, 1, 1], (6, 6, 6), pts, walls)
    assert_same(g, o, sample_cells=16)


@pytest.mark.parametrize("n", [1000, 3000])
@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("kind", ["axes", "central", "sphere"])
def test_bench_distributions_bitwise(oracle_mod, kind, precision, n):
    """The distributions of the reference's criterion benches
    (benches/distributions.rs) on their box and bin heuristic (ceil(N^(1/3))
    bins per axis): generators crowding three mid-planes, a dense central box
    with an empty shell, and generators on a sphere (needle-shaped cells).
    The sphere's centre cell takes the block tier: 16-warp blocks at 1,000
    generators, 32-warp blocks at 3,000."""
    from common import bench_distribution
    pts = bench_distribution(kind, n, 70 + len(kind))
    g = int(np.ceil(n ** (1.0 / 3.0)))
    gt = gpu_tess([0, 0, 0], [100, 100, 100], (g, g, g), pts, precision=precision)
    o = oracle_tess(oracle_mod, [0, 0, 0], [100, 100, 100], (g, g, g), pts)
    assert_same(gt, o, sample_cells=6)


def test_sphere_surface_10k_huge_cell(oracle_mod):
    """10,000 generators on a sphere plus its centre (the reference's own
    benchmark distribution at its larger size): the centre's cell has 9,999
    faces and ~20,000 vertices, beyond every shared-memory and large
    capacity; the huge tier builds it with the oracle's bits."""
    from common import bench_distribution
    pts = bench_distribution("sphere", 10000, 81)
    g = gpu_tess([0, 0, 0], [100, 100, 100], (22, 22, 22), pts)
    o = oracle_tess(oracle_mod, [0, 0, 0], [100, 100, 100], (22, 22, 22), pts)
    assert g.summaries()[2][0] == 9999
    assert g.fallback_counts()["overflow"] > 0
    assert_same(g, o, sample_cells=3)


@pytest.mark.parametrize("stride", [2, 3])
def test_calculate_strided_shards(oracle_mod, stride):
    """calculate_strided computes interleaved chunks of cell ids; the shards'
    cells together equal one calculate() (each cell bitwise the oracle's), and
    the cells a shard skips read as empty."""
    import vorothree_b200 as v
    pts = blobs(20000, 6, 0.03, 0.6, 91)
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(20, 20, 20))
    t.set_generators(pts)
    o = oracle_tess(oracle_mod, [0, 0, 0], [1, 1, 1], (20, 20, 20), pts)
    ov, oc, on = o.summaries()
    ooff, oids = o.neighbors()
    n = len(pts)
    chunk = 999
    seen = np.zeros(n, bool)
    for phase in range(stride):
        t.calculate_strided(chunk, stride, phase)
        gv, gc, gn = t.summaries()
        goff, gids = t.neighbors()
        mine = ((np.arange(n) // chunk) % stride) == phase
        assert np.array_equal(gv[mine], ov[mine]) and np.array_equal(gn[mine], on[mine])
        assert np.array_equal(gc[mine], oc[mine])
        assert not gv[~mine].any() and not gn[~mine].any()
        for i in np.nonzero(mine)[0][::97]:
            assert np.array_equal(gids[goff[i]:goff[i + 1]], oids[ooff[i]:ooff[i + 1]])
        assert t.get_cell(int(np.nonzero(~mine)[0][0])).face_neighbors().size == 0
        seen |= mine
    assert seen.all()
    with pytest.raises(v.VoronoidError):
        t.export_cells(0, 10)
    t.close()


@pytest.mark.parametrize("kind,n", [("central", 3000), ("axes", 3000), ("sphere", 1000), ("uniform", 20000)])
def test_batched_plane_tests_bitwise(oracle_mod, kind, n):
    """The walk's variant that tests the candidates' planes together after a
    run of clips that changed nothing (tuning noop_run) passes over exactly
    the clips the reference makes without effect: every cell equals the
    oracle's, bit for bit, on the reference's bench distributions (the
    central box's edge cells clip with thousands of candidates, nearly all
    without effect)."""
    import vorothree_b200 as v
    from common import bench_distribution
    pts = bench_distribution(kind, n, 90 + len(kind))
    g = int(np.ceil(n ** (1.0 / 3.0)))
    o = oracle_tess(oracle_mod, [0, 0, 0], [100, 100, 100], (g, g, g), pts)
    for run, layout in ((1, "slots"), (3, "slots"), (2, "full")):
        t = v.Tessellation(v.BoundingBox([0, 0, 0], [100, 100, 100]), v.Algorithm3DGrid(g, g, g))
        t.set_tuning({"noop_run": run, "fast_layout": layout})
        assert t.get_tuning()["noop_run"] == run
        t.set_generators(pts)
        t.calculate()
        assert_same(t, o, check_counters=False)
        t.close()


@pytest.mark.parametrize("m", [4, 5])
def test_symmetric_hub_cell_bitwise(oracle_mod, m):
    """A centre generator and one generator in every primitive lattice
    direction (|coordinates| <= m) on a sphere: the centre's cell (578 faces at
    m = 4, 1,154 at m = 5) reaches the block-per-cell tier, and the symmetric
    directions make many planes meet at one point (the reference keeps a
    vertex per plane triple there: 3,456 vertices at m = 4).  The slot layout
    follows the reference's vertices there too; every cell equals the
    oracle's bit for bit."""
    import itertools
    import math
    dirs = [v for v in itertools.product(range(-m, m + 1), repeat=3)
            if v != (0, 0, 0) and math.gcd(math.gcd(abs(v[0]), abs(v[1])), abs(v[2])) == 1]
    d = np.asarray(dirs, np.float64)
    d /= np.linalg.norm(d, axis=1)[:, None]
    pts = np.vstack([[50.0, 50.0, 50.0], 50.0 + 30.0 * d])
    g = int(np.ceil(len(pts) ** (1.0 / 3.0)))
    gt = gpu_tess([0, 0, 0], [100, 100, 100], (g, g, g), pts)
    o = oracle_tess(oracle_mod, [0, 0, 0], [100, 100, 100], (g, g, g), pts)
    assert gt.summaries()[2][0] == len(pts) - 1
    assert_same(gt, o, sample_cells=4)


def test_hub_cell_with_walls_and_batched_plane_tests(oracle_mod):
    """The centre of generators on a sphere (a cell the block-per-cell tier
    builds on the slot layout) with a plane wall and a sphere wall clipping it
    first, and the same input with the walk's batched plane tests on: every
    cell equals the oracle's, bit for bit."""
    import vorothree_b200 as v
    from common import bench_distribution
    pts = bench_distribution("sphere", 2500, 77)
    walls = [v.Wall(WALL, v.PlaneGeometry([50.0, 50.0, 58.0], [-0.1, -0.2, -1.0])),
             v.Wall(WALL - 1, v.SphereGeometry([50.0, 50.0, 50.0], 40.0))]
    g = int(np.ceil(len(pts) ** (1.0 / 3.0)))
    o = oracle_tess(oracle_mod, [0, 0, 0], [100, 100, 100], (g, g, g), pts, walls)
    for run in (-1, 4):
        t = v.Tessellation(v.BoundingBox([0, 0, 0], [100, 100, 100]), v.Algorithm3DGrid(g, g, g))
        t.set_tuning({"noop_run": run})
        t.set_generators(pts)
        for w in walls:
            t.add_wall(w)
        t.calculate()
        assert t.summaries()[2][0] > 500
        assert_same(t, o, check_counters=False)
        t.close()
