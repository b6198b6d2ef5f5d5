"""GPU: cylinder, cone, torus and convex-polyhedron walls (wall_3d.rs:107-365,
462-708) bit for bit against the oracle, alone and combined, with the walls
added before and after the generators, in both precisions; plus the
reference's own volume tests for these walls (tests/volumes.rs:68-105)."""
import math

import numpy as np
import pytest

from common import uniform
from test_gpu_parity import PRECISIONS, assert_same, gpu_tess

pytestmark = pytest.mark.gpu

WALL = -1000


def oracle_add(t, w):
    import vorothree_b200 as v
    g = w.geometry
    if isinstance(g, v.PlaneGeometry):
        t.add_wall_plane(g.point, g.normal, w.id())
    elif isinstance(g, v.SphereGeometry):
        t.add_wall_sphere(g.center, g.radius, w.id())
    elif isinstance(g, v.CylinderGeometry):
        t.add_wall_cylinder(g.center, g.axis, g.radius, w.id())
    elif isinstance(g, v.ConeGeometry):
        t.add_wall_cone(g.tip, g.axis, g.angle, w.id())
    elif isinstance(g, v.TorusGeometry):
        t.add_wall_torus(g.center, g.axis, g.major_radius, g.minor_radius, w.id())
    else:
        t.add_wall_polyhedron(g.points, g.normals, w.id())


def oracle_tess(oracle_mod, bmin, bmax, grid, pts, walls, walls_first):
    t = oracle_mod.OracleTessellation(bmin, bmax, *grid)
    if walls_first:
        for w in walls:
            oracle_add(t, w)
        t.set_generators(pts)
    else:
        t.set_generators(pts)
        for w in walls:
            oracle_add(t, w)
    t.calculate()
    return t


def wall_sets():
    import vorothree_b200 as v
    P = v.ConvexPolyhedronGeometry
    return {
        "cylinder": [v.Wall(WALL, v.CylinderGeometry([5, 5, 5], [0.2, 0.1, 1.0], 4.0))],
        "cone": [v.Wall(WALL, v.ConeGeometry([5, 5, -1], [0.1, 0.0, 1.0], 0.45))],
        "torus": [v.Wall(WALL, v.TorusGeometry([5, 5, 5], [0.0, 0.3, 1.0], 3.0, 1.6))],
        "tetrahedron": [v.Wall(WALL, P.new_tetrahedron([5, 5, 5], 4.5))],
        "hexahedron": [v.Wall(WALL, P.new_hexahedron([5, 5, 5], 4.5))],
        "octahedron": [v.Wall(WALL, P.new_octahedron([5, 5, 5], 4.5))],
        "dodecahedron": [v.Wall(WALL, P.new_dodecahedron([5, 5, 5], 4.5))],
        "icosahedron": [v.Wall(WALL, P.new_icosahedron([5, 5, 5], 4.5))],
        "combined": [v.Wall(WALL, v.CylinderGeometry([5, 5, 5], [0, 0, 1], 4.5)),
                     v.Wall(WALL - 1, v.PlaneGeometry([5, 5, 5], [0.3, -1.0, 0.2])),
                     v.Wall(WALL - 2, P.new_dodecahedron([5, 5, 5], 6.0)),
                     v.Wall(WALL - 3, v.SphereGeometry([5, 5, 5], 5.5))],
    }


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("name", ["cylinder", "cone", "torus", "tetrahedron", "hexahedron", "octahedron",
                                  "dodecahedron", "icosahedron", "combined"])
@pytest.mark.parametrize("walls_first", [True, False])
def test_walls_bitwise(oracle_mod, name, walls_first, precision):
    walls = wall_sets()[name]
    pts = uniform(4000, 0.0, 10.0, 30)
    g = gpu_tess([0, 0, 0], [10, 10, 10], (8, 8, 8), pts, walls, walls_first=walls_first, precision=precision)
    o = oracle_tess(oracle_mod, [0, 0, 0], [10, 10, 10], (8, 8, 8), pts, walls, walls_first)
    assert g.count_generators() > 100
    assert_same(g, o, sample_cells=6)


def lattice(size=10.0, n=20):
    step = size / n
    ax = np.arange(n) * step + step / 2
    return np.array([[x, y, z] for x in ax for y in ax for z in ax])


def test_reference_wall_volumes():
    import vorothree_b200 as v
    # tests/volumes.rs:68-105: cylinder and dodecahedron on the 20^3 lattice, grid 5^3, within 1%
    cases = [(v.CylinderGeometry([5, 5, 5], [0, 0, 1], 4.0), math.pi * 16.0 * 10.0)]
    xi = math.sqrt((5.0 + 2.0 * math.sqrt(5.0)) / 15.0)
    a = 2.0 * 4.0 * xi * math.sqrt(10.0) / math.sqrt(25.0 + 11.0 * math.sqrt(5.0))
    cases.append((v.ConvexPolyhedronGeometry.new_dodecahedron([5, 5, 5], 4.0),
                  (15.0 + 7.0 * math.sqrt(5.0)) / 4.0 * a ** 3))
    for geom, exp in cases:
        t = v.Tessellation(v.BoundingBox([0, 0, 0], [10, 10, 10]), v.Algorithm3DGrid(5, 5, 5))
        t.set_generators(lattice())
        t.add_wall(v.Wall(WALL, geom))
        t.calculate()
        vol, _, _ = t.summaries()
        assert abs(vol.sum() - exp) / exp < 0.01


def test_wall_errors():
    import vorothree_b200 as v
    with pytest.raises(ValueError):
        v.Wall(-5, v.CylinderGeometry([0, 0, 0], [0, 0, 1], 1.0))
    with pytest.raises(ValueError):
        v.ConvexPolyhedronGeometry([0, 0, 0, 1, 1, 1], [0, 0, 1])
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(2, 2, 2))
    big = v.ConvexPolyhedronGeometry(np.zeros((257, 3)), np.tile([0.0, 0.0, 1.0], (257, 1)))
    with pytest.raises(v.VoronoidError):
        t.add_wall(v.Wall(WALL, big))


@pytest.mark.parametrize("name", ["cylinder", "cone", "torus", "dodecahedron", "combined"])
def test_set_generator_under_walls_bitwise(oracle_mod, name):
    """Tessellation::set_generator (tessellation.rs:70-92) tests the new point
    against every wall kind before Algorithm3DGrid::update_generator
    (algo_3d_grid.rs:132-143) moves it between bins: moves the walls reject and
    out-of-range indices change nothing, accepted ones follow the reference's
    swap_remove/push bin order."""
    walls = wall_sets()[name]
    pts = uniform(3000, 0.0, 10.0, 31)
    g = gpu_tess([0, 0, 0], [10, 10, 10], (8, 8, 8), pts, walls, walls_first=True)
    o = oracle_tess(oracle_mod, [0, 0, 0], [10, 10, 10], (8, 8, 8), pts, walls, True)
    n = g.count_generators()
    assert n == o.count_generators()
    rng = np.random.Generator(np.random.PCG64(32))
    moves = [(int(rng.integers(0, n)), rng.uniform(0.0, 10.0, 3)) for _ in range(60)]
    moves += [(n, [5.0, 5.0, 5.0]), (n + 7, [5.0, 5.0, 5.0])]
    for i, p in moves:
        g.set_generator(i, p)
        o.set_generator(i, p)
    assert np.array_equal(g.generators(), o.generators())
    g.calculate()
    o.calculate()
    assert_same(g, o, sample_cells=6)


@pytest.mark.parametrize("name,count", [("torus", 3000), ("dodecahedron", 2500), ("combined", 20000)])
def test_random_generators_bitwise(oracle_mod, name, count):
    """Tessellation::random_generators (tessellation.rs:96-121), seeded: the
    device's batched candidates and wall filter keep the oracle's points (the
    first `count` inside the walls in attempt order), and the cells match."""
    import vorothree_b200 as v
    walls = wall_sets()[name]
    g = v.Tessellation(v.BoundingBox([0, 0, 0], [10, 10, 10]), v.Algorithm3DGrid(8, 8, 8))
    g.set_instrumentation(True)
    o = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 8, 8, 8)
    for w in walls:
        g.add_wall(w)
        oracle_add(o, w)
    seed = 0x5EED0000 + count
    assert g.random_generators(count, seed) == o.random_generators(count, seed) == count
    g.calculate()
    o.calculate()
    assert_same(g, o, sample_cells=4)


def test_random_generators_attempt_cap(oracle_mod):
    # ~2000 attempts per accepted point: the count * 1000 cap ends the loop
    # early, after the same attempts on both sides
    import vorothree_b200 as v
    g = v.Tessellation(v.BoundingBox([0, 0, 0], [10, 10, 10]), v.Algorithm3DGrid(4, 4, 4))
    o = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 4, 4, 4)
    g.add_wall(v.Wall(WALL, v.SphereGeometry([5, 5, 5], 0.492)))
    o.add_wall_sphere([5, 5, 5], 0.492, WALL)
    for seed in (7, 8, 9):
        n = g.random_generators(50, seed)
        assert n == o.random_generators(50, seed) and 5 < n < 50
        assert np.array_equal(g.generators(), o.generators())
    assert g.random_generators(0, 1) == 0 and g.count_generators() == 0


def _random_wall(rng, lo, hi, k):
    """A wall of a random kind around the box's middle, sized to keep a good
    share of the generators."""
    import vorothree_b200 as v
    c = lo + (hi - lo) * rng.uniform(0.4, 0.6, 3)
    ext = float(np.linalg.norm(hi - lo)) / 2.0
    axis = rng.normal(size=3)
    kind = int(rng.integers(0, 6))
    wid = WALL - k
    if kind == 0:
        return v.Wall(wid, v.PlaneGeometry(list(c), list(axis)))
    if kind == 1:
        return v.Wall(wid, v.SphereGeometry(list(c), ext * rng.uniform(0.6, 0.9)))
    if kind == 2:
        return v.Wall(wid, v.CylinderGeometry(list(c), list(axis), ext * rng.uniform(0.5, 0.8)))
    if kind == 3:
        tip = c - axis / np.linalg.norm(axis) * ext * 1.5
        return v.Wall(wid, v.ConeGeometry(list(tip), list(axis), rng.uniform(0.7, 1.2)))
    if kind == 4:
        return v.Wall(wid, v.TorusGeometry(list(c), list(axis), ext * 0.45, ext * rng.uniform(0.35, 0.45)))
    P = v.ConvexPolyhedronGeometry
    maker = [P.new_tetrahedron, P.new_hexahedron, P.new_octahedron, P.new_dodecahedron, P.new_icosahedron][
        int(rng.integers(0, 5))]
    return v.Wall(wid, maker(list(c), ext * rng.uniform(0.9, 1.3)))


@pytest.mark.parametrize("seed", range(12))
def test_random_configurations_bitwise(oracle_mod, seed):
    """Random boxes, grids, generator distributions and 0-3 walls of random
    kinds, in both precisions: every cell equal to the oracle's."""
    from common import bench_distribution
    rng = np.random.Generator(np.random.PCG64(500 + seed))
    lo = rng.uniform(-50, 50, 3)
    hi = lo + rng.uniform(0.5, 20, 3)
    n = int(rng.integers(500, 4000))
    kind = ["uniform", "axes", "central", "uniform"][seed % 4]
    pts = bench_distribution(kind, n, 600 + seed, lo, hi)
    grid = tuple(int(x) for x in rng.integers(1, 16, 3))
    walls = [_random_wall(rng, lo, hi, k) for k in range(int(rng.integers(0, 4)))]
    precision = "mixed" if seed % 3 == 2 else "fp64"
    g = gpu_tess(list(lo), list(hi), grid, pts, walls, walls_first=bool(seed % 2), precision=precision)
    o = oracle_tess(oracle_mod, list(lo), list(hi), grid, pts, walls, bool(seed % 2))
    assert_same(g, o, check_counters=(precision == "fp64"), sample_cells=4)
