"""GPU parity at the benchmark configurations' full sizes.

The other parity tests run 1k-100k generators; these run the inputs the
benchmark times, through the same public API, and compare every cell with the
oracle bit for bit:
  * 1,048,576 generators uniform in the unit cube, grid 100^3, no walls, in
    both precisions (FP64, and FP32 classification under its error bound);
  * 4,194,304 generators, 70% in 64 Gaussian blobs (sigma 0.01) and 30%
    uniform, clipped by a sphere wall r = 0.45 at the centre, on the grid the
    autotuner picks for them (the oracle's search order is truncated there:
    the complete table of that grid does not fit in host memory, and a
    truncated one gives the same walk, which the oracle checks per cell);
  * the 4096-member batch (N log-uniform in [64, 65536], half with a sphere
    wall) in one launch, every member against its own oracle tessellation,
    and members after two Lloyd steps replayed from the captured graph.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NTHREADS = os.cpu_count() or 1


def oracle_with_table(oracle_mod, bmin, bmax, grid, pts, walls=(), k=0):
    """The oracle tessellation, with a truncated search order of k bins per
    axis (doubled until no cell walks off it) when k > 0."""
    while True:
        o = oracle_mod.OracleTessellation(bmin, bmax, *grid, order_k=k)
        for c, r in walls:
            o.add_wall_sphere(c, r, -1000)
        o.set_generators(pts)
        try:
            o.calculate(NTHREADS)
            return o
        except RuntimeError:
            assert k > 0
            k *= 2


def assert_bitwise(g, o):
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


@pytest.fixture(scope="module")
def uniform_1m(oracle_mod):
    from vorothree_b200.workloads import uniform_cube
    pts = uniform_cube(1_048_576, 0)
    return pts, oracle_with_table(oracle_mod, [0, 0, 0], [1, 1, 1], (100, 100, 100), pts)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_uniform_1m_grid100_bitwise(uniform_1m, precision):
    import vorothree_b200 as v
    pts, o = uniform_1m
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(100, 100, 100))
    t.set_precision(precision)
    t.set_generators(pts)
    t.calculate()
    assert t.count_cells() == 1_048_576
    assert_bitwise(t, o)
    t.close()


def test_clustered_4m_sphere_wall_autotuned_grid_bitwise(oracle_mod):
    import vorothree_b200 as v
    from vorothree_b200 import autotune
    from vorothree_b200.workloads import clustered_blobs
    pts, _ = clustered_blobs(4_194_304, 0)
    bounds = v.BoundingBox([0, 0, 0], [1, 1, 1])
    grid = autotune.choose_grid(pts, bounds)
    wall = ([0.5, 0.5, 0.5], 0.45)
    o = oracle_with_table(oracle_mod, [0, 0, 0], [1, 1, 1], grid, pts, [wall], k=32)
    for precision in ("mixed", "fp64"):
        t = v.Tessellation(bounds, v.Algorithm3DGrid(*grid))
        t.set_precision(precision)
        t.add_wall(v.Wall(v.WALL_ID_MAX, v.SphereGeometry(*wall)))
        kept = t.set_generators(pts)
        t.calculate()
        assert kept == o.count_generators() > 1_000_000
        assert sum(t.fallback_counts().values()) > 0  # the overflow tiers run at this size
        assert_bitwise(t, o)
        t.close()


@pytest.fixture(scope="module")
def batch_4096():
    import vorothree_b200 as v
    from vorothree_b200.workloads import batch_members
    members = batch_members(4096, 0)
    b = v.TessellationBatch()
    for edge, grid, pts, sphere in members:
        walls = [v.Wall(v.WALL_ID_MAX, v.SphereGeometry(*sphere))] if sphere else []
        b.add(v.BoundingBox([0, 0, 0], list(edge)), grid, pts, walls)
    b.commit()
    return members, b


def member_oracle(oracle_mod, member, relax_steps=0):
    """A batch member's oracle tessellation after `relax_steps` Lloyd steps;
    its truncated search order (large grids) is doubled and the whole chain
    redone whenever a cell walks off it."""
    edge, grid, pts, sphere = member
    walls = [sphere] if sphere else []
    k = 8 if (2 * grid[0] + 1) * (2 * grid[1] + 1) * (2 * grid[2] + 1) > 20000 else 0
    while True:
        o = oracle_with_table(oracle_mod, [0, 0, 0], list(edge), grid, pts, walls, k=k)
        try:
            for _ in range(relax_steps):
                o.relax()
                o.calculate(NTHREADS)
            return o
        except RuntimeError:
            assert k > 0
            k *= 2


def test_batch_4096_members_bitwise(oracle_mod, batch_4096):
    members, b = batch_4096
    b.calculate()
    assert b.total_cells() > 20_000_000
    for i, m in enumerate(members):
        o = member_oracle(oracle_mod, m)
        gv, gc, gn = b.summaries(i)
        ov, oc, on = o.summaries()
        assert np.array_equal(gn, on), (i, np.nonzero(gn != on)[0][:5])
        assert np.array_equal(gv, ov), i
        assert np.array_equal(gc, oc), i
        del o


def test_batch_4096_lloyd_steps_bitwise(oracle_mod, batch_4096):
    """Two Lloyd steps (the first eager, the second replayed from the graph it
    captures) on the whole batch; 64 members spread over the batch against
    the oracle's relax + calculate chain."""
    members, b = batch_4096
    b.calculate()
    b.lloyd(1)
    b.lloyd(1)
    for i in np.linspace(0, len(members) - 1, 64).astype(int):
        o = member_oracle(oracle_mod, members[i], relax_steps=2)
        assert np.array_equal(b.generators(int(i)), o.generators())
        gv, gc, gn = b.summaries(int(i))
        ov, oc, on = o.summaries()
        assert np.array_equal(gn, on), i
        assert np.array_equal(gv, ov), i
        assert np.array_equal(gc, oc), i
