"""GPU: calculate_sealed and prune_boundaries (tessellation.rs:234-385)
bit for bit against the oracle: the sealed cells (summaries, neighbour ids,
face areas, sampled polytopes), the seal log, and the prune logs on sealed
and unsealed cells."""
import numpy as np
import pytest

from common import uniform
from test_gpu_parity import assert_same
from test_gpu_walls import oracle_add

pytestmark = pytest.mark.gpu

WALL = -1000


def walls_of(name):
    import vorothree_b200 as v
    return {
        "sphere": [v.Wall(WALL, v.SphereGeometry([5, 5, 5], 4.5))],
        "cylinder+plane": [v.Wall(WALL, v.CylinderGeometry([5, 5, 5], [0.1, 0.2, 1.0], 4.2)),
                           v.Wall(WALL - 1, v.PlaneGeometry([5, 5, 5], [1.0, 0.2, 0.0]))],
        "torus": [v.Wall(WALL, v.TorusGeometry([5, 5, 5], [0, 0, 1], 3.0, 1.8))],
        "cone+sphere": [v.Wall(WALL, v.ConeGeometry([5, 5, 0.5], [0, 0, 1], 0.5)),
                        v.Wall(WALL - 1, v.SphereGeometry([5, 5, 5], 4.8))],
        "dodecahedron": [v.Wall(WALL, v.ConvexPolyhedronGeometry.new_dodecahedron([5, 5, 5], 4.5))],
    }[name]


def pair(oracle_mod, name, n=4000, seed=40):
    import vorothree_b200 as v
    pts = uniform(n, 0.0, 10.0, seed)
    walls = walls_of(name)
    g = v.Tessellation(v.BoundingBox([0, 0, 0], [10, 10, 10]), v.Algorithm3DGrid(7, 7, 7))
    o = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 7, 7, 7)
    g.set_generators(pts)
    o.set_generators(pts)
    for w in walls:
        g.add_wall(w)
        oracle_add(o, w)
    return g, o


@pytest.mark.parametrize("name", ["sphere", "cylinder+plane", "torus", "cone+sphere", "dodecahedron"])
def test_sealed_and_pruned_bitwise(oracle_mod, name):
    g, o = pair(oracle_mod, name)
    # prune on the plain cells
    g.calculate()
    o.calculate()
    g.prune_boundaries()
    o.prune_boundaries()
    assert np.array_equal(g.prune_log, o.prune_log())
    assert np.array_equal(g.prune_pos_log, o.prune_pos_log())
    # sealed cells, their log, and prune on them
    g.calculate_sealed()
    o.calculate_sealed()
    assert_same(g, o, check_counters=False, sample_cells=12)
    assert np.array_equal(g.seal_log, o.seal_log())
    if name != "dodecahedron":
        assert len(g.seal_log) > 0
    else:
        assert len(g.seal_log) == 0  # planar walls are never sealed
    g.prune_boundaries()
    o.prune_boundaries()
    assert np.array_equal(g.prune_log, o.prune_log())
    assert np.array_equal(g.prune_pos_log, o.prune_pos_log())
    # calculate clears the logs
    g.calculate()
    assert len(g.seal_log) == 0 and len(g.prune_log) == 0


def test_sealed_dense_blob_and_relax(oracle_mod):
    """Sealing cells that need the large-capacity pass, then a relax step
    from the sealed centroids."""
    import vorothree_b200 as v
    rng = np.random.Generator(np.random.PCG64(41))
    pts = np.concatenate([5.0 + rng.normal(0.0, 0.3, size=(3000, 3)), rng.uniform(0, 10, size=(500, 3))])
    w = v.Wall(WALL, v.SphereGeometry([5, 5, 5], 1.2))
    g = v.Tessellation(v.BoundingBox([0, 0, 0], [10, 10, 10]), v.Algorithm3DGrid(3, 3, 3))
    o = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 3, 3, 3)
    for t in (g, o):
        t.set_generators(pts)
    g.add_wall(w)
    oracle_add(o, w)
    g.calculate_sealed()
    o.calculate_sealed()
    assert_same(g, o, check_counters=False, sample_cells=4)
    assert np.array_equal(g.seal_log, o.seal_log())
    g.relax()
    o.relax()
    g.calculate_sealed()
    o.calculate_sealed()
    assert_same(g, o, check_counters=False, sample_cells=4)
    assert np.array_equal(g.seal_log, o.seal_log())


def test_sealed_huge_cell(oracle_mod):
    """A cell that only the block tier holds, sealed: the centre of generators
    on a sphere inside a cylinder wall is adjacent to the ~2,000 sphere
    generators the wall keeps and gains ~1,400 seal clips (3,469 faces); the
    seal pass rebuilds it with a thread block, bit for bit the oracle's."""
    import vorothree_b200 as v
    from common import bench_distribution
    pts = bench_distribution("sphere", 10000, 93)
    w = v.Wall(WALL, v.CylinderGeometry([50.3, 50, 50], [0, 0, 1], 20.0))
    g = v.Tessellation(v.BoundingBox([0, 0, 0], [100, 100, 100]), v.Algorithm3DGrid(13, 13, 13))
    o = oracle_mod.OracleTessellation([0, 0, 0], [100, 100, 100], 13, 13, 13)
    for t in (g, o):
        t.set_generators(pts)
    g.add_wall(w)
    oracle_add(o, w)
    g.calculate_sealed()
    o.calculate_sealed()
    assert g.summaries()[2][0] == 3469
    assert_same(g, o, check_counters=False, sample_cells=3)
    assert np.array_equal(g.seal_log, o.seal_log())
    g.prune_boundaries()
    o.prune_boundaries()
    assert np.array_equal(g.prune_log, o.prune_log())
    assert np.array_equal(g.prune_pos_log, o.prune_pos_log())
