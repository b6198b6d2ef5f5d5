"""GPU: bulk polytope export (vd_tess_export_cells) behind Tessellation.cells
and Tessellation.map (tessellation.rs:391-412, 524-526): every cell equal, bit
for bit, to what get_cell gives -- cells rebuilt by the device pass, cells
left to get_cell's larger tiers, cells outside a calculate_range (empty), and
the sealed polytopes."""
import numpy as np
import pytest

from common import uniform
from test_gpu_parity import gpu_tess

pytestmark = pytest.mark.gpu

WALL = -1000


def assert_export_matches(t, begin=0, end=None, only=None):
    x = t.export_cells(begin, end)
    end = t.count_cells() if end is None else end
    vo, fo, ho = x["v_off"], x["f_off"], x["h_off"]
    assert len(vo) == end - begin + 1
    for k in (range(end - begin) if only is None else only):
        c = t.get_cell(begin + k)
        assert np.array_equal(x["vertices"][3 * vo[k]:3 * vo[k + 1]], c.vertices().reshape(-1)), k
        assert np.array_equal(x["face_counts"][fo[k]:fo[k + 1]], c.face_counts()), k
        assert np.array_equal(x["face_indices"][ho[k]:ho[k + 1]], c.face_indices()), k
        assert np.array_equal(x["face_neighbors"][fo[k]:fo[k + 1]], c.face_neighbors()), k
    return x


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_export_equals_get_cell(precision):
    import vorothree_b200 as v
    walls = [v.Wall(WALL, v.SphereGeometry([0.5, 0.5, 0.5], 0.48))]
    t = gpu_tess([0, 0, 0], [1, 1, 1], (8, 8, 8), uniform(3000, 0, 1, 61), walls, precision=precision)
    x = assert_export_matches(t)
    assert x["v_off"][-1] > 20 * t.count_cells()
    # sub-ranges, and an empty one
    assert_export_matches(t, 100, 357)
    e = t.export_cells(5, 5)
    assert e["v_off"].tolist() == [0] and e["vertices"].size == 0


def test_export_overflow_cells():
    # a dense blob on a coarse grid: some cells outgrow the shared-memory
    # capacities and are rebuilt by the medium and large export tiers
    rng = np.random.Generator(np.random.PCG64(17))
    pts = np.concatenate([0.5 + rng.normal(0.0, 0.01, size=(2500, 3)), rng.uniform(0, 1, size=(300, 3))])
    t = gpu_tess([0, 0, 0], [1, 1, 1], (4, 4, 4), pts)
    assert t.fallback_counts()["overflow"] > 0
    # every cell's face count; whole polytopes for the blob cells (where the
    # overflowing ones are) and a sample of the rest
    _, _, nf = t.summaries()
    x = t.export_cells()
    assert np.array_equal(np.diff(x["f_off"]), nf)
    assert_export_matches(t, only=sorted(set(range(0, 2500, 7)) | set(range(2500, 2800, 25))))


def test_export_after_calculate_range():
    t = gpu_tess([0, 0, 0], [1, 1, 1], (6, 6, 6), uniform(1200, 0, 1, 62))
    t.calculate_range(300, 700)
    x = assert_export_matches(t, 250, 750)
    sizes = np.diff(x["v_off"])
    assert (sizes[:50] == 0).all() and (sizes[-50:] == 0).all() and (sizes[50:450] > 0).all()


def test_export_sealed():
    import vorothree_b200 as v
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [10, 10, 10]), v.Algorithm3DGrid(6, 6, 6))
    t.set_generators(uniform(800, 0, 10, 63))
    t.add_wall(v.Wall(WALL, v.CylinderGeometry([5, 5, 5], [0, 0.2, 1], 4.0)))
    t.calculate_sealed()
    assert_export_matches(t, 0, 120)


def test_cells_and_map():
    t = gpu_tess([0, 0, 0], [1, 1, 1], (5, 5, 5), uniform(400, 0, 1, 64))
    cells = t.cells()
    assert len(cells) == 400
    for i in (0, 17, 399):
        c = t.get_cell(i)
        assert np.array_equal(cells[i].vertices(), c.vertices())
        assert np.array_equal(cells[i].face_indices(), c.face_indices())
    vol, _, nf = t.summaries()
    got = t.map(lambda c: (c.volume(), len(c.face_counts())))
    assert [g[0] for g in got] == vol.tolist() and [g[1] for g in got] == nf.tolist()


@pytest.mark.parametrize("n", [90, 400])
def test_export_large_cell(n):
    # the centre of generators on a sphere with n-1 faces: 89 fit the medium
    # tier, 399 only the large one (global scratch)
    from common import bench_distribution
    t = gpu_tess([0, 0, 0], [100, 100, 100], (6, 6, 6), bench_distribution("sphere", n, 83))
    x = assert_export_matches(t)
    assert x["f_off"][1] - x["f_off"][0] == n - 1


def test_export_sealed_large_cell():
    import vorothree_b200 as v
    from common import bench_distribution
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [100, 100, 100]), v.Algorithm3DGrid(6, 6, 6))
    t.set_generators(bench_distribution("sphere", 400, 84))
    t.add_wall(v.Wall(WALL, v.CylinderGeometry([50, 50, 50], [0.1, 0.2, 1], 45.0)))
    t.calculate_sealed()
    x = assert_export_matches(t)
    assert x["f_off"][1] - x["f_off"][0] >= 399


def test_export_huge_cell():
    # the centre of generators on a sphere: a cell only the huge tier holds,
    # exported through get_cell
    from common import bench_distribution
    t = gpu_tess([0, 0, 0], [100, 100, 100], (12, 12, 12), bench_distribution("sphere", 1500, 82))
    x = assert_export_matches(t, 0, 40)
    assert x["f_off"][1] - x["f_off"][0] == 1499
