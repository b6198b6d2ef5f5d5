"""GPU: the face pool -- face slots of cells with more than the 48 per-cell
slots (the medium, large and huge tiers' cells).

Cells that finish in the medium tier with 49-112 faces need pool slots on a
fresh handle, before any large-tier pass has run; a cell rebuilt alone by
get_cell must not move the other cells' pooled faces.  Each case compares the
neighbour ids and face areas with the oracle exactly.
"""
import numpy as np
import pytest

from common import bench_distribution

pytestmark = pytest.mark.gpu


def two_spheres(n_each, seed):
    """Two clusters, each a centre point surrounded by n_each points on a
    sphere of radius 12: each centre's cell has n_each faces."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for c in ([30.0, 50.0, 50.0], [70.0, 50.0, 50.0]):
        v = rng.normal(size=(n_each, 3))
        v /= np.linalg.norm(v, axis=1)[:, None]
        out.append(np.asarray([c]))
        out.append(np.asarray(c) + 12.0 * v)
    return np.concatenate(out)


def check_csr(g, o):
    gv, _, gn = g.summaries()
    ov, _, on = o.summaries()
    assert np.array_equal(gn, on)
    assert np.array_equal(gv, ov)
    goff, gids = g.neighbors()
    ooff, oids = o.neighbors()
    assert np.array_equal(goff, ooff)
    assert np.array_equal(gids, oids)
    _, gar = g.face_areas()
    _, oar = o.face_areas()
    assert np.array_equal(gar, oar)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_medium_tier_cells_on_a_fresh_handle(oracle_mod, precision):
    """80 points on a sphere around its centre, grid 5^3: the centre cell has
    79 faces and finishes in the medium tier, the first tier to use the pool
    on this handle."""
    import vorothree_b200 as v
    pts = bench_distribution("sphere", 80, 41)
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [100, 100, 100]), v.Algorithm3DGrid(5, 5, 5))
    t.set_precision(precision)
    t.set_generators(pts)
    t.calculate()
    o = oracle_mod.OracleTessellation([0, 0, 0], [100, 100, 100], 5, 5, 5)
    o.set_generators(pts)
    o.calculate()
    assert o.summaries()[2][0] == 79
    assert t.fallback_counts()["overflow"] > 0
    check_csr(t, o)


def test_get_cell_keeps_other_cells_pooled_faces(oracle_mod):
    """Two cells with 70 faces each share the pool; rebuilding one of them
    with get_cell (which finalizes it again) leaves the other's slots, and
    results read afterwards still equal the oracle's."""
    import vorothree_b200 as v
    pts = two_spheres(70, 42)
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [100, 100, 100]), v.Algorithm3DGrid(4, 4, 4))
    t.set_generators(pts)
    t.calculate()
    o = oracle_mod.OracleTessellation([0, 0, 0], [100, 100, 100], 4, 4, 4)
    o.set_generators(pts)
    o.calculate()
    on = o.summaries()[2]
    assert on[0] == 70 and on[71] == 70
    check_csr(t, o)
    for i in (71, 0, 71):
        gcell = t.get_cell(i)
        ov_, ofc, ofi, ofn = o.get_cell(i).export()
        assert np.array_equal(gcell.face_neighbors(), ofn)
    check_csr(t, o)


def test_pool_grows_across_tiers(oracle_mod):
    """Many cells beyond the per-cell slots in one tessellation: 40 clusters
    of a centre and 60 sphere points each (2,440 generators) on a coarse grid,
    so the medium tier pools 40 x 60 faces and the pool is sized before it."""
    import vorothree_b200 as v
    rng = np.random.Generator(np.random.PCG64(43))
    centres = rng.uniform(15.0, 85.0, size=(40, 3))
    pts = []
    for c in centres:
        d = rng.normal(size=(60, 3))
        d /= np.linalg.norm(d, axis=1)[:, None]
        pts.append(c[None, :])
        pts.append(c + 2.0 * d)
    pts = np.concatenate(pts)
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [100, 100, 100]), v.Algorithm3DGrid(8, 8, 8))
    t.set_generators(pts)
    t.calculate()
    o = oracle_mod.OracleTessellation([0, 0, 0], [100, 100, 100], 8, 8, 8)
    o.set_generators(pts)
    o.calculate()
    assert (o.summaries()[2] > 48).sum() >= 40
    check_csr(t, o)
