"""GPU: the first tier's two polytope layouts give the same tessellation.

The slot layout (default) rewrites only the faces a clip cuts and keeps each
untouched face's rotation as a counter; the full layout rewrites every face
loop per clip, as the reference does.  Every output -- volumes, centroids,
face counts, neighbour ids in face order, face areas -- must be identical
between them and equal to the oracle's, on inputs that exercise the slot
layout's hand-off to the medium tier (lattices, whose vertices sit in the
1e-9 band; dense clusters; walls), in both precisions, for single
tessellations and for batches.
"""
import numpy as np
import pytest

from common import blobs, uniform

pytestmark = pytest.mark.gpu

WALL = -1000


def run(bmin, bmax, grid, pts, layout, precision="fp64", walls=()):
    import vorothree_b200 as v
    t = v.Tessellation(v.BoundingBox(bmin, bmax), v.Algorithm3DGrid(*grid))
    t.set_precision(precision)
    t.set_fast_layout(layout)
    for w in walls:
        t.add_wall(w)
    t.set_generators(pts)
    t.calculate()
    out = t.summaries() + (t.neighbors()[1], t.face_areas()[1], t.fallback_counts())
    t.close()
    return out


def oracle_run(oracle_mod, bmin, bmax, grid, pts, walls=()):
    o = oracle_mod.OracleTessellation(bmin, bmax, *grid)
    for w in walls:
        g = w.geometry
        if hasattr(g, "radius"):
            o.add_wall_sphere(g.center, g.radius, w.id())
        else:
            o.add_wall_plane(g.point, g.normal, w.id())
    o.set_generators(pts)
    o.calculate()
    return o.summaries() + (o.neighbors()[1], o.face_areas()[1])


def lattice(n):
    a = (np.arange(n) + 0.5) / n
    return np.stack(np.meshgrid(a, a, a, indexing="ij"), -1).reshape(-1, 3)


def cases():
    import vorothree_b200 as v
    return [
        ("uniform", [0, 0, 0], [1, 1, 1], (20, 20, 20), uniform(30000, 0.0, 1.0, 51), ()),
        ("blobs", [0, 0, 0], [1, 1, 1], (24, 24, 24), np.clip(blobs(20000, 6, 0.02, 0.8, 52), 0, 1), ()),
        ("lattice", [0, 0, 0], [1, 1, 1], (10, 10, 10), lattice(12), ()),
        ("jittered lattice", [0, 0, 0], [1, 1, 1], (10, 10, 10),
         lattice(12) + np.random.Generator(np.random.PCG64(53)).normal(0, 1e-12, size=(1728, 3)), ()),
        ("sphere wall", [0, 0, 0], [1, 1, 1], (16, 16, 16), uniform(12000, 0.0, 1.0, 54),
         (v.Wall(WALL, v.SphereGeometry([0.5, 0.5, 0.5], 0.4)),)),
        ("plane walls", [0, 0, 0], [1, 1, 1], (16, 16, 16), uniform(12000, 0.0, 1.0, 55),
         (v.Wall(WALL, v.PlaneGeometry([0.5, 0.5, 0.5], [1, 1, 0])),
          v.Wall(WALL - 1, v.PlaneGeometry([0.3, 0.3, 0.3], [0, 0, 1])))),
    ]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_layouts_equal_and_equal_the_oracle(oracle_mod, precision):
    for name, bmin, bmax, grid, pts, walls in cases():
        a = run(bmin, bmax, grid, pts, "slots", precision, walls)
        b = run(bmin, bmax, grid, pts, "full", precision, walls)
        o = oracle_run(oracle_mod, bmin, bmax, grid, pts, walls)
        for k in range(5):
            assert np.array_equal(a[k], b[k]), (name, k)
            assert np.array_equal(a[k], o[k]), (name, k)


def test_uniform_input_stays_in_the_slot_tier():
    """General-position input: the slot layout finishes (nearly) every cell
    itself; the hand-off to the medium tier is for degenerate cells."""
    a = run([0, 0, 0], [1, 1, 1], (40, 40, 40), uniform(100000, 0.0, 1.0, 56), "slots")
    assert a[5]["overflow"] < 100, a[5]


def test_batch_layouts_equal():
    import vorothree_b200 as v
    from vorothree_b200.workloads import batch_members
    members = batch_members(48, 57)
    res = {}
    for layout in ("slots", "full"):
        b = v.TessellationBatch()
        b.set_fast_layout(layout)
        for edge, grid, pts, sphere in members:
            walls = [v.Wall(v.WALL_ID_MAX, v.SphereGeometry(*sphere))] if sphere else []
            b.add(v.BoundingBox([0, 0, 0], list(edge)), grid, pts, walls)
        b.commit()
        b.calculate()
        b.lloyd(2)
        res[layout] = [b.summaries(i) for i in range(len(members))]
        b.close()
    for x, y in zip(res["slots"], res["full"]):
        for k in range(3):
            assert np.array_equal(x[k], y[k])
