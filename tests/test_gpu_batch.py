"""GPU: batches of tessellations (vd_batch_*) against standalone tessellations.

Every batch member must equal, bit for bit, a standalone Tessellation built
from the same bounds, grid, walls and generators (which itself equals the
oracle bit for bit, see test_gpu_parity.py) -- after calculate and after
every Lloyd step.
"""
import numpy as np
import pytest

from common import blobs, uniform

pytestmark = pytest.mark.gpu

WALL = -1000


def members(seed=0):
    import vorothree_b200 as v
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    # (bounds, grid, generators, walls)
    out.append(([0, 0, 0], [1, 1, 1], (10, 10, 10), uniform(1000, 0, 1, seed + 1), []))
    out.append(([0, 0, 0], [3, 1, 2], (9, 3, 6), uniform(700, 0, 1, seed + 2) * [3, 1, 2], []))
    out.append(([0, 0, 0], [10, 10, 10], (8, 8, 8), uniform(3000, 0, 10, seed + 3),
                [v.Wall(WALL, v.SphereGeometry([5, 5, 5], 4.0))]))
    out.append(([-1, -1, -1], [1, 1, 1], (4, 4, 4), uniform(64, -1, 1, seed + 4),
                [v.Wall(WALL, v.PlaneGeometry([0, 0, 0], [1, 1, 0])),
                 v.Wall(WALL - 1, v.SphereGeometry([0, 0, 0], 0.9))]))
    out.append(([0, 0, 0], [1, 1, 1], (3, 3, 3), np.zeros((0, 3)), []))  # empty member
    out.append(([0, 0, 0], [1, 1, 1], (5, 5, 5), uniform(50, 0, 1, seed + 5),
                [v.Wall(WALL, v.SphereGeometry([5, 5, 5], 0.1))]))  # wall removes all
    out.append(([0, 0, 0], [1, 1, 1], (20, 20, 20), blobs(5000, 4, 0.02, 0.7, seed + 6),
                [v.Wall(WALL, v.SphereGeometry([0.5, 0.5, 0.5], 0.45))]))
    sizes = np.exp(rng.uniform(np.log(64), np.log(4096), size=6)).round().astype(int)
    for k, n in enumerate(sizes):
        edge = rng.uniform(1, 10, size=3)
        g = int(np.ceil(n ** (1 / 3)))
        walls = [v.Wall(WALL, v.SphereGeometry(list(edge / 2), 0.5 * edge.min()))] if k % 2 == 0 else []
        out.append(([0, 0, 0], list(edge), (g, g, g), uniform(int(n), 0, 1, seed + 10 + k) * edge, walls))
    return out


def standalone(m, precision="fp64"):
    import vorothree_b200 as v
    bmin, bmax, grid, pts, walls = m
    t = v.Tessellation(v.BoundingBox(bmin, bmax), v.Algorithm3DGrid(*grid))
    t.set_precision(precision)
    for w in walls:
        t.add_wall(w)
    t.set_generators(pts)
    t.calculate()
    return t


def build_batch(ms, precision="fp64"):
    import vorothree_b200 as v
    b = v.TessellationBatch()
    b.set_precision(precision)
    for bmin, bmax, grid, pts, walls in ms:
        b.add(v.BoundingBox(bmin, bmax), grid, pts, walls)
    b.commit()
    b.calculate()
    return b


def assert_member_equal(b, k, t):
    assert b.count_cells(k) == t.count_cells() == t.count_generators()
    assert np.array_equal(b.generators(k), t.generators())
    bv, bc, bn = b.summaries(k)
    tv, tc, tn = t.summaries()
    assert np.array_equal(bn, tn), k
    assert np.array_equal(bv, tv), k
    assert np.array_equal(bc, tc), k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_standalone(precision):
    ms = members(0)
    b = build_batch(ms, precision)
    for k, m in enumerate(ms):
        assert_member_equal(b, k, standalone(m, precision))
    assert b.count_cells(4) == 0 and b.count_cells(5) == 0


def test_batch_lloyd_equals_repeated_relax():
    ms = members(1)
    b = build_batch(ms)
    ts = [standalone(m) for m in ms]
    for step in range(3):
        b.lloyd(1)
        for t in ts:
            t.relax()
            t.calculate()
        for k, t in enumerate(ts):
            assert_member_equal(b, k, t)
    # several steps in one call replay the captured graph
    b.lloyd(2)
    for t in ts:
        for _ in range(2):
            t.relax()
            t.calculate()
    for k, t in enumerate(ts):
        assert_member_equal(b, k, t)


def test_batch_table_extension():
    # a member on a large grid with few generators must lengthen its search order
    ms = [([0, 0, 0], [1, 1, 1], (80, 80, 80), uniform(300, 0, 1, 6), []),
          ([0, 0, 0], [1, 1, 1], (10, 10, 10), uniform(1000, 0, 1, 7), [])]
    b = build_batch(ms)
    for k, m in enumerate(ms):
        assert_member_equal(b, k, standalone(m))


def test_batch_volumes_fill_boxes():
    ms = [m for m in members(2) if not m[4]]
    b = build_batch(ms)
    for k, (bmin, bmax, grid, pts, walls) in enumerate(ms):
        if len(pts) == 0:
            continue
        vol, _, _ = b.summaries(k)
        box = np.prod(np.subtract(bmax, bmin))
        assert abs(vol.sum() - box) < 1e-9 * box


def test_batch_dense_blob_overflow_tiers():
    rng = np.random.Generator(np.random.PCG64(18))
    dense = np.concatenate([0.5 + rng.normal(0.0, 0.01, size=(2500, 3)), rng.uniform(0, 1, size=(300, 3))])
    ms = [([0, 0, 0], [1, 1, 1], (4, 4, 4), dense, []),
          ([0, 0, 0], [1, 1, 1], (10, 10, 10), uniform(1000, 0, 1, 19), [])]
    b = build_batch(ms)
    for k, m in enumerate(ms):
        assert_member_equal(b, k, standalone(m))


def test_batch_and_server_take_every_wall_kind():
    """Batch members and served requests with cylinder, cone, torus and
    polyhedron walls equal standalone tessellations bit for bit."""
    import vorothree_b200 as v
    P = v.ConvexPolyhedronGeometry
    wallsets = [
        [v.Wall(WALL, v.CylinderGeometry([5, 5, 5], [0.1, 0.0, 1.0], 4.0))],
        [v.Wall(WALL, v.ConeGeometry([5, 5, 0.5], [0, 0, 1], 0.5))],
        [v.Wall(WALL, v.TorusGeometry([5, 5, 5], [0, 1, 1], 3.0, 1.7))],
        [v.Wall(WALL, P.new_icosahedron([5, 5, 5], 4.5)), v.Wall(WALL - 1, P.new_tetrahedron([5, 5, 5], 6.0))],
    ]
    ms = [([0, 0, 0], [10, 10, 10], (7, 7, 7), uniform(3000, 0, 10, 60 + k), w) for k, w in enumerate(wallsets)]
    b = build_batch(ms)
    srv = v.TessellationServer(slots=2, hbm_budget_bytes=4 << 30)
    tickets = [srv.submit(v.BoundingBox(m[0], m[1]), m[2], m[3], m[4]) for m in ms]
    for k, m in enumerate(ms):
        t = standalone(m)
        assert_member_equal(b, k, t)
        vol, cen, nf = srv.take(tickets[k])
        tv, tc, tn = t.summaries()
        assert np.array_equal(vol, tv) and np.array_equal(cen, tc) and np.array_equal(nf, tn)
    srv.close()


def test_batch_huge_cells():
    """Members whose cells outgrow the large tier (the centres of generators on
    a sphere, 1,999 and 2,999 faces) go to the batch's block tier and equal
    standalone tessellations bit for bit; Lloyd steps take them too."""
    from common import bench_distribution
    ms = [([0, 0, 0], [100, 100, 100], (13, 13, 13), bench_distribution("sphere", 2000, 90), []),
          ([0, 0, 0], [1, 1, 1], (10, 10, 10), uniform(1000, 0, 1, 91), []),
          ([0, 0, 0], [100, 100, 100], (15, 15, 15), bench_distribution("sphere", 3000, 92), [])]
    b = build_batch(ms)
    ts = [standalone(m) for m in ms]
    for k, t in enumerate(ts):
        assert_member_equal(b, k, t)
    assert b.summaries(2)[2][0] == 2999
    b.lloyd(2)
    for t in ts:
        for _ in range(2):
            t.relax()
            t.calculate()
    for k, t in enumerate(ts):
        assert_member_equal(b, k, t)


def test_batch_reset_takes_new_members():
    """A batch reset after a calculate (and a Lloyd step) takes a new set of
    members, larger than the first, and computes them as a fresh batch does:
    each equals its standalone tessellation bit for bit."""
    import vorothree_b200 as v
    first, second = members(5)[:6], members(9)
    b = build_batch(first)
    b.calculate()
    b.lloyd(1)
    b.reset()
    for bmin, bmax, grid, pts, walls in second:
        b.add(v.BoundingBox(bmin, bmax), grid, pts, walls)
    b.commit()
    b.calculate()
    for k, m in enumerate(second):
        t = standalone(m)
        gv, gc, gn = b.summaries(k)
        sv, sc, sn = t.summaries()
        assert np.array_equal(gn, sn) and np.array_equal(gv, sv) and np.array_equal(gc, sc), k
        t.close()
    b.close()
