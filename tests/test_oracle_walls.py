"""CPU: the oracle's cylinder, cone, torus and convex-polyhedron walls
(wall_3d.rs:107-365, 462-708) against the reference's own known answers
(tests/volumes.rs:68-105: cylinder and dodecahedron volumes on the 20^3
lattice within 1%; tests/neighbors.rs:180-200: dodecahedron reciprocity) and
against analytic volumes for the cone and the torus, which the reference's
tests do not cover."""
import math

import numpy as np
import pytest

from common import uniform

WALL = -1000


def lattice(size=10.0, n=20):
    step = size / n
    ax = np.arange(n) * step + step / 2
    return np.array([[x, y, z] for x in ax for y in ax for z in ax])


def total_volume(o):
    vol, _, _ = o.summaries()
    return vol.sum()


def box_tess(oracle_mod, pts, add):
    t = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 5, 5, 5)
    t.set_generators(pts)
    add(t)
    t.calculate(1)
    return t


def test_cylinder_volume(oracle_mod):
    t = box_tess(oracle_mod, lattice(), lambda t: t.add_wall_cylinder([5, 5, 5], [0, 0, 1], 4.0, WALL))
    exp = math.pi * 16.0 * 10.0
    assert abs(total_volume(t) - exp) / exp < 0.01


def dodecahedron_volume(radius):
    xi = math.sqrt((5.0 + 2.0 * math.sqrt(5.0)) / 15.0)
    dist = radius * xi
    a = 2.0 * dist * math.sqrt(10.0) / math.sqrt(25.0 + 11.0 * math.sqrt(5.0))
    return (15.0 + 7.0 * math.sqrt(5.0)) / 4.0 * a ** 3


def test_dodecahedron_volume(oracle_mod):
    pts, nrm = oracle_mod.regular_polyhedron(12, [5, 5, 5], 4.0)
    t = box_tess(oracle_mod, lattice(), lambda t: t.add_wall_polyhedron(pts, nrm, WALL))
    exp = dodecahedron_volume(4.0)
    assert abs(total_volume(t) - exp) / exp < 0.01


@pytest.mark.parametrize("faces,vol_of_r1", [
    (4, 8.0 / (9.0 * math.sqrt(3.0))),          # regular tetrahedron, circumradius 1
    (6, 8.0 / (3.0 * math.sqrt(3.0))),          # cube
    (8, 4.0 / 3.0),                              # octahedron
    (20, 2.536150710120),                        # icosahedron
])
def test_regular_polyhedra_volumes(oracle_mod, faces, vol_of_r1):
    pts, nrm = oracle_mod.regular_polyhedron(faces, [5, 5, 5], 4.0)
    assert len(pts) == faces
    # planar walls: every cell is cut exactly, so the total is the solid's volume
    t = box_tess(oracle_mod, lattice(), lambda t: t.add_wall_polyhedron(pts, nrm, WALL))
    exp = vol_of_r1 * 64.0
    assert abs(total_volume(t) - exp) / exp < 1e-9


def test_dodecahedron_reciprocity(oracle_mod):
    pts_w, nrm_w = oracle_mod.regular_polyhedron(12, [15, 15, 15], 10.0)
    t = oracle_mod.OracleTessellation([0, 0, 0], [30, 30, 30], 5, 5, 5)
    t.set_generators(uniform(100, 0.0, 30.0, 3))
    t.add_wall_polyhedron(pts_w, nrm_w, WALL)
    t.calculate(1)
    off, ids = t.neighbors()
    nb = [set(int(x) for x in ids[off[i]:off[i + 1]] if x >= 0) for i in range(t.count_cells())]
    for i, s in enumerate(nb):
        for j in s:
            assert i in nb[j]


def test_cone_volume(oracle_mod):
    ang = 0.4
    t = box_tess(oracle_mod, lattice(), lambda t: t.add_wall_cone([5, 5, 0], [0, 0, 1], ang, WALL))
    r = 10.0 * math.tan(ang)
    exp = math.pi * r * r * 10.0 / 3.0
    assert abs(total_volume(t) - exp) / exp < 0.03


def test_torus_volume(oracle_mod):
    t = box_tess(oracle_mod, lattice(), lambda t: t.add_wall_torus([5, 5, 5], [0, 0, 1], 3.0, 1.5, WALL))
    exp = 2.0 * math.pi ** 2 * 3.0 * 1.5 ** 2
    assert abs(total_volume(t) - exp) / exp < 0.03


def test_wall_filters(oracle_mod):
    # contains(): generators outside a wall are dropped at set_generators
    pts = uniform(4000, 0.0, 10.0, 8)
    t = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 5, 5, 5)
    t.add_wall_torus([5, 5, 5], [0, 0, 2], 3.0, 1.5, WALL)
    kept = t.set_generators(pts)
    d = pts - 5.0
    rho = np.sqrt(d[:, 0] ** 2 + d[:, 1] ** 2)
    inside = np.sqrt((rho - 3.0) ** 2 + d[:, 2] ** 2) <= 1.5
    assert kept == int(inside.sum())
    t = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 5, 5, 5)
    t.add_wall_cone([5, 5, 0], [0, 0, 3], 0.4, WALL)
    kept = t.set_generators(pts)
    h = pts[:, 2]
    rr = np.sqrt((pts[:, 0] - 5) ** 2 + (pts[:, 1] - 5) ** 2)
    assert kept == int(((h >= 0) & (rr <= h * math.tan(0.4))).sum())


def test_set_generator_bins(oracle_mod):
    """set_generator (tessellation.rs:70-92) against a list-of-lists model of
    Algorithm3DGrid's bins (algo_3d_grid.rs:109-143): swap_remove from the old
    bin, push onto the new one; moves outside a wall and out-of-range indices
    are ignored."""
    pts = uniform(400, 0.0, 10.0, 9)
    t = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 4, 4, 4)
    t.add_wall_cylinder([5, 5, 5], [0, 0, 1], 4.5, WALL)
    n = t.set_generators(pts)
    gens = t.generators().reshape(-1, 3).copy()
    model = [[] for _ in range(64)]
    bin_of = []
    for i, p in enumerate(gens):
        b = t.bin_index(*p)
        model[b].append(i)
        bin_of.append(b)
    assert t.bins() == model
    rng = np.random.Generator(np.random.PCG64(10))
    moved = rejected = 0
    for _ in range(300):
        i = int(rng.integers(0, n + 3))
        p = rng.uniform(0.0, 10.0, 3)
        t.set_generator(i, p)
        if i >= n or math.hypot(p[0] - 5, p[1] - 5) > 4.5:
            rejected += 1
            continue
        moved += 1
        b = t.bin_index(*p)
        if b != bin_of[i]:
            old = model[bin_of[i]]
            k = old.index(i)
            old[k] = old[-1]
            old.pop()
            model[b].append(i)
            bin_of[i] = b
        gens[i] = p
    assert moved > 100 and rejected > 50
    assert t.bins() == model
    assert np.array_equal(t.generators().reshape(-1, 3), gens)


def sealed_pair(oracle_mod, walls, n=3000, seed=12):
    pts = uniform(n, 0.0, 10.0, seed)
    out = []
    for sealed in (False, True):
        t = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 6, 6, 6)
        t.set_generators(pts)
        for kind, args in walls:
            getattr(t, "add_wall_" + kind)(*args)
        (t.calculate_sealed if sealed else t.calculate)(1)
        out.append(t)
    return out


@pytest.mark.parametrize("walls", [
    [("sphere", ([5, 5, 5], 4.5, WALL))],
    [("cylinder", ([5, 5, 5], [0, 0.2, 1], 4.0, WALL)), ("plane", ([5, 5, 5], [1, 0, 0], WALL - 1))],
    [("torus", ([5, 5, 5], [0, 0, 1], 3.0, 1.8, WALL))],
])
def test_calculate_sealed_structure(oracle_mod, walls):
    """calculate_sealed only ever clips cells that touch a curved wall, with
    a plane whose id is that wall's; the seal log lists each such clip."""
    plain, sealed = sealed_pair(oracle_mod, walls)
    pv, _, _ = plain.summaries()
    sv, _, _ = sealed.summaries()
    log = sealed.seal_log().reshape(-1, 3)
    assert len(log) > 0
    curved = {a[-1] for k, a in walls if k != "plane"}
    assert set(log[:, 2]) <= curved
    changed = set(np.nonzero(sv != pv)[0])
    assert changed <= set(log[:, 0])
    assert np.all(sv <= pv + 1e-12)
    # every logged neighbour is a face neighbour of the cell before sealing
    off, ids = plain.neighbors()
    for i, j, _ in log[:50]:
        assert j in ids[off[i]:off[i + 1]]
    # calculate clears the log
    sealed.calculate(1)
    assert len(sealed.seal_log()) == 0


def test_prune_boundaries_log(oracle_mod):
    _, t = sealed_pair(oracle_mod, [("sphere", ([5, 5, 5], 4.5, WALL))])
    t.prune_boundaries()
    log = t.prune_log().reshape(-1, 4)
    pos = t.prune_pos_log().reshape(-1, 3)
    assert len(log) > 0 and log[:, 3].sum() == len(pos)
    # the shared vertices lie on tangent planes of the sphere: just outside it
    r = np.linalg.norm(pos - 5.0, axis=1)
    assert np.all(r >= 4.5 - 1e-9) and np.all(r < 5.0)
    assert set(log[:, 2]) == {WALL}


def _splitmix64_at(seed, k):
    m = 2 ** 64 - 1
    z = (seed + (k + 1) * 0x9E3779B97F4A7C15) & m
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    return z ^ (z >> 31)


def test_random_generators_oracle(oracle_mod):
    """random_generators (tessellation.rs:96-121) with a seed: SplitMix64's
    published first outputs for seed 0, a pure-Python restatement of the
    attempt loop, and the count * 1000 attempt cap."""
    assert [_splitmix64_at(0, k) for k in range(4)] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4,
                                                         0x06C45D188009454F, 0xF88BB8A8724C81EC]
    lo, hi = [-1.0, 0.0, 2.0], [3.0, 10.0, 2.5]
    t = oracle_mod.OracleTessellation(lo, hi, 4, 4, 4)
    t.add_wall_sphere([1.0, 5.0, 2.25], 2.0, WALL)
    seed = 0xDEADBEEF12345
    assert t.random_generators(200, seed) == 200
    want, a = [], 0
    while len(want) < 200:
        p = [lo[c] + float(_splitmix64_at(seed, 3 * a + c) >> 11) * 2.0 ** -53 * (hi[c] - lo[c]) for c in range(3)]
        if (p[0] - 1.0) ** 2 + (p[1] - 5.0) ** 2 + (p[2] - 2.25) ** 2 <= 4.0:
            want.append(p)
        a += 1
    assert np.array_equal(t.generators().reshape(-1, 3), np.asarray(want))
    # a region that takes ~2000 attempts per point: the cap of 50 * 1000
    # attempts stops the loop early
    t = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 4, 4, 4)
    t.add_wall_sphere([5, 5, 5], 0.492, WALL)
    n = t.random_generators(50, 7)
    assert 5 < n < 50
    t.calculate(1)
    assert t.count_cells() == n


def _oracle_wall(oracle_mod, w):
    import vorothree_b200 as v
    t = oracle_mod.OracleTessellation([0, 0, 0], [10, 10, 10], 2, 2, 2)
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
    return t


def test_host_wall_queries_match_oracle(oracle_mod):
    """Wall::contains and Wall::cut through the library's host entry points
    (the functions its kernels use) against the oracle, bit for bit, for every
    wall kind at points spread over and around the walls."""
    import vorothree_b200 as v
    P = v.ConvexPolyhedronGeometry
    walls = [v.Wall(WALL, v.PlaneGeometry([5, 5, 5], [0.3, -1.0, 0.2])),
             v.Wall(WALL, v.SphereGeometry([5, 5, 5], 3.5)),
             v.Wall(WALL, v.CylinderGeometry([5, 5, 5], [0.2, 0.1, 1.0], 4.0)),
             v.Wall(WALL, v.ConeGeometry([5, 5, -1], [0.1, 0.0, 1.0], 0.45)),
             v.Wall(WALL, v.TorusGeometry([5, 5, 5], [0.0, 0.3, 1.0], 3.0, 1.6)),
             v.Wall(WALL, P.new_dodecahedron([5, 5, 5], 4.5)),
             v.Wall(WALL, P.new_tetrahedron([5, 5, 5], 4.5))]
    rng = np.random.Generator(np.random.PCG64(41))
    pts = np.concatenate([rng.uniform(-2, 12, size=(1500, 3)), [[5, 5, 5], [5, 5, -1], [5, 5, 8], [8, 5, 5]]])
    for w in walls:
        o = _oracle_wall(oracle_mod, w)
        for p in pts:
            assert w.contains(p) == o.wall_contains(0, p), (w.geometry, p)
            got = []
            w.cut(p, lambda a, b: got.append((a, b)))
            want = o.wall_cut(0, p)
            assert len(got) == len(want), (w.geometry, p)
            for (a, b), (c, d) in zip(got, want):
                assert np.array_equal(a, c) and np.array_equal(b, d), (w.geometry, p)


def test_grid_bin_index_matches_oracle(oracle_mod):
    import vorothree_b200 as v
    rng = np.random.Generator(np.random.PCG64(42))
    for (lo, hi, n) in [([0, 0, 0], [1, 1, 1], (10, 10, 10)), ([-5, 2, 0], [7, 3, 0.5], (13, 4, 7))]:
        b = v.BoundingBox(lo, hi)
        g = v.Algorithm3DGrid.new(*n, b)
        o = oracle_mod.OracleTessellation(lo, hi, *n)
        ext = np.asarray(hi, float) - np.asarray(lo, float)
        pts = np.asarray(lo) + rng.uniform(-0.2, 1.2, size=(3000, 3)) * ext
        pts[:5] = hi
        for p in pts:
            assert g.get_bin_index(*p) == o.bin_index(*p), p
