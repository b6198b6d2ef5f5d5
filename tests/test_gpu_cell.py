"""GPU: the standalone cell API (Cell3DFaces on the device) against the oracle.

Ports the reference's own cell unit tests (cell_3d_faces.rs:576-593) and
checks long random clip sequences bit for bit against the oracle's
restatement of clip_with_scratch: the polytope (vertices, face order, face
neighbours), the clip's returned (modified, max radius^2), and the measures.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def same_polytope(g, o):
    ov, ofc, ofi, ofn = o.export()
    assert np.array_equal(g.vertices(), ov)
    assert np.array_equal(g.face_counts(), ofc)
    assert np.array_equal(g.face_indices(), ofi)
    assert np.array_equal(g.face_neighbors(), ofn)
    assert g.volume() == o.volume()
    assert np.array_equal(g.centroid(), o.centroid())
    for k in range(len(ofc)):
        assert g.face_area(k) == o.face_area(k)


def test_reference_cell_unit_tests():
    import vorothree_b200 as v
    # test_cell_faces_box
    cell = v.Cell3DFaces.new(0, v.BoundingBox([0, 0, 0], [1, 1, 1]))
    assert abs(cell.volume() - 1.0) < 1e-6
    assert abs(cell.centroid()[0] - 0.5) < 1e-6
    assert list(cell.face_neighbors()) == [-5, -6, -3, -4, -1, -2]
    # test_cell_faces_clip
    cell.clip([0.5, 0.5, 0.5], [1.0, 0.0, 0.0], 10)
    assert abs(cell.volume() - 0.5) < 1e-6
    assert 10 in cell.neighbors()
    assert cell.id() == 0


def test_random_clip_sequences_bitwise(oracle_mod):
    import vorothree_b200 as v
    rng = np.random.Generator(np.random.PCG64(40))
    for trial in range(12):
        lo = rng.uniform(-5, 0, size=3)
        hi = lo + rng.uniform(0.5, 5, size=3)
        g = v.Cell3DFaces.new(trial, v.BoundingBox(lo, hi))
        o = oracle_mod.OracleCell.new(trial, lo, hi)
        gen = lo + rng.uniform(0.3, 0.7, size=3) * (hi - lo)
        for k in range(60):
            # bisector-like planes around the generator, at shrinking distances
            d = rng.normal(size=3)
            d *= rng.uniform(0.05, 1.0) * np.linalg.norm(hi - lo) / np.linalg.norm(d)
            point = gen + 0.5 * d
            mod_g, r2 = g.clip(point, d, k, generator=gen)
            mod_o = o.clip(point, d, k)
            assert mod_g == mod_o, (trial, k)
            if mod_o and not o.is_empty():
                assert r2 == o.max_radius_sq(gen)
            else:
                assert r2 == 0.0
            if k % 15 == 14:
                same_polytope(g, o)
        same_polytope(g, o)
        assert g.max_radius_sq(gen) == o.max_radius_sq(gen)


def test_clip_to_empty_and_noop(oracle_mod):
    import vorothree_b200 as v
    g = v.Cell3DFaces.new(3, v.BoundingBox([0, 0, 0], [1, 1, 1]))
    assert g.clip([2, 2, 2], [1, 1, 1], 1) == (False, 0.0)   # all inside
    assert g.volume() == 1.0
    assert g.clip([-1, 0, 0], [1, 0, 0], 2)[0]               # all outside
    assert g.is_empty() and g.volume() == 0.0 and len(g.face_counts()) == 0
    assert g.clip([0.5, 0.5, 0.5], [1, 0, 0], 3) == (False, 0.0)  # an empty cell stays empty


def test_clip_a_computed_cell(oracle_mod):
    """A tessellation's computed cell moves to the device and clips like the
    oracle's copy of the same cell."""
    import vorothree_b200 as v
    rng = np.random.Generator(np.random.PCG64(41))
    pts = rng.uniform(0, 1, size=(500, 3))
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(6, 6, 6))
    t.set_generators(pts)
    t.calculate()
    ot = oracle_mod.OracleTessellation([0, 0, 0], [1, 1, 1], 6, 6, 6)
    ot.set_generators(pts)
    ot.calculate()
    for i in (0, 17, 250, 499):
        gc = t.get_cell(i)
        oc = ot.get_cell(i).clone()
        same_polytope(gc, oc)
        for k in range(5):
            n = rng.normal(size=3)
            p = pts[i] + 0.02 * rng.normal(size=3)
            gm, _ = gc.clip(p, n, 1000 + k)
            assert gm == oc.clip(p, n, 1000 + k)
        same_polytope(gc, oc)


def test_cell_create_validation():
    import vorothree_b200 as v
    from vorothree_b200 import VoronoidError
    bad = v.Cell3DFaces(0, np.zeros(9), [3], [0, 1, 7], [-1])  # face entry names a missing vertex
    with pytest.raises(VoronoidError):
        bad.clip([0, 0, 0], [1, 0, 0], 1)
