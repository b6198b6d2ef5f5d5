"""GPU: the C ABI's error behaviour (status codes, messages, and a handle
that stays usable after a refused call), mirroring where the reference
panics, ignores or returns an error (wall/mod.rs:24-32, tessellation.rs:73-75,
126-148)."""
import ctypes as C

import numpy as np
import pytest

from common import uniform

pytestmark = pytest.mark.gpu


def lib():
    from vorothree_b200 import _lib
    return _lib, _lib.load()


def d3(v):
    a = np.asarray(v, np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def test_null_and_bad_arguments():
    _lib, L = lib()
    h = C.c_void_p()
    lo, plo = d3([0, 0, 0])
    hi, phi = d3([1, 1, 1])
    assert L.vd_tess_create(plo, phi, 0, 4, 4, C.byref(h)) == _lib.VD_EINVAL
    assert L.vd_last_error(None)  # a message for the failed create
    assert L.vd_tess_calculate(None) == _lib.VD_EINVAL
    assert L.vd_tess_destroy(None) == _lib.VD_EINVAL or L.vd_tess_destroy(None) == _lib.VD_OK


def test_results_before_calculate_and_recovery():
    import vorothree_b200 as v
    _lib, L = lib()
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(4, 4, 4))
    t.set_generators(uniform(200, 0, 1, 1))
    for call in (t.summaries, t.neighbors, t.face_areas, t.export_cells):
        with pytest.raises(v.VoronoidError) as e:
            call()
        assert e.value.code == _lib.VD_ESTATE
    # no cells yet: get_cell gives None and cells() an empty list, as the
    # reference's Option and Vec do before calculate
    assert t.get_cell(0) is None and t.cells() == []
    # a bad range is refused and changes nothing
    with pytest.raises(v.VoronoidError) as e:
        t.calculate_range(150, 300)
    assert e.value.code == _lib.VD_EINVAL
    t.calculate()
    vol, _, nf = t.summaries()
    assert abs(vol.sum() - 1.0) < 1e-9 and (nf > 0).all()
    # out-of-range cells: None (Rust's Option), an empty export range is fine
    assert t.get_cell(200) is None
    with pytest.raises(v.VoronoidError):
        t.export_cells(5, 300)
    # set_generator past the end is ignored (tessellation.rs:73-75)
    before = t.generators()
    t.set_generator(10_000, [0.5, 0.5, 0.5])
    assert np.array_equal(t.generators(), before)


def test_wall_ids_and_limits_through_the_abi():
    import vorothree_b200 as v
    _lib, L = lib()
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(3, 3, 3))
    p, pp = d3([0.5, 0.5, 0.5])
    n, pn = d3([0, 0, 1])
    # Wall::new panics for id > WALL_ID_MAX; the ABI refuses it
    assert L.vd_tess_add_wall_plane(t._h, pp, pn, -999) == _lib.VD_EINVAL
    assert L.vd_last_error(t._h)
    assert L.vd_tess_add_wall_plane(t._h, pp, pn, -1000) == _lib.VD_OK
    # a polyhedron with a negative plane count is refused
    assert L.vd_tess_add_wall_polyhedron(t._h, pp, pn, -1, -1001) == _lib.VD_EINVAL
    t.set_generators(uniform(100, 0, 1, 2))
    t.calculate()
    assert t.count_cells() == int((uniform(100, 0, 1, 2)[:, 2] >= 0.5).sum())


def test_export_argument_checks():
    import vorothree_b200 as v
    _lib, L = lib()
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(3, 3, 3))
    t.set_generators(uniform(50, 0, 1, 3))
    t.calculate()
    off = np.zeros(51, np.int64)
    i64 = C.POINTER(C.c_int64)
    verts = np.zeros(10, np.float64)
    # offsets are required; the four polytope arrays come together or not at all
    assert L.vd_tess_export_cells(t._h, 0, 50, None, None, None, None, None, None, None) == _lib.VD_EINVAL
    assert L.vd_tess_export_cells(t._h, 0, 50, off.ctypes.data_as(i64), off.ctypes.data_as(i64),
                                  off.ctypes.data_as(i64), C.c_void_p(verts.ctypes.data), None, None,
                                  None) == _lib.VD_EINVAL
    assert L.vd_tess_export_cells(t._h, 10, 5, off.ctypes.data_as(i64), off.ctypes.data_as(i64),
                                  off.ctypes.data_as(i64), None, None, None, None) == _lib.VD_EINVAL
    x = t.export_cells(0, 50)
    assert x["v_off"][-1] > 0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nan_and_inf_generators_match_the_oracle(oracle_mod, precision):
    """Non-finite generators are not an error in the reference: without walls
    set_generators keeps them (tessellation.rs:43-67), get_bin_index clamps
    and truncates them (NaN to bin 0, +-inf to the edge bins,
    algo_3d_grid.rs:98-107), and every comparison with a NaN distance is
    false, so such a cell stays the box and no other cell is clipped by it.
    With a sphere wall the filter drops them.  Each case equals the oracle
    (NaN outputs compare equal to NaN)."""
    import vorothree_b200 as v
    pts = uniform(3000, 0.0, 1.0, 71)
    pts[10] = [np.nan, 0.5, 0.5]
    pts[20] = [0.5, np.inf, 0.5]
    pts[30] = [-np.inf, 0.2, 0.9]
    pts[40] = [np.nan, np.nan, np.nan]
    for walls in ((), (("sphere", [0.5, 0.5, 0.5], 0.45),)):
        t = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(12, 12, 12))
        t.set_precision(precision)
        o = oracle_mod.OracleTessellation([0, 0, 0], [1, 1, 1], 12, 12, 12)
        for _, c, r in walls:
            t.add_wall(v.Wall(v.WALL_ID_MAX, v.SphereGeometry(c, r)))
            o.add_wall_sphere(c, r, v.WALL_ID_MAX)
        assert t.set_generators(pts) == o.set_generators(pts)
        t.calculate()
        o.calculate()
        assert np.array_equal(t.generators(), o.generators(), equal_nan=True)
        for a, b in zip(t.summaries(), o.summaries()):
            assert np.array_equal(a, b, equal_nan=True)
        assert np.array_equal(t.neighbors()[1], o.neighbors()[1])
        assert np.array_equal(t.face_areas()[1], o.face_areas()[1], equal_nan=True)
        t.close()
