"""GPU: the allocation-free entry point vd_calculate_noalloc.

It serves callers that cannot allocate device memory themselves (an
application that owns the GPU's memory and hands out fixed buffers, a
framework memory pool, a latency-critical loop).  The test calls it through
the C ABI with caller-owned device buffers, twice in a row on different
inputs, and checks each result against the regular entry points
(vd_tess_set_generators + vd_tess_calculate) with the same exact-equality
tolerance as the other FP64 parity tests.  This file is named so that pytest
collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from common import bench_distribution, blobs, uniform

pytestmark = pytest.mark.gpu


def noalloc(L, bmin, bmax, grid, pts):
    import torch
    n = len(pts)
    d_xyz = torch.from_numpy(np.ascontiguousarray(pts, np.float64)).cuda()
    vol = torch.full((max(n, 1),), -1.0, dtype=torch.float64, device="cuda")
    cen = torch.full((max(n, 1), 3), -1.0, dtype=torch.float64, device="cuda")
    nf = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    mn = np.asarray(bmin, np.float64)
    mx = np.asarray(bmax, np.float64)
    rc = L.vd_calculate_noalloc(mn.ctypes.data_as(C.POINTER(C.c_double)), mx.ctypes.data_as(C.POINTER(C.c_double)),
                                grid[0], grid[1], grid[2], C.c_void_p(d_xyz.data_ptr()), n,
                                C.c_void_p(vol.data_ptr()), C.c_void_p(cen.data_ptr()),
                                C.c_void_p(nf.data_ptr()), None)
    torch.cuda.synchronize()
    return rc, vol[:n].cpu().numpy(), cen[:n].cpu().numpy(), nf[:n].cpu().numpy()


def regular(bmin, bmax, grid, pts):
    import vorothree_b200 as v
    t = v.Tessellation(v.BoundingBox(bmin, bmax), v.Algorithm3DGrid(*grid))
    t.set_generators(pts)
    t.calculate()
    out = t.summaries()
    fb = t.fallback_counts()
    t.close()
    return out + (fb,)


def test_noalloc_matches_regular_two_calls():
    import vorothree_b200 as v
    L = v.load()
    cases = [
        ([0, 0, 0], [1, 1, 1], (16, 16, 16), uniform(6000, 0.0, 1.0, 21)),
        ([-2, 0, 1], [3, 4, 2], (9, 7, 3), uniform(700, 0.0, 1.0, 22) * [5, 4, 1] + [-2, 0, 1]),
    ]
    for bmin, bmax, grid, pts in cases:
        rc, vol, cen, nf = noalloc(L, bmin, bmax, grid, pts)
        assert rc == 0, L.vd_last_error(None)
        rv, rcen, rnf, _ = regular(bmin, bmax, grid, pts)
        assert np.array_equal(nf, rnf)
        assert np.array_equal(vol, rv)
        assert np.array_equal(cen, rcen)
        box = np.prod(np.subtract(bmax, bmin))
        assert abs(vol.sum() - box) < 1e-9 * box


def test_noalloc_rejects_oversized_requests():
    import vorothree_b200 as v
    L = v.load()
    rc, *_ = noalloc(L, [0, 0, 0], [1, 1, 1], (8, 8, 8), uniform(8193, 0.0, 1.0, 1))
    assert rc == 1 and b"8192" in L.vd_last_error(None)
    rc, *_ = noalloc(L, [0, 0, 0], [1, 1, 1], (21, 21, 21), uniform(100, 0.0, 1.0, 1))
    assert rc == 1 and b"search-order" in L.vd_last_error(None)


def test_noalloc_large_capacity_pass_two_calls():
    """Inputs whose cells outgrow the shared-memory pass go through the
    large-capacity pass in the scratch array: the centre of 80 points on a
    sphere (79 faces, pooled beyond the 48 per-cell face slots) and a dense
    blob on a coarse grid.  Each call equals the regular path exactly."""
    import vorothree_b200 as v
    L = v.load()
    cases = [
        ([0, 0, 0], [100, 100, 100], (4, 4, 4), bench_distribution("sphere", 80, 31)),
        ([0, 0, 0], [1, 1, 1], (6, 6, 6), np.clip(blobs(5000, 2, 0.02, 0.9, 32), 0.0, 1.0)),
    ]
    for bmin, bmax, grid, pts in cases:
        rc, vol, cen, nf = noalloc(L, bmin, bmax, grid, pts)
        assert rc == 0, L.vd_last_error(None)
        rv, rcen, rnf, fb = regular(bmin, bmax, grid, pts)
        assert sum(fb.values()) > 0, "the case must leave the shared-memory pass"
        assert np.array_equal(nf, rnf)
        assert np.array_equal(vol, rv)
        assert np.array_equal(cen, rcen)


def test_noalloc_block_tier_cell_is_an_overflow():
    """The centre of 3,000 points on a sphere has 2,999 faces: beyond the
    large-capacity pass, so the call reports VD_EOVERFLOW instead of a result
    (the regular entry points build it in their block-per-cell tier)."""
    import vorothree_b200 as v
    from vorothree_b200._lib import VD_EOVERFLOW
    L = v.load()
    pts = bench_distribution("sphere", 3000, 33)
    rc, *_ = noalloc(L, [0, 0, 0], [100, 100, 100], (14, 14, 14), pts)
    assert rc == VD_EOVERFLOW
    assert b"large polytope capacity" in L.vd_last_error(None)
