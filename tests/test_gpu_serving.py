"""GPU: the serving loop.  Requests of different sizes, distributions and
walls are submitted together (they overlap on the device); each result must
equal, bit for bit, the same request computed alone by a standalone
Tessellation."""
import threading

import numpy as np
import pytest

from common import blobs, uniform

pytestmark = pytest.mark.gpu

WALL = -1000


def requests(seed):
    import vorothree_b200 as v
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k in range(12):
        n = int(round(np.exp(rng.uniform(np.log(500), np.log(60000)))))
        pts = blobs(n, 6, 0.02, 0.7, seed * 100 + k) if k % 3 == 0 else uniform(n, 0, 1, seed * 100 + k)
        walls = []
        if k % 4 == 1:
            walls.append(v.Wall(WALL, v.SphereGeometry([0.5, 0.5, 0.5], rng.uniform(0.3, 0.5))))
        if k % 4 == 2:
            nrm = rng.normal(size=3)
            walls.append(v.Wall(WALL - 1, v.PlaneGeometry([0.5, 0.5, 0.5], list(nrm))))
        g = max(1, int(np.ceil(n ** (1 / 3))))
        out.append((v.BoundingBox([0, 0, 0], [1, 1, 1]), (g, g, g), pts, walls))
    return out


def alone(req):
    import vorothree_b200 as v
    b, grid, pts, walls = req
    t = v.Tessellation(b, v.Algorithm3DGrid(*grid))
    for w in walls:
        t.add_wall(w)
    t.set_generators(pts)
    t.calculate()
    return t.summaries()


def test_served_results_equal_alone():
    import vorothree_b200 as v
    reqs = requests(3)
    srv = v.TessellationServer(slots=4, hbm_budget_bytes=8 << 30)
    tickets = [srv.submit(*r) for r in reqs]
    got = [srv.take(t) for t in tickets]
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["p99_s"] >= st["p50_s"] > 0
    for r, (vol, cen, nf) in zip(reqs, got):
        av, ac, an = alone(r)
        assert np.array_equal(nf, an) and np.array_equal(vol, av) and np.array_equal(cen, ac)
    srv.close()


def test_admission_respects_budget_and_threads():
    import vorothree_b200 as v
    reqs = requests(4)
    # a budget that admits about one large request at a time still serves all
    srv = v.TessellationServer(slots=3, hbm_budget_bytes=200 << 20)
    results = {}

    def client(idx):
        t = srv.submit(*reqs[idx])
        results[idx] = srv.take(t)
    th = [threading.Thread(target=client, args=(i,)) for i in range(len(reqs))]
    for x in th:
        x.start()
    for x in th:
        x.join()
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["peak_bytes"] <= (200 << 20)
    for i, r in enumerate(reqs):
        av, ac, an = alone(r)
        vol, cen, nf = results[i]
        assert np.array_equal(vol, av)
    srv.close()


def test_request_over_budget_rejected():
    import vorothree_b200 as v
    srv = v.TessellationServer(slots=1, hbm_budget_bytes=1 << 20)
    with pytest.raises(v.VoronoidError):
        srv.submit(v.BoundingBox([0, 0, 0], [1, 1, 1]), (10, 10, 10), uniform(20000, 0, 1, 1))
    srv.close()


def test_text_requests_equal_alone():
    """Requests whose generators arrive as read_generators text (tessellation.rs:
    153-171), mixed with array requests: each equals the array request alone;
    text that is not UTF-8 is refused at submit."""
    import vorothree_b200 as v
    reqs = requests(5)[:6]
    srv = v.TessellationServer(slots=3, hbm_budget_bytes=8 << 30)
    tickets = []
    for k, (b, grid, pts, walls) in enumerate(reqs):
        if k % 2 == 0:
            text = "".join(f"{i} {x!r} {y!r} {z!r}\n" for i, (x, y, z) in enumerate(pts.tolist()))
            tickets.append(srv.submit_text(b, grid, text, walls))
        else:
            tickets.append(srv.submit(b, grid, pts, walls))
    for r, t in zip(reqs, tickets):
        vol, cen, nf = srv.take(t)
        av, ac, an = alone(r)
        assert np.array_equal(nf, an) and np.array_equal(vol, av) and np.array_equal(cen, ac)
    with pytest.raises(v.VoronoidError):
        srv.submit_text(reqs[0][0], reqs[0][1], b"0 0.5 0.5 \xff\n")
    srv.close()


def alone_faces(req):
    import vorothree_b200 as v
    b, grid, pts, walls = req
    t = v.Tessellation(b, v.Algorithm3DGrid(*grid))
    for w in walls:
        t.add_wall(w)
    t.set_generators(pts)
    t.calculate()
    out = t.summaries() + t.neighbors() + (t.face_areas()[1],)
    t.close()
    return out


def test_face_results_equal_alone_and_requests_overlap():
    """With face results on, each request also returns its neighbour-id and
    face-area CSR, equal to the standalone tessellation's; with four slots
    and a queue of twelve, at least two requests run on the GPU at once."""
    import vorothree_b200 as v
    reqs = requests(6)
    srv = v.TessellationServer(slots=4, hbm_budget_bytes=8 << 30)
    srv.set_face_results(True)
    tickets = [srv.submit(*r) for r in reqs]
    got = [srv.take_faces(t) for t in tickets]
    assert srv.concurrency()["peak_running"] >= 2
    for r, (vol, cen, nf, off, ids, ar) in zip(reqs, got):
        av, ac, an, aoff, aids, aar = alone_faces(r)
        assert np.array_equal(nf, an) and np.array_equal(vol, av) and np.array_equal(cen, ac)
        assert np.array_equal(off, aoff) and np.array_equal(ids, aids) and np.array_equal(ar, aar)
    srv.close()


def test_cancel_queued_request():
    """One slot: a large request runs while two wait; cancelling a waiting
    one drops it (its take reports VD_ECANCELED), the other still runs and
    equals its standalone result; a finished request cannot be cancelled."""
    import vorothree_b200 as v
    from vorothree_b200._lib import VD_ECANCELED
    srv = v.TessellationServer(slots=1, hbm_budget_bytes=8 << 30)
    b = v.BoundingBox([0, 0, 0], [1, 1, 1])
    big = (b, (100, 100, 100), uniform(1_000_000, 0, 1, 81), [])
    small = requests(7)[:2]
    t0 = srv.submit(*big)
    t1 = srv.submit(*small[0])
    t2 = srv.submit(*small[1])
    assert srv.cancel(t2) is True
    with pytest.raises(v.VoronoidError) as e:
        srv.take(t2)
    assert e.value.code == VD_ECANCELED
    vol, cen, nf = srv.take(t1)
    av, ac, an = alone(small[0])
    assert np.array_equal(vol, av) and np.array_equal(nf, an)
    srv.wait(t0)
    assert srv.cancel(t0) is False
    srv.take(t0)
    srv.close()


def test_allocation_failure_inside_a_request():
    """A device allocation that fails inside a request (injected on the host:
    the library's next allocation reports out-of-memory, as a full GPU would)
    fails that request with VD_ENOMEM; the slot then serves the next request,
    whose result equals its standalone result."""
    import vorothree_b200 as v
    from vorothree_b200._lib import VD_ENOMEM, load
    L = load()
    srv = v.TessellationServer(slots=1, hbm_budget_bytes=8 << 30)
    reqs = requests(8)
    try:
        L.vd_debug_fail_allocations(1)
        t0 = srv.submit(*reqs[0])
        with pytest.raises(v.VoronoidError) as e:
            srv.take(t0)
        assert e.value.code == VD_ENOMEM
    finally:
        L.vd_debug_fail_allocations(0)
    for r in reqs[:3]:
        vol, cen, nf = srv.take(srv.submit(*r))
        av, ac, an = alone(r)
        assert np.array_equal(vol, av) and np.array_equal(nf, an) and np.array_equal(cen, ac)
    srv.close()


def test_small_requests_merge_into_batches_and_equal_alone():
    """Small requests waiting together are computed as one batch (one binning
    pass, one persistent clip launch over all their cells): with one slot and
    a burst of submissions the queue holds runs of them.  Each result equals
    the request computed alone, bit for bit; a request asking for face
    results in the middle of the burst runs alone and its CSR is complete;
    with merging off no batch is formed."""
    import vorothree_b200 as v
    reqs = requests(7) + requests(8)
    for merge in (True, False):
        srv = v.TessellationServer(slots=1, hbm_budget_bytes=8 << 30)
        if merge:
            srv.set_merging(max_members=64)
        tickets = [srv.submit(*r) for r in reqs]
        srv.set_face_results(True)
        b, grid, pts, walls = reqs[5]
        tf = srv.submit(b, grid, pts, walls)
        srv.set_face_results(False)
        tickets += [srv.submit(*r) for r in reqs[:6]]
        got = [srv.take(t) for t in tickets]
        vol, cen, nf, off, ids, ar = srv.take_faces(tf)
        ms = srv.merge_stats()
        if merge:
            assert ms["groups"] >= 1 and ms["merged_requests"] >= 2
        else:
            assert ms == {"groups": 0, "merged_requests": 0}
        for r, (gv, gc, gn) in zip(reqs + reqs[:6], got):
            av, ac, an = alone(r)
            assert np.array_equal(gn, an) and np.array_equal(gv, av) and np.array_equal(gc, ac)
        t = v.Tessellation(b, v.Algorithm3DGrid(*grid))
        for w in walls:
            t.add_wall(w)
        t.set_generators(pts)
        t.calculate()
        so, si = t.neighbors()
        assert np.array_equal(off, so) and np.array_equal(ids, si) and np.array_equal(nf, t.summaries()[2])
        assert srv.stats()["completed"] == len(tickets) + 1
        srv.close()
