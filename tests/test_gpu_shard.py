"""GPU: the device-resident form of the sharded calculate.  device_summaries
must read the same bits the host copies give, and calculate_sharded_device
(calculate_range, in-place slices, an NCCL all-gather) must equal calculate()
on one rank.  Several ranks need several GPUs; the pack/unpack of uneven
ranges is covered on the CPU by test_shard_gloo.py."""
import os
import socket

import numpy as np
import pytest

from common import blobs

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _child(port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    try:
        import datetime
        import torch
        import torch.distributed as dist
        import vorothree_b200 as v
        torch.cuda.set_device(0)
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=60))
    except Exception as ex:  # reported to the parent
        q.put((False, repr(ex)))
        return
    try:
        pts = blobs(60000, 8, 0.03, 0.5, 44)
        t = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(30, 30, 30))
        t.add_wall(v.Wall(-1000, v.SphereGeometry([0.5, 0.5, 0.5], 0.47)))
        t.set_generators(pts)
        t.calculate()
        hv, hc, hn = t.summaries()
        dv, dc, dn = v.device_summaries(t)
        ok = (np.array_equal(dv.cpu().numpy(), hv) and np.array_equal(dc.cpu().numpy(), hc)
              and np.array_equal(dn.cpu().numpy(), hn))
        # the same generators through an NCCL broadcast into device memory
        t2 = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(30, 30, 30))
        t2.add_wall(v.Wall(-1000, v.SphereGeometry([0.5, 0.5, 0.5], 0.47)))
        ok = ok and v.set_generators_broadcast(t2, pts) == t.count_generators()
        ok = ok and np.array_equal(t2.generators(), t.generators())
        t2.close()
        sv, sc, sn = v.calculate_sharded_device(t)
        ok = ok and sv.is_cuda and sn.dtype == torch.int32
        ok = ok and (np.array_equal(sv.cpu().numpy(), hv) and np.array_equal(sc.cpu().numpy(), hc)
                     and np.array_equal(sn.cpu().numpy(), hn))
        # the interleaved split with the face CSR, on the device and via the host
        t.calculate()
        hoff, hids = t.neighbors()
        _, har = t.face_areas()
        for fn in (v.calculate_sharded_faces_device, v.calculate_sharded_faces):
            out = fn(t, chunk=777)
            out = [x.cpu().numpy() if hasattr(x, "cpu") else x for x in out]
            for got, want in zip(out, (hv, hc, hn, hoff, hids, har)):
                ok = ok and np.array_equal(got, want)
        t.close()
        q.put((ok, None))
    except Exception as ex:  # reported to the parent
        q.put((False, repr(ex)))
    finally:
        dist.destroy_process_group()


def test_sharded_device_nccl_one_rank():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_child, args=(_free_port(), q))
    p.start()
    ok, err = q.get(timeout=300)
    p.join(timeout=60)
    assert err is None, err
    assert ok
