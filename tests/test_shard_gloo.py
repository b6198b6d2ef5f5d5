"""Sharding one tessellation's cells over processes (CPU, gloo, worlds 2 and 3).

Each rank computes its id range -- here with the oracle, standing in for the
GPU on this CPU-only test -- and gather_summaries assembles the full result
on every rank; it must equal one full calculate() bit for bit.  The GPU
side of the split (calculate_range) is checked in test_gpu_parity.py.
"""
import os
import socket

import numpy as np
import pytest

from common import uniform


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    import datetime
    import torch.distributed as dist
    from oracle.oracle import OracleTessellation
    from vorothree_b200.shard import cell_range, gather_summaries, gather_summaries_tensors
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=60))
        pts = uniform(6000, 0.0, 1.0, 31)
        t = OracleTessellation([0, 0, 0], [1, 1, 1], 12, 12, 12)
        t.add_wall_sphere([0.5, 0.5, 0.5], 0.46, -1000)
        n = t.set_generators(pts)
        b, e = cell_range(n, rank, world)
        t.calculate_range(b, e, 1)
        vol, cen, nf = t.summaries()
        gv, gc, gn = gather_summaries(vol[b:e], cen[b:e], nf[b:e], n)
        full = OracleTessellation([0, 0, 0], [1, 1, 1], 12, 12, 12)
        full.add_wall_sphere([0.5, 0.5, 0.5], 0.46, -1000)
        full.set_generators(pts)
        full.calculate(1)
        fv, fc, fn = full.summaries()
        ok = np.array_equal(gv, fv) and np.array_equal(gc, fc) and np.array_equal(gn, fn)
        # the tensor form (the one calculate_sharded_device runs over NCCL)
        import torch
        tv, tc, tn = gather_summaries_tensors(torch.from_numpy(vol[b:e].copy()), torch.from_numpy(cen[b:e].copy()),
                                              torch.from_numpy(nf[b:e].copy()), n)
        ok = ok and np.array_equal(tv.numpy(), fv) and np.array_equal(tc.numpy(), fc) and np.array_equal(tn.numpy(), fn)
        ok = ok and tn.dtype == torch.int32
        dist.destroy_process_group()
        q.put((rank, ok, None))
    except Exception as ex:  # reported to the parent
        q.put((rank, False, repr(ex)))


def test_cell_range_partition():
    from vorothree_b200.shard import cell_range
    for n in (0, 1, 7, 1000, 1 << 20):
        for world in (1, 2, 3, 8):
            ranges = [cell_range(n, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(ranges[k][1] == ranges[k + 1][0] for k in range(world - 1))
            sizes = [e - b for b, e in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        cell_range(10, 2, 2)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_summaries_gloo(oracle_mod, world):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    for rank, ok, err in sorted(results):
        assert err is None, f"rank {rank}: {err}"
        assert ok, f"rank {rank}: gathered summaries differ from a full calculate"


def _rank_chunks(rank, world, port, q):
    """Interleaved split with the face CSR: each rank computes its chunks
    (the oracle stands in for the GPU) and gather_cells_tensors assembles
    summaries, neighbour ids and face areas equal to one full calculate."""
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    import datetime
    import torch
    import torch.distributed as dist
    from common import blobs
    from oracle.oracle import OracleTessellation
    from vorothree_b200.shard import cell_chunks, gather_cells_tensors
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=60))
        pts = np.clip(blobs(5000, 4, 0.03, 0.6, 33), 0.0, 1.0)
        chunk = 300
        t = OracleTessellation([0, 0, 0], [1, 1, 1], 12, 12, 12)
        t.add_wall_sphere([0.5, 0.5, 0.5], 0.47, -1000)
        n = t.set_generators(pts)
        vs, cs, fs, ids, ars = [], [], [], [], []
        for b, e in cell_chunks(n, rank, world, chunk):
            t.calculate_range(b, e, 1)
            v, c, f = t.summaries()
            off, nb = t.neighbors()
            _, ar = t.face_areas()
            vs.append(v[b:e])
            cs.append(c[b:e])
            fs.append(f[b:e])
            ids.append(nb[off[b]:off[e]])
            ars.append(ar[off[b]:off[e]])
        cat = lambda xs, dt, shape=(0,): torch.from_numpy(np.concatenate(xs).astype(dt)) if xs else \
            torch.zeros(shape, dtype=getattr(torch, np.dtype(dt).name))  # noqa: E731
        gv, gc, gf, goff, gids, gar = gather_cells_tensors(
            cat(vs, np.float64), cat(cs, np.float64, (0, 3)), cat(fs, np.int32), n, chunk,
            ids=cat(ids, np.int32), areas=cat(ars, np.float64))
        full = OracleTessellation([0, 0, 0], [1, 1, 1], 12, 12, 12)
        full.add_wall_sphere([0.5, 0.5, 0.5], 0.47, -1000)
        full.set_generators(pts)
        full.calculate(1)
        fv, fc, fn = full.summaries()
        foff, fids = full.neighbors()
        _, far = full.face_areas()
        ok = (np.array_equal(gv.numpy(), fv) and np.array_equal(gc.numpy(), fc) and np.array_equal(gf.numpy(), fn)
              and np.array_equal(goff.numpy(), foff) and np.array_equal(gids.numpy(), fids)
              and np.array_equal(gar.numpy(), far) and gids.dtype == torch.int32)
        dist.destroy_process_group()
        q.put((rank, ok, None))
    except Exception as ex:  # reported to the parent
        q.put((rank, False, repr(ex)))


def test_cell_chunks_partition():
    from vorothree_b200.shard import cell_chunks
    for n in (0, 1, 7, 1000, 100_003):
        for world in (1, 2, 3, 8):
            for chunk in (1, 5, 4096):
                ids = sorted(i for r in range(world) for b, e in cell_chunks(n, r, world, chunk) for i in range(b, e))
                assert ids == list(range(n))
    with pytest.raises(ValueError):
        cell_chunks(10, 0, 2, 0)


@pytest.mark.parametrize("world", [2, 3])
def test_interleaved_split_with_faces_gloo(oracle_mod, world):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_chunks, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    for rank, ok, err in sorted(results):
        assert err is None, f"rank {rank}: {err}"
        assert ok, f"rank {rank}: gathered cells differ from a full calculate"
