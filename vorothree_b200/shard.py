"""One tessellation split across processes, one process per GPU.

A cell depends only on its own generator and on the shared, read-only
generator set and bins (compute_cell, tessellation.rs:414-475), so the cells
of one tessellation shard with no exchange during the computation: every
rank holds all generators, computes a contiguous range of cell ids
(Tessellation.calculate_range), and the per-cell summaries are gathered at
the end -- the only collective, and it moves results, not work.

    import torch.distributed as dist
    dist.init_process_group("nccl")            # one rank per GPU
    t = Tessellation(bounds, Algorithm3DGrid(100, 100, 100))
    t.set_generators(points)                   # same points on every rank
    vol, cen, nfaces = calculate_sharded(t)    # full arrays on every rank

calculate_sharded_device does the same without leaving the GPU: each rank's
slice is read in place from the library's device buffers and the all-gather
runs over NCCL (NVLink between the GPUs of a node), so the results arrive as
CUDA tensors on every rank and never pass through host memory.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Tuple

import numpy as np


def cell_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous, balanced split of the ids [0, n) into `world` ranges; the
    first n % world ranges hold one cell more."""
    if world <= 0 or not 0 <= rank < world or n < 0:
        raise ValueError(f"bad shard: n={n} rank={rank} world={world}")
    q, r = divmod(n, world)
    begin = rank * q + min(rank, r)
    return begin, begin + q + (1 if rank < r else 0)


def cell_chunks(n: int, rank: int, world: int, chunk: int) -> List[Tuple[int, int]]:
    """The id ranges of this rank in an interleaved split: chunk k of
    [0, n) (ids [k chunk, (k + 1) chunk)) belongs to rank k % world.  Every
    rank gets an equal share of every part of the id order, so an input whose
    cost varies along it -- the clustered configuration lists its 64 blobs'
    generators first and the background after -- keeps the ranks balanced."""
    if world <= 0 or not 0 <= rank < world or n < 0 or chunk <= 0:
        raise ValueError(f"bad shard: n={n} rank={rank} world={world} chunk={chunk}")
    return [(b, min(b + chunk, n)) for b in range(rank * chunk, n, world * chunk)]


def chunk_count(n: int, rank: int, world: int, chunk: int) -> int:
    return sum(e - b for b, e in cell_chunks(n, rank, world, chunk))


def _device_for(group):
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def gather_summaries(vol: np.ndarray, cen: np.ndarray, nfaces: np.ndarray, n: int, group=None):
    """All-gather of every rank's slice of the per-cell summaries.

    vol[k], cen[k], nfaces[k] are the results of cell begin + k of this
    rank's range (cell_range(n, rank, world)).  Returns the full arrays
    (vol[n], cen[n, 3], nfaces[n]) on every rank.
    """
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    begin, end = cell_range(n, rank, world)
    if len(vol) != end - begin:
        raise ValueError(f"rank {rank} holds {len(vol)} cells, its range has {end - begin}")
    width = -(-n // world) if n else 0
    dev = _device_for(group)
    pack = torch.zeros((width, 5), dtype=torch.float64)
    k = end - begin
    pack[:k, 0] = torch.from_numpy(np.asarray(vol, np.float64))
    pack[:k, 1:4] = torch.from_numpy(np.asarray(cen, np.float64).reshape(-1, 3))
    pack[:k, 4] = torch.from_numpy(np.asarray(nfaces, np.int32).astype(np.float64))
    pack = pack.to(dev)
    parts = [torch.empty_like(pack) for _ in range(world)]
    dist.all_gather(parts, pack, group=group)
    out_v = np.empty(n, np.float64)
    out_c = np.empty((n, 3), np.float64)
    out_f = np.empty(n, np.int32)
    for r, p in enumerate(parts):
        b, e = cell_range(n, r, world)
        a = p[:e - b].cpu().numpy()
        out_v[b:e] = a[:, 0]
        out_c[b:e] = a[:, 1:4]
        out_f[b:e] = a[:, 4].astype(np.int32)
    return out_v, out_c, out_f


def calculate_sharded(tess, group=None, rank: Optional[int] = None, world: Optional[int] = None):
    """calculate() of `tess` split over the ranks of `group`: this rank
    computes its id range on its GPU, then the summaries are all-gathered.
    Every rank must hold the same generators and walls."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if world is None else world
    rank = dist.get_rank(group) if rank is None else rank
    n = tess.count_generators()
    begin, end = cell_range(n, rank, world)
    tess.calculate_range(begin, end)
    vol, cen, nf = tess.summaries()
    return gather_summaries(vol[begin:end], cen[begin:end], nf[begin:end], n, group)


class _DeviceView:
    """A library device buffer as torch sees it through the CUDA array
    interface (no copy).  torch takes no read-only flag, so the views are
    writable; writing them changes the tessellation's results."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def device_summaries(tess):
    """(vol[n], cen[n, 3], nfaces[n]) of the last calculate as CUDA tensors
    that view the tessellation's own device buffers (no copy), ordered after
    its stream.  They stay valid until the next set_generators, calculate or
    close of `tess`; clone them to keep them longer."""
    import torch
    from ._lib import check
    n = tess.count_cells()
    dev = torch.device("cuda", torch.cuda.current_device())
    if n == 0:
        return (torch.empty(0, dtype=torch.float64, device=dev), torch.empty((0, 3), dtype=torch.float64, device=dev),
                torch.empty(0, dtype=torch.int32, device=dev))
    dv, dc, dn = C.c_void_p(), C.c_void_p(), C.c_void_p()
    check(tess._L.vd_tess_device_results(tess._h, C.byref(dv), C.byref(dc), C.byref(dn)), tess._h)
    torch.cuda.current_stream().wait_stream(torch.cuda.ExternalStream(tess.stream()))
    vol = torch.as_tensor(_DeviceView(dv.value, (n,), "<f8"), device=dev)
    cen = torch.as_tensor(_DeviceView(dc.value, (n, 3), "<f8"), device=dev)
    nf = torch.as_tensor(_DeviceView(dn.value, (n,), "<i4"), device=dev)
    return vol, cen, nf


def gather_summaries_tensors(vol, cen, nfaces, n: int, group=None):
    """gather_summaries for tensors on the process group's device: rank r
    passes the results of its cell range (cell_range(n, r, world)); every rank
    gets (vol[n], cen[n, 3], nfaces[n]) on the same device.  One all-gather of
    a padded (width, 5) float64 block per rank; face counts travel as exact
    float64 integers."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    begin, end = cell_range(n, rank, world)
    k = end - begin
    if vol.shape[0] != k or cen.shape[0] != k or nfaces.shape[0] != k:
        raise ValueError(f"rank {rank} holds {vol.shape[0]} cells, its range has {k}")
    width = -(-n // world) if n else 0
    pack = torch.zeros((width, 5), dtype=torch.float64, device=vol.device)
    pack[:k, 0] = vol
    pack[:k, 1:4] = cen.reshape(-1, 3)
    pack[:k, 4] = nfaces.to(torch.float64)
    parts = [torch.empty_like(pack) for _ in range(world)]
    dist.all_gather(parts, pack, group=group)
    full = torch.cat([p[:cell_range(n, r, world)[1] - cell_range(n, r, world)[0]] for r, p in enumerate(parts)])
    return full[:, 0].contiguous(), full[:, 1:4].contiguous(), full[:, 4].to(torch.int32)


def calculate_sharded_device(tess, group=None):
    """calculate_sharded with the results kept on the GPU: this rank computes
    its id range, its slice of the summaries is read in place from the
    library's device buffers, and an NCCL all-gather assembles the full
    arrays as CUDA tensors on every rank.  Needs a process group on the NCCL
    backend; every rank must hold the same generators and walls."""
    import torch.distributed as dist
    if dist.get_backend(group) != "nccl":
        raise ValueError("calculate_sharded_device needs an NCCL process group; use calculate_sharded")
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n = tess.count_generators()
    begin, end = cell_range(n, rank, world)
    tess.calculate_range(begin, end)
    vol, cen, nf = device_summaries(tess)
    return gather_summaries_tensors(vol[begin:end], cen[begin:end], nf[begin:end], n, group)


def set_generators_broadcast(tess, points=None, src: int = 0, group=None) -> int:
    """set_generators on every rank from the generators rank `src` holds: the
    array (host array or CUDA tensor, (n, 3) float64) crosses to the other
    GPUs in one NCCL broadcast into device memory and each rank filters and
    bins it there (set_generators_device), so no rank stages it through host
    memory.  Other ranks pass points=None.  Returns the kept count."""
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) != "nccl":
        raise ValueError("set_generators_broadcast needs an NCCL process group")
    dev = torch.device("cuda", torch.cuda.current_device())
    rank = dist.get_rank(group)
    n = torch.zeros(1, dtype=torch.int64, device=dev)
    if rank == src:
        pts = torch.as_tensor(points, dtype=torch.float64).reshape(-1, 3)
        n[0] = pts.shape[0]
    dist.broadcast(n, src=src, group=group)
    buf = torch.empty((int(n.item()), 3), dtype=torch.float64, device=dev)
    if rank == src:
        buf.copy_(pts)
    dist.broadcast(buf, src=src, group=group)
    # the library reads the buffer on its own stream
    torch.cuda.current_stream().synchronize()
    kept = tess.set_generators_device(buf.data_ptr(), buf.shape[0])
    torch.cuda.synchronize()
    return kept


def gather_cells_tensors(vol, cen, nfaces, n: int, chunk: int, group=None, ids=None, areas=None):
    """The all-gather of an interleaved split (cell_chunks): rank r passes the
    results of its cells in id order -- vol[k], cen[k], nfaces[k] and, when
    ids / areas are given, the concatenation of those cells' neighbour ids and
    face areas (nfaces[k] each, face order) -- as tensors on the process
    group's device.  Every rank gets the full arrays on that device:
    (vol[n], cen[n, 3], nfaces[n]) and, with ids / areas, the CSR
    (offsets[n + 1] int64, ids int32, areas float64) of the whole
    tessellation, as Tessellation.neighbors / face_areas give it.  One
    all-gather of a padded (width, 5) float64 block; with faces, one of the
    face totals and one each of the padded ids and areas."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    counts = [chunk_count(n, r, world, chunk) for r in range(world)]
    k = counts[rank]
    if vol.shape[0] != k or cen.shape[0] != k or nfaces.shape[0] != k:
        raise ValueError(f"rank {rank} holds {vol.shape[0]} cells, its chunks have {k}")
    dev = vol.device
    width = max(counts) if counts else 0
    pack = torch.zeros((width, 5), dtype=torch.float64, device=dev)
    pack[:k, 0] = vol
    pack[:k, 1:4] = cen.reshape(-1, 3)
    pack[:k, 4] = nfaces.to(torch.float64)
    parts = [torch.empty_like(pack) for _ in range(world)]
    dist.all_gather(parts, pack, group=group)
    full = torch.empty((n, 5), dtype=torch.float64, device=dev)
    for r, p in enumerate(parts):
        o = 0
        for b, e in cell_chunks(n, r, world, chunk):
            full[b:e] = p[o:o + e - b]
            o += e - b
    out_v = full[:, 0].contiguous()
    out_c = full[:, 1:4].contiguous()
    out_f = full[:, 4].to(torch.int32)
    if ids is None and areas is None:
        return out_v, out_c, out_f
    # the face CSR: totals, then the padded ids and areas
    tot = torch.tensor([int(ids.shape[0]) if ids is not None else int(areas.shape[0])], dtype=torch.int64,
                       device=dev)
    tots = [torch.empty_like(tot) for _ in range(world)]
    dist.all_gather(tots, tot, group=group)
    tots = [int(t.item()) for t in tots]
    tmax = max(tots) if tots else 0
    fcount = out_f.clamp(min=0).to(torch.int64)
    off = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    off[1:] = torch.cumsum(fcount, 0)
    offh = off.cpu().numpy()
    res_ids = res_ar = None
    for name, src, dt in (("ids", ids, torch.int32), ("areas", areas, torch.float64)):
        if src is None:
            continue
        padded = torch.zeros(max(tmax, 1), dtype=dt, device=dev)
        padded[:src.shape[0]] = src
        got = [torch.empty_like(padded) for _ in range(world)]
        dist.all_gather(got, padded, group=group)
        out = torch.empty(int(offh[n]), dtype=dt, device=dev)
        for r, g in enumerate(got):
            o = 0
            for b, e in cell_chunks(n, r, world, chunk):
                lo, hi = int(offh[b]), int(offh[e])
                out[lo:hi] = g[o:o + hi - lo]
                o += hi - lo
        if name == "ids":
            res_ids = out
        else:
            res_ar = out
    return out_v, out_c, out_f, off, res_ids, res_ar


def _local_cells(n: int, rank: int, world: int, chunk: int) -> np.ndarray:
    cc = cell_chunks(n, rank, world, chunk)
    return np.concatenate([np.arange(b, e) for b, e in cc]) if cc else np.zeros(0, np.int64)


def calculate_sharded_faces(tess, group=None, chunk: int = 4096):
    """calculate() of `tess` split over the ranks of `group` in interleaved
    chunks (cell_chunks): this rank computes its chunks on its GPU
    (calculate_strided), and every rank receives the whole tessellation's
    summaries and face CSR as host arrays: (vol[n], cen[n, 3], nfaces[n],
    offsets[n + 1], neighbour ids, face areas).  Every rank must hold the same
    generators and walls."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n = tess.count_generators()
    tess.calculate_strided(chunk, world, rank)
    vol, cen, nf = tess.summaries()
    off, ids = tess.neighbors()
    _, ar = tess.face_areas()
    mine = _local_cells(n, rank, world, chunk)
    sel = np.concatenate([np.arange(off[i], off[i + 1]) for i in mine]) if len(mine) else np.zeros(0, np.int64)
    dev = _device_for(group)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    out = gather_cells_tensors(t(vol[mine]), t(cen[mine]), t(nf[mine]), n, chunk, group,
                               ids=t(ids[sel]), areas=t(ar[sel]))
    return tuple(x.cpu().numpy() for x in out)


def device_neighbors(tess):
    """(offsets[n + 1] int64, ids int32, areas float64) of the last calculate
    as CUDA tensors that view the tessellation's own device buffers (no
    copy); valid until the next call that changes `tess`."""
    import torch
    from ._lib import check
    n = tess.count_cells()
    dev = torch.device("cuda", torch.cuda.current_device())
    do, di, da = C.c_void_p(), C.c_void_p(), C.c_void_p()
    tot = C.c_int64()
    check(tess._L.vd_tess_device_neighbors(tess._h, C.byref(do), C.byref(di), C.byref(da), C.byref(tot)), tess._h)
    off = torch.as_tensor(_DeviceView(do.value, (n + 1,), "<i8"), device=dev)
    if tot.value == 0:
        return off, torch.empty(0, dtype=torch.int32, device=dev), torch.empty(0, dtype=torch.float64, device=dev)
    ids = torch.as_tensor(_DeviceView(di.value, (tot.value,), "<i4"), device=dev)
    ar = torch.as_tensor(_DeviceView(da.value, (tot.value,), "<f8"), device=dev)
    return off, ids, ar


def calculate_sharded_faces_device(tess, group=None, chunk: int = 4096):
    """calculate_sharded_faces with every result kept on the GPU: this rank's
    cells and their face CSR are selected in place from the library's device
    buffers and the NCCL all-gathers assemble the whole tessellation's
    summaries and CSR as CUDA tensors on every rank."""
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) != "nccl":
        raise ValueError("calculate_sharded_faces_device needs an NCCL process group")
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n = tess.count_generators()
    tess.calculate_strided(chunk, world, rank)
    vol, cen, nf = device_summaries(tess)
    off, ids, ar = device_neighbors(tess)
    dev = vol.device
    mine = torch.from_numpy(_local_cells(n, rank, world, chunk)).to(dev)
    # the face entries of this rank's chunks, in id order (each chunk's faces
    # are contiguous in the CSR)
    offh = off.cpu().numpy()
    segs = [(int(offh[b]), int(offh[e])) for b, e in cell_chunks(n, rank, world, chunk)]
    fsel = torch.cat([torch.arange(lo, hi, device=dev) for lo, hi in segs]) if segs else \
        torch.zeros(0, dtype=torch.int64, device=dev)
    return gather_cells_tensors(vol.index_select(0, mine), cen.index_select(0, mine), nf.index_select(0, mine), n,
                                chunk, group, ids=ids.index_select(0, fsel), areas=ar.index_select(0, fsel))
