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
from typing import Optional, Tuple

import numpy as np


def cell_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous, balanced split of the ids [0, n) into `world` ranges; the
    first n % world ranges hold one cell more."""
    if world <= 0 or not 0 <= rank < world or n < 0:
        raise ValueError(f"bad shard: n={n} rank={rank} world={world}")
    q, r = divmod(n, world)
    begin = rank * q + min(rank, r)
    return begin, begin + q + (1 if rank < r else 0)


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
