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
"""
from __future__ import annotations

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
