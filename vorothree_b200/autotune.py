"""Autotuner for the grid's bin density.

The one launch parameter of the hot path that depends on the input is the
bin grid of Algorithm3DGrid: too coarse and a cell scans many far
generators of its own bin (dense clusters), too fine and the shell walk
opens many empty bins (sparse regions).  The clip kernel's own shape (one
warp per cell, 4 warps per block, 7 blocks per SM, the polytope staged in
shared memory) is fixed by its register and shared-memory budget and needs
no tuning.

The tuner times Tessellation.calculate on the GPU for a ladder of bin
densities and records the fastest per input class: (distribution, size
bucket).  `choose_grid` looks the class of a new input up in the table
(the committed `autotune_table.json` next to this file, or one given) and
falls back to a density rule when the class was never tuned.

    from vorothree_b200 import autotune
    grid = autotune.choose_grid(points, bounds)          # (nx, ny, nz)
    table = autotune.tune(points, bounds, walls)          # measure and record
"""
from __future__ import annotations

import json
import math
import os
from typing import Dict, Iterable, Optional, Sequence, Tuple

import numpy as np

TABLE_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune_table.json")
# bins per axis = factor * (N / V)^(1/3) * edge: factor 1 is one generator per bin
FACTORS = (0.6, 0.8, 1.0, 1.25, 1.6, 2.0, 2.5, 3.2, 4.0, 5.0)
# the ladders the default table is tuned over: clustered input never wins
# with bins coarser than one generator each, uniform input never with bins
# much finer
LADDER = {"uniform": (0.6, 0.8, 1.0, 1.25, 1.6, 2.0), "clustered": (1.0, 1.6, 2.0, 2.5, 3.2, 4.0, 5.0)}
DEFAULT_FACTOR = {"uniform": 1.0, "clustered": 2.5}
_SAMPLE = 1 << 16


def grid_for(n: int, bounds, factor: float) -> Tuple[int, int, int]:
    """Bins per axis for n generators in `bounds` at the given density factor
    (near-cubic bins)."""
    edge = np.subtract(bounds.max, bounds.min).astype(np.float64)
    vol = float(np.prod(edge))
    per = (max(n, 1) / vol) ** (1.0 / 3.0) if vol > 0 else 1.0
    return tuple(max(1, int(round(factor * per * e))) for e in edge)


def distribution_class(points, bounds, seed: int = 0) -> str:
    """'uniform' or 'clustered', from the bin occupancy of a sample.

    A sample of up to 65,536 points is binned at one point per bin; Poisson
    (uniform) input leaves e^-1 = 37% of the bins empty, clustered input far
    more.  Only the sample is inspected."""
    pts = np.asarray(points, np.float64).reshape(-1, 3)
    n = len(pts)
    if n < 64:
        return "uniform"
    rng = np.random.Generator(np.random.PCG64(seed))
    s = pts if n <= _SAMPLE else pts[rng.choice(n, _SAMPLE, replace=False)]
    lo = np.asarray(bounds.min, np.float64)
    hi = np.asarray(bounds.max, np.float64)
    g = np.asarray(grid_for(len(s), bounds, 1.0))
    idx = np.clip(((s - lo) / (hi - lo) * g).astype(np.int64), 0, g - 1)
    lin = idx[:, 0] + g[0] * (idx[:, 1] + g[1] * idx[:, 2])
    empty = 1.0 - len(np.unique(lin)) / float(np.prod(g))
    return "clustered" if empty > 0.55 else "uniform"


def size_bucket(n: int) -> int:
    """log2 size bucket, rounded to even exponents (1k, 4k, 16k, ...)."""
    return 2 * int(round(math.log2(max(n, 1)) / 2.0))


def key(cls: str, n: int) -> str:
    return f"{cls}/2^{size_bucket(n)}"


def load_table(path: Optional[str] = None) -> Dict[str, dict]:
    p = path or TABLE_PATH
    if not os.path.exists(p):
        return {}
    with open(p) as f:
        return json.load(f).get("entries", {})


def record(entries: Dict[str, dict], path: Optional[str] = None, device: str = ""):
    p = path or TABLE_PATH
    data = {"what": "bin density factor per (distribution, size bucket); "
                    "bins per axis = factor * (N/V)^(1/3) * edge",
            "device": device, "entries": entries}
    with open(p, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)


def lookup(cls: str, n: int, entries: Optional[Dict[str, dict]] = None) -> float:
    """Tuned factor of the nearest tuned size bucket of this class, or the
    class default."""
    entries = load_table() if entries is None else entries
    want = size_bucket(n)
    best, dist = None, None
    for k, e in entries.items():
        c, b = k.split("/2^")
        if c != cls:
            continue
        d = abs(int(b) - want)
        if dist is None or d < dist:
            best, dist = e["factor"], d
    return DEFAULT_FACTOR[cls] if best is None else float(best)


def choose_grid(points, bounds, entries: Optional[Dict[str, dict]] = None) -> Tuple[int, int, int]:
    """The grid the tuner would use for this input."""
    pts = np.asarray(points, np.float64).reshape(-1, 3)
    cls = distribution_class(pts, bounds)
    return grid_for(len(pts), bounds, lookup(cls, len(pts), entries))


def tune(points, bounds, walls: Sequence = (), factors: Iterable[float] = FACTORS, reps: int = 3,
         precision: str = "fp64", entries: Optional[Dict[str, dict]] = None) -> Dict[str, dict]:
    """Time calculate() on the GPU for each density factor (best of `reps`
    after one warm-up) and record the fastest under this input's class.
    Returns the updated table entries (not written to disk; see record)."""
    from .tessellation import Algorithm3DGrid, Tessellation
    pts = np.asarray(points, np.float64).reshape(-1, 3)
    cls = distribution_class(pts, bounds)
    entries = dict(load_table() if entries is None else entries)
    trials = []
    for f in factors:
        g = grid_for(len(pts), bounds, f)
        t = Tessellation(bounds, Algorithm3DGrid(*g))
        try:
            t.set_precision(precision)
            for w in walls:
                t.add_wall(w)
            t.set_generators(pts)
            t.calculate()
            best = None
            for _ in range(reps):
                t.calculate()
                tm = t.timings()
                ms = tm["clip_ms"] + tm["fallback_ms"]
                best = ms if best is None else min(best, ms)
            trials.append({"factor": f, "grid": list(g), "ms": best})
        finally:
            t.close()
    win = min(trials, key=lambda r: r["ms"])
    entries[key(cls, len(pts))] = {"factor": win["factor"], "ms": win["ms"], "n": len(pts), "trials": trials}
    return entries


def synthetic(cls: str, n: int, seed: int = 0) -> np.ndarray:
    """Seeded inputs of each class in the unit cube: i.i.d. uniform, or 70% in
    64 isotropic Gaussian blobs (sigma 0.01, centres uniform) + 30% uniform."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if cls == "uniform":
        return rng.uniform(0.0, 1.0, size=(n, 3))
    nb = int(round(0.7 * n))
    centres = rng.uniform(0.0, 1.0, size=(64, 3))
    return np.concatenate([centres[np.arange(nb) % 64] + rng.normal(0.0, 0.01, size=(nb, 3)),
                           rng.uniform(0.0, 1.0, size=(n - nb, 3))])


def main(argv=None):
    """Tune the default table on this GPU over seeded synthetic inputs of
    both classes, sizes 2^10 .. 2^22, and write it next to this file.

        python -m vorothree_b200.autotune [--out PATH] [--max-log2 22]
    """
    import argparse
    import torch
    from .tessellation import BoundingBox
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=TABLE_PATH)
    ap.add_argument("--max-log2", type=int, default=22)
    a = ap.parse_args(argv)
    b = BoundingBox([0, 0, 0], [1, 1, 1])
    entries: Dict[str, dict] = {}
    for cls in ("uniform", "clustered"):
        for e in range(10, a.max_log2 + 1, 2):
            pts = synthetic(cls, 1 << e, seed=e)
            if distribution_class(pts, b) != cls:
                continue
            entries = tune(pts, b, factors=LADDER[cls], reps=3 if e < 22 else 1, entries=entries)
            k = key(cls, len(pts))
            print(k, entries[k]["factor"], round(entries[k]["ms"], 3), flush=True)
    record(entries, a.out, device=torch.cuda.get_device_name(0))


if __name__ == "__main__":
    main()
