"""Autotuner: the bin density and the launch choices of the clip tiers.

What it picks, per input class (distribution, size bucket):
  * the bin grid of Algorithm3DGrid: too coarse and a cell scans many far
    generators of its own bin (dense clusters), too fine and the shell walk
    opens many empty bins (sparse regions);
  * the first tier's polytope layout ("slots": a clip rewrites only the
    faces it cuts; "full": every face loop per clip) and, for the slot
    layout, its register budget -- 5, 6 or 7 blocks of four warps per SM, the
    compiled variants (more resident warps against more spills).
and once for the tessellation, on inputs with cells adjacent to thousands of
others (the reference's sphere-surface benchmark distribution):
  * the hand-off to the block-per-cell tier: how few cells left after the
    medium tier go there directly, how many blocks it runs at once, and up to
    which tessellation size its blocks are 16 warps wide instead of 32;
and per input, from its coarse occupancy (`hollow`):
  * the walk's batched plane tests, for inputs that leave large parts of the
    box empty.
None of these changes a result: every choice computes the same doubles.

The tuner times Tessellation.calculate on the GPU (coordinate descent: bin
density first, then the layout, then its blocks per SM) and records the
fastest per class in a table (the committed `autotune_table.json` next to
this file, or one given).  `choose` looks the class of a new input up and
falls back to the defaults when the class was never tuned.

    from vorothree_b200 import autotune
    grid, tuning = autotune.choose(points, bounds)      # (nx, ny, nz), settings
    t = Tessellation(bounds, Algorithm3DGrid(*grid)); t.set_tuning(tuning)
    table = autotune.tune(points, bounds, walls)         # measure and record
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
# the first tier's choices the tuner searches, and the library's defaults
LAYOUTS = ("slots", "full")
BLOCKS_PER_SM = (5, 6, 7)
DEFAULT_TUNING = {"fast_layout": "slots", "fast_blocks_per_sm": 7, "noop_run": -1}
# the block-per-cell tier's hand-off, searched once (HANDOFF_KEY)
HANDOFF_KEY = "handoff"
DIRECT_MAX = (1, 16, 64, 256)
NARROW_MAX = (500, 2000, 5000, 1 << 30)
DEFAULT_HANDOFF = {"huge_direct_max": 64, "huge_blocks_max": 64, "huge_narrow_max": 1 << 30}


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
    data = {"what": "per (distribution, size bucket): bin density factor (bins per axis = factor * (N/V)^(1/3) "
                    "* edge) and the first tier's layout / blocks per SM; 'handoff': the block-per-cell "
                    "tier's thresholds (results never depend on any of these)",
            "device": device, "entries": entries}
    with open(p, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)


def _nearest(cls: str, n: int, entries: Dict[str, dict]) -> Optional[dict]:
    want = size_bucket(n)
    best, dist = None, None
    for k, e in entries.items():
        if "/2^" not in k:
            continue
        c, b = k.split("/2^")
        if c != cls:
            continue
        d = abs(int(b) - want)
        if dist is None or d < dist:
            best, dist = e, d
    return best


def lookup(cls: str, n: int, entries: Optional[Dict[str, dict]] = None) -> float:
    """Tuned factor of the nearest tuned size bucket of this class, or the
    class default."""
    entries = load_table() if entries is None else entries
    e = _nearest(cls, n, entries)
    return DEFAULT_FACTOR[cls] if e is None else float(e["factor"])


def lookup_tuning(cls: str, n: int, entries: Optional[Dict[str, dict]] = None) -> dict:
    """The launch settings (Tessellation.set_tuning) for this class and size:
    the first tier's choices of the nearest tuned size bucket and the table's
    hand-off thresholds, each falling back to the library's defaults."""
    entries = load_table() if entries is None else entries
    out = dict(DEFAULT_TUNING)
    e = _nearest(cls, n, entries)
    if e is not None:
        out.update({k: e["tuning"][k] for k in DEFAULT_TUNING if k in e.get("tuning", {})})
    out.update(DEFAULT_HANDOFF)
    h = entries.get(HANDOFF_KEY)
    if h is not None:
        out.update({k: h["tuning"][k] for k in DEFAULT_HANDOFF if k in h.get("tuning", {})})
    return out


def choose_grid(points, bounds, entries: Optional[Dict[str, dict]] = None) -> Tuple[int, int, int]:
    """The grid the tuner would use for this input."""
    pts = np.asarray(points, np.float64).reshape(-1, 3)
    cls = distribution_class(pts, bounds)
    return grid_for(len(pts), bounds, lookup(cls, len(pts), entries))


# the walk's batched plane tests (tuning noop_run) for hollow inputs: after
# this many clips in a row that changed nothing
NOOP_RUN_HOLLOW = 8
HOLLOW_EMPTY = 0.25


def hollow(points, bounds) -> bool:
    """Whether the generators leave large parts of the box empty: more than a
    quarter of the 4 x 4 x 4 equal parts of the box hold none (a dense central
    box, generators on a sphere).  The cells at the edge of such a region reach
    far into the empty part, and their walks clip with thousands of candidates,
    nearly all without effect; the walk's batched plane tests pass over those
    clips (central box, 10,000 generators: 7.2 against 3.6 ms), and cost
    instructions on other inputs (uniform: about 10%)."""
    pts = np.asarray(points, np.float64).reshape(-1, 3)
    if len(pts) == 0:
        return False
    lo = np.asarray(bounds.min, np.float64)
    hi = np.asarray(bounds.max, np.float64)
    idx = np.clip(((pts - lo) / (hi - lo) * 4).astype(np.int64), 0, 3)
    lin = idx[:, 0] + 4 * (idx[:, 1] + 4 * idx[:, 2])
    return 1.0 - len(np.unique(lin)) / 64.0 > HOLLOW_EMPTY


def input_tuning(points, bounds, entries: Optional[Dict[str, dict]] = None) -> dict:
    """The launch settings for this input: the table's for its class and size,
    with the walk's batched plane tests on when the input is hollow."""
    pts = np.asarray(points, np.float64).reshape(-1, 3)
    tun = lookup_tuning(distribution_class(pts, bounds), len(pts), entries)
    if hollow(pts, bounds):
        tun["noop_run"] = NOOP_RUN_HOLLOW
    return tun


def choose(points, bounds, entries: Optional[Dict[str, dict]] = None) -> Tuple[Tuple[int, int, int], dict]:
    """(grid, launch settings) the tuner would use for this input."""
    pts = np.asarray(points, np.float64).reshape(-1, 3)
    cls = distribution_class(pts, bounds)
    return grid_for(len(pts), bounds, lookup(cls, len(pts), entries)), input_tuning(pts, bounds, entries)


def _time(points, bounds, grid, walls, tuning: dict, reps: int, precision: str) -> float:
    """Best device time of calculate() (clip passes, fallback tiers included)
    over `reps` runs after one warm-up."""
    from .tessellation import Algorithm3DGrid, Tessellation
    t = Tessellation(bounds, Algorithm3DGrid(*grid))
    try:
        t.set_precision(precision)
        t.set_tuning(tuning)
        for w in walls:
            t.add_wall(w)
        t.set_generators(points)
        t.calculate()
        best = None
        for _ in range(reps):
            t.calculate()
            tm = t.timings()
            ms = tm["clip_ms"] + tm["fallback_ms"]
            best = ms if best is None else min(best, ms)
        return best
    finally:
        t.close()


def tune(points, bounds, walls: Sequence = (), factors: Iterable[float] = FACTORS, reps: int = 3,
         precision: str = "fp64", entries: Optional[Dict[str, dict]] = None, layouts: Sequence[str] = LAYOUTS,
         blocks: Sequence[int] = BLOCKS_PER_SM) -> Dict[str, dict]:
    """Time calculate() on the GPU (best of `reps` after one warm-up) over the
    density factors with the default launch settings, then over the first
    tier's layouts and (slot layout) blocks per SM at the best factor, and
    record the fastest under this input's class.  Returns the updated table
    entries (not written to disk; see record)."""
    pts = np.asarray(points, np.float64).reshape(-1, 3)
    cls = distribution_class(pts, bounds)
    entries = dict(load_table() if entries is None else entries)
    trials = []
    for f in factors:
        g = grid_for(len(pts), bounds, f)
        trials.append({"factor": f, "grid": list(g), "tuning": dict(DEFAULT_TUNING),
                       "ms": _time(pts, bounds, g, walls, DEFAULT_TUNING, reps, precision)})
    win = min(trials, key=lambda r: r["ms"])
    g = win["grid"]
    for layout in layouts:
        for nb in (blocks if layout == "slots" else (6,)):
            tun = dict(DEFAULT_TUNING, fast_layout=layout, fast_blocks_per_sm=nb)
            if tun == DEFAULT_TUNING:
                continue
            trials.append({"factor": win["factor"], "grid": list(g), "tuning": tun,
                           "ms": _time(pts, bounds, g, walls, tun, reps, precision)})
    best = min((r for r in trials if r["factor"] == win["factor"]), key=lambda r: r["ms"])
    entries[key(cls, len(pts))] = {"factor": win["factor"], "tuning": best["tuning"], "ms": best["ms"],
                                   "n": len(pts), "trials": trials}
    return entries


def tune_handoff(cases, reps: int = 2, entries: Optional[Dict[str, dict]] = None) -> Dict[str, dict]:
    """The block-per-cell tier's thresholds: `cases` is a list of (points,
    bounds, grid) whose cells include ones beyond the large tier (e.g. the
    sphere-surface distribution); the setting with the least total time over
    them is recorded under HANDOFF_KEY."""
    entries = dict(load_table() if entries is None else entries)
    trials = []
    for dm in DIRECT_MAX:
        for nm in NARROW_MAX:
            tun = dict(DEFAULT_TUNING, huge_direct_max=dm, huge_narrow_max=nm,
                       huge_blocks_max=DEFAULT_HANDOFF["huge_blocks_max"])
            ms = [_time(p, b, g, (), tun, reps, "fp64") for p, b, g in cases]
            trials.append({"tuning": {k: tun[k] for k in DEFAULT_HANDOFF}, "ms": ms, "total_ms": sum(ms)})
    win = min(trials, key=lambda r: r["total_ms"])
    entries[HANDOFF_KEY] = {"tuning": win["tuning"], "total_ms": win["total_ms"], "trials": trials,
                            "cases": [len(p) for p, _, _ in cases]}
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

        python -m vorothree_b200.autotune [--out PATH] [--max-log2 22] [--handoff-only]

    --handoff-only keeps the table's first-tier entries and searches the
    block-per-cell tier's thresholds again.
    """
    import argparse
    import torch
    from .tessellation import BoundingBox
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=TABLE_PATH)
    ap.add_argument("--max-log2", type=int, default=22)
    ap.add_argument("--handoff-only", action="store_true")
    a = ap.parse_args(argv)
    from .workloads import bench_distribution
    b = BoundingBox([0, 0, 0], [1, 1, 1])
    entries: Dict[str, dict] = dict(load_table()) if a.handoff_only else {}
    for cls in () if a.handoff_only else ("uniform", "clustered"):
        for e in range(10, a.max_log2 + 1, 2):
            pts = synthetic(cls, 1 << e, seed=e)
            if distribution_class(pts, b) != cls:
                continue
            entries = tune(pts, b, factors=LADDER[cls], reps=3 if e < 22 else 1, entries=entries)
            k = key(cls, len(pts))
            print(k, entries[k]["factor"], entries[k]["tuning"], round(entries[k]["ms"], 3), flush=True)
    # the reference's sphere-surface distribution: one cell per tessellation
    # adjacent to every other generator
    box = BoundingBox([0, 0, 0], [100, 100, 100])
    cases = []
    for n in (1000, 3000, 10000):
        g = int(np.ceil(n ** (1.0 / 3.0)))
        cases.append((bench_distribution("sphere", n, 11), box, (g, g, g)))
    entries = tune_handoff(cases, entries=entries)
    print(HANDOFF_KEY, entries[HANDOFF_KEY]["tuning"], round(entries[HANDOFF_KEY]["total_ms"], 3), flush=True)
    record(entries, a.out, device=torch.cuda.get_device_name(0))


if __name__ == "__main__":
    main()
