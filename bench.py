#!/usr/bin/env python
"""Benchmark of the 3D tessellation hot path (cells/s) on B200.

Workload (one step): 1,048,576 generators i.i.d. uniform in the unit cube
(f64, seeded PCG64), Algorithm3DGrid 100^3 bins, Cell3DFaces, no walls:
set_generators (wall filter + binning) followed by calculate(), i.e. every
cell's polytope with its volume, centroid, face areas and neighbour ids.

    python bench.py [--gpus N --steps K --warmup W] [--precision fp64|mixed]
    python bench.py --impl reference ...   # the reference's algorithm on the host cores

`value` times device-resident input (CUDA events on the library's stream,
L2 flushed between steps); `e2e` times the same step through the C ABI with
host buffers, including the host->device copy of the generators and the
device->host copy of every result (summaries, neighbour ids, face areas).
With N GPUs (torchrun) every rank builds its own independent tessellation
(weak scaling, no collective on the data path); the step time is the max over
ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

N_GEN = 1_048_576
GRID = 100
METRIC = "3D cells/s @1M gens"
WORKLOAD = "1,048,576 uniform generators in the unit cube, grid 100^3, no walls"

# Algorithmic FP64 operations per counted event (the flop model of the clip kernel).
FLOPS_PER = {
    "classified": 8,      # (v-p).n: 3 sub, 3 mul, 2 add
    "candidates": 15,     # d = q-g, |d|^2, midpoint, 4R^2
    "intersections": 19,  # t = ds/(ds-de), v = a + t(b-a), radius
    "kept": 8,            # radius of a kept vertex
    "triangles": 50,      # volume/centroid fan triangle (27) + face-area triangle (23)
}


def set_workload(n: int, grid: int):
    global N_GEN, GRID, WORKLOAD
    N_GEN, GRID = n, grid
    WORKLOAD = f"{n:,} uniform generators in the unit cube, grid {grid}^3, no walls"


def flop_count(cnt: dict) -> int:
    return sum(FLOPS_PER[k] * int(cnt[k]) for k in FLOPS_PER)


def uniform(n, seed):
    from vorothree_b200.workloads import uniform_cube
    return uniform_cube(n, seed)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def load_profile(precision: str) -> dict:
    """The committed ncu summary of the clip kernel (DRAM bytes per launch,
    warp instructions per cell)."""
    p = os.path.join(ROOT, "profiles", f"clip_{precision}_uniform_1M.json")
    if not os.path.exists(p):
        return {}
    with open(p) as f:
        return json.load(f)


def load_traffic(precision: str):
    """DRAM bytes per clip-kernel launch from the committed ncu summary."""
    return load_profile(precision).get("dram_bytes_per_launch")


def cpu_baseline(pts, nthreads: int, sample: int, extras: dict = None, keep: list = None):
    """The oracle (a C restatement of the reference's calculate) on the host
    cores over a bounded sample of the same tessellation's cells.  `extras`,
    when given, gets the search-order table build (the Algorithm3DGrid::new
    constructor, outside calculate) and a one-thread rate over a smaller
    sample.  `keep`, when given, receives the oracle tessellation if the
    sample is every cell (the parity check compares against it)."""
    from oracle.oracle import OracleTessellation
    t0 = time.perf_counter()
    t = OracleTessellation([0, 0, 0], [1, 1, 1], GRID, GRID, GRID)
    build = time.perf_counter() - t0
    t.set_generators(pts)
    if extras is not None:
        # one thread first: the timed run below is the last calculate, so the
        # oracle then holds every cell of the sample
        one = min(sample, 65536)
        b1 = (len(pts) - one) // 2
        t1 = time.perf_counter()
        t.calculate_range(b1, b1 + one, 1)
        d1 = time.perf_counter() - t1
        extras.update({"one_thread_value": one / d1, "one_thread_sample": f"{one} cells ({d1:.2f} s)",
                       "search_order_build_s": build})
    begin = (len(pts) - sample) // 2
    t0 = time.perf_counter()
    t.calculate_range(begin, begin + sample, nthreads)
    dt = time.perf_counter() - t0
    if keep is not None and sample == len(pts):
        keep.append(t)
    return sample / dt, dt


def parity_leg(tess, step, oracle, precisions) -> dict:
    """Every cell of the benchmark tessellation against the oracle's, bit for
    bit, in each precision: volumes, centroids, face counts, neighbour ids in
    face order and face areas."""
    ov, oc, on = oracle.summaries()
    ooff, oids = oracle.neighbors()
    _, oar = oracle.face_areas()
    out = {"cells": int(len(ov)), "compared": "volume, centroid, face count, neighbour ids, face areas",
           "checker": "oracle (C restatement of the reference's calculate), every cell"}
    for p in precisions:
        tess.set_precision(p)
        step()
        gv, gc, gn = tess.summaries()
        goff, gids = tess.neighbors()
        _, gar = tess.face_areas()
        bad = (gv != ov) | (gn != on) | np.any(gc != oc, axis=1)
        ok_csr = np.array_equal(goff, ooff) and np.array_equal(gids, oids) and np.array_equal(gar, oar)
        out[p] = {"bitwise_equal": bool(not bad.any() and ok_csr), "mismatched_cells": int(bad.sum()),
                  "neighbour_csr_equal": bool(ok_csr)}
    return out


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    nthreads = os.cpu_count() or 1
    pts = uniform(N_GEN, 0)
    from oracle.oracle import OracleTessellation
    t = OracleTessellation([0, 0, 0], [1, 1, 1], GRID, GRID, GRID)
    t.set_generators(pts)
    sample = min(args.ref_sample or N_GEN, N_GEN)
    begin = (N_GEN - sample) // 2
    for _ in range(args.warmup):
        t.calculate_range(begin, begin + sample, nthreads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        t.calculate_range(begin, begin + sample, nthreads)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * statistics.mean(times)
    value = sample / (ms / 1e3)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded PCG64 uniform)",
        "config": {"workload": WORKLOAD, "n_generators": N_GEN, "grid": [GRID] * 3,
                   "step": f"calculate() over a bounded sample of {sample} cells of the tessellation"},
        "cpu_baseline": {"value": value, "unit": "cells/s", "cores": nthreads, "kind": "port",
                         "sample": f"{sample} of {N_GEN} cells per step, OpenMP dynamic schedule"},
        "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference is Rust and no Rust toolchain exists here; this arm times the oracle, "
                "a C restatement of the reference's calculate()",
    }
    print(json.dumps(line), flush=True)
    return 0


def e2e_leg(args, L, _lib, tess, pts):
    """Same step through the C ABI with pinned host buffers: H2D of the
    generators, calculate, D2H of summaries, neighbour ids and face areas."""
    h_in = C.c_void_p()
    _lib.check(L.vd_host_alloc(3 * N_GEN * 8, C.byref(h_in)))
    C.memmove(h_in, pts.ctypes.data, 3 * N_GEN * 8)
    vol_b = C.c_void_p()
    cen_b = C.c_void_p()
    nf_b = C.c_void_p()
    _lib.check(L.vd_host_alloc(N_GEN * 8, C.byref(vol_b)))
    _lib.check(L.vd_host_alloc(3 * N_GEN * 8, C.byref(cen_b)))
    _lib.check(L.vd_host_alloc(N_GEN * 4, C.byref(nf_b)))
    tot = tess.total_faces()
    off_b = C.c_void_p()
    ids_b = C.c_void_p()
    ar_b = C.c_void_p()
    _lib.check(L.vd_host_alloc((N_GEN + 1) * 8, C.byref(off_b)))
    _lib.check(L.vd_host_alloc(int(tot * 1.2) * 4, C.byref(ids_b)))
    _lib.check(L.vd_host_alloc(int(tot * 1.2) * 8, C.byref(ar_b)))
    h = tess._h
    kept = C.c_size_t()
    e2e_ms = []
    total_faces = C.c_int64()
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        _lib.check(L.vd_tess_set_generators(h, C.cast(h_in, C.POINTER(C.c_double)), N_GEN, C.byref(kept)), h)
        _lib.check(L.vd_tess_calculate(h), h)
        _lib.check(L.vd_tess_get_cell_summaries(h, vol_b, cen_b, nf_b), h)
        _lib.check(L.vd_tess_total_faces(h, C.byref(total_faces)), h)
        _lib.check(L.vd_tess_get_neighbors(h, off_b, ids_b), h)
        _lib.check(L.vd_tess_get_face_areas(h, None, ar_b), h)
        dt = time.perf_counter() - t0
        if it >= args.warmup:
            e2e_ms.append(1e3 * dt)
    e2e = statistics.mean(e2e_ms)
    tf = total_faces.value
    h2d = 3 * N_GEN * 8
    d2h = N_GEN * (8 + 24 + 4) + (N_GEN + 1) * 8 + tf * (4 + 8)
    for b in (h_in, vol_b, cen_b, nf_b, off_b, ids_b, ar_b):
        L.vd_host_free(b)

    return e2e, h2d, d2h


def issue_roof(args, clip_ms: float, clk: dict):
    """The roof that binds this kernel: instruction issue.  Achieved warp
    instructions per second (the ncu count per cell of the committed profile
    x cells / the clip kernel's event time) against one instruction per cycle
    per SM sub-partition (4 per SM) at the sampled SM clock."""
    import torch
    per_cell = load_profile(args.precision).get("warp_instructions_per_cell")
    mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz")
    if not per_cell or not mhz:
        return None
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    achieved = per_cell * N_GEN / (clip_ms / 1e3) / 1e9
    peak = sms * 4 * mhz * 1e6 / 1e9
    return {"achieved": achieved, "peak": peak, "unit": "G warp-instructions/s", "frac": achieved / peak,
            "note": "instruction issue, the roof this kernel meets (ncu: issue active ~80%); "
                    "warp instructions per cell from the committed ncu profile"}


# algorithmic bytes per cell of the clip kernel: the generator (24 B) and its
# bin-ordered copy (32 B) in; volume, centroid, face and vertex counts
# (8 + 24 + 4 + 4 B) and ~15.5 face slots of neighbour id + area (12 B) out
CLIP_BYTES_PER_CELL = 24 + 32 + 8 + 24 + 4 + 4 + 15.5 * 12


def hbm_roof(clip_ms: float):
    """The HBM roof of the clip kernel: algorithmic bytes over its event time,
    against the measured copy bandwidth (MEASURED_PEAKS.json) or the pool's
    earlier measurement of 6.65 TB/s when that file is absent."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    peak, src = 6650.0, "fallback 6.65 TB/s (MEASURED_PEAKS.json absent)"
    if os.path.exists(path):
        with open(path) as f:
            m = json.load(f)
        if m.get("hbm_gbs"):
            peak, src = float(m["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs"
    achieved = CLIP_BYTES_PER_CELL * N_GEN / (clip_ms / 1e3) / 1e9
    return {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": src,
            "bytes_per_cell": CLIP_BYTES_PER_CELL}


def autotuned_leg(args, v, d_pts, flush):
    """The same generators on the grid the autotuner picks for them (a
    different bin grid, so a different but equally exact tessellation: each
    grid's results equal the oracle's on that grid); device-timed like
    `value`, L2 flushed before each step."""
    import torch
    from vorothree_b200 import autotune
    pts = d_pts.cpu().numpy()
    bounds = v.BoundingBox([0, 0, 0], [1, 1, 1])
    g = autotune.choose_grid(pts, bounds)
    t = v.Tessellation(bounds, v.Algorithm3DGrid(*g))
    t.set_precision(args.precision)
    stream = torch.cuda.ExternalStream(t.stream(), device=d_pts.device)
    times = []
    for it in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t.set_generators_device(d_pts.data_ptr(), N_GEN)
        t.calculate()
        e1.record(stream)
        e1.synchronize()
        if it >= args.warmup:
            times.append(e0.elapsed_time(e1))
    t.close()
    ms = statistics.mean(times)
    return {"grid": list(g), "value": N_GEN / (ms / 1e3), "ms_per_step": ms,
            "note": "same step on the autotuner's grid for this input"}


def tuning_args(args) -> dict:
    """The first tier's launch settings from the command line (profiling and
    A/B runs; the defaults are the library's)."""
    out = {}
    if args.fast_layout:
        out["fast_layout"] = args.fast_layout
    if args.fast_blocks:
        out["fast_blocks_per_sm"] = args.fast_blocks
    return out


def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    import vorothree_b200 as v
    from vorothree_b200 import _lib

    L = v.load()
    pts = uniform(N_GEN, rank)
    d_pts = torch.from_numpy(pts).to(f"cuda:{local}")
    tess = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(GRID, GRID, GRID))
    tess.set_precision(args.precision)
    tess.set_tuning(tuning_args(args))
    stream = torch.cuda.ExternalStream(tess.stream(), device=f"cuda:{local}")
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def step():
        tess.set_generators_device(d_pts.data_ptr(), N_GEN)
        tess.calculate()

    # the event counters of this input (deterministic) for the flop model,
    # from one instrumented run outside the timed region
    tess.set_instrumentation(True)
    step()
    counters = tess.counters()
    tess.set_instrumentation(False)

    def barrier():
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed(precision):
        """K device-timed steps (L2 flushed before each), after W warm-up steps."""
        tess.set_precision(precision)
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        sm, cm, bm = [], [], []
        c0 = C.c_uint64()
        L.vd_launch_count(C.byref(c0))
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            sm.append(e0.elapsed_time(e1))
            tm = tess.timings()
            cm.append(tm["clip_ms"])
            bm.append(tm["bin_ms"])
        c1 = C.c_uint64()
        L.vd_launch_count(C.byref(c1))
        launches.append(int(c1.value - c0.value))
        return sm, cm, bm

    launches = []
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    step_ms, clip_ms, bin_ms = timed(args.precision)
    other = None
    if not args.no_mixed:
        alt = "mixed" if args.precision == "fp64" else "fp64"
        osm, ocm, _ = timed(alt)
        other = (alt, osm, ocm)
        tess.set_precision(args.precision)
    barrier()
    clk = clocks.stop()
    ms = statistics.mean(step_ms)
    if ws > 1:
        tt = torch.tensor([ms], device=f"cuda:{local}", dtype=torch.float64)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        ms = float(tt.item())
    value = ws * N_GEN / (ms / 1e3)
    fb = tess.fallback_counts()

    # ---- end to end through the C ABI with pinned host buffers ----
    e2e, h2d, d2h = e2e_leg(args, L, _lib, tess, pts) if not args.no_e2e else (None, None, None)
    if e2e is not None and ws > 1:
        tt = torch.tensor([e2e], device=f"cuda:{local}", dtype=torch.float64)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        e2e = float(tt.item())
    line = None
    if rank == 0:
        flops = flop_count(counters)
        clip = statistics.mean(clip_ms)
        peak = C.c_double()
        _lib.check(L.vd_measure_fma_peak(1, C.byref(peak)))
        achieved = flops / (clip / 1e3) / 1e12
        traffic = load_traffic(args.precision)
        line = {
            "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32-classify/f64",
            "data": "synthetic (seeded PCG64 uniform; rank r uses seed r)",
            "config": {"workload": WORKLOAD, "n_generators": N_GEN, "grid": [GRID] * 3,
                       "precision": args.precision, "step": "set_generators (device input) + calculate",
                       "l2": "flushed (512 MiB write) before every timed step",
                       "parallelism": f"{ws} independent tessellations, one per GPU"},
            "phases_ms": {"binning": statistics.mean(bin_ms), "clip_kernel": clip},
            "roofline": {"bound": "fp64", "kernel": "k_clip_sparse (warp-per-cell clip + reductions, slot layout)",
                         "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                         "frac": achieved / peak.value,
                         "peak_source": "FP64 FMA-chain microbenchmark run live by bench.py on this GPU, right "
                                        "after the timed steps (MEASURED_PEAKS.json has no FP64 figure)",
                         "peak_clock_mhz": clk.get("sm_mhz"),
                         "flops_per_launch": flops, "traffic": traffic,
                         "issue": issue_roof(args, clip, clk), "hbm": hbm_roof(clip),
                         "note": "bound names the kernel's only arithmetic roof (FP64 pipe, no tensor cores);"
                                 " it is issue-bound (roofline.issue), far from HBM (roofline.hbm)"},
            "e2e": None if e2e is None else {
                "value": N_GEN / (e2e / 1e3) * ws, "unit": "cells/s", "ms_per_step": e2e,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches[0],
            "gpu_launches_note": "kernels this library launched during the K timed steps (binning + clip)",
            "clocks": clk,
            "fallback_cells": fb,
        }
        if ws == 1 and not args.no_autotuned:
            line["autotuned_grid"] = autotuned_leg(args, v, d_pts, flush)
        if other is not None:
            alt, osm, ocm = other
            oms = statistics.mean(osm)
            line[alt] = {"value": ws * N_GEN / (oms / 1e3), "ms_per_step": oms,
                         "clip_kernel_ms": statistics.mean(ocm),
                         f"speedup_vs_{args.precision}": ms / oms,
                         "note": "same outputs bit for bit (mixed decisions equal FP64's)"}
        if ws == 1 and not args.no_serving:
            reqs = serving_requests(24)
            srv = v.TessellationServer(slots=4, hbm_budget_bytes=32 << 30, precision=args.precision)
            for r in reqs[:2]:
                srv.take(srv.submit(*r))
            res = serve_at_rate(srv, reqs, 30.0)
            srv.close()
            line["serving"] = dict(res, note="Poisson arrivals; sizes log-uniform [1e3,1e6], half clustered, "
                                             "0-2 walls; 4 slots; p50/p99 = submit-to-result latency")
        if ws == 1 and not args.no_cpu_baseline:
            nthreads = os.cpu_count() or 1
            sample = min(args.cpu_sample or N_GEN, N_GEN)
            extras = {}
            keep = []
            cv, cdt = cpu_baseline(pts, nthreads, sample, extras, keep)
            line["cpu_baseline"] = dict({"value": cv, "unit": "cells/s", "cores": nthreads, "kind": "port",
                                         "sample": f"{sample} of {N_GEN} cells of the same tessellation "
                                                   f"({cdt:.2f} s wall)"}, **extras)
            if keep:
                line["parity"] = parity_leg(tess, step, keep[0], ["fp64", "mixed"])
                tess.set_precision(args.precision)
                del keep[:]
        if ws == 1 and not args.no_side_configs:
            # the other benchmark configurations, each in its own key: the
            # clustered input, the batch with Lloyd steps, the serving sweep
            line["clustered"] = blobs_leg(args, 4_194_304, args.precision, 3)
            line["batched"] = batched_leg(args, args.ntess, 3, args.lloyd_steps)
            line["serving_sweep"] = serving_leg(args, args.serve_requests, args.serve_rates)
            line["serving_sweep"]["burst"] = burst_leg(args)
        print(json.dumps(line), flush=True)
    tess.close()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def batched_members(ntess: int, seed: int = 0):
    from vorothree_b200.workloads import batch_members
    return batch_members(ntess, seed)


def bounds_of(edge):
    import vorothree_b200 as v
    return v.BoundingBox([0, 0, 0], list(edge))


def batched_leg(args, ntess: int, calc_steps: int, lloyd_steps: int) -> dict:
    """Config: many independent tessellations in one persistent launch, then
    Lloyd steps (relax -> calculate) replayed from a CUDA graph."""
    import vorothree_b200 as v
    t0 = time.perf_counter()
    ms = batched_members(ntess)
    b = v.TessellationBatch()
    b.set_precision(args.precision)
    for edge, grid, pts, sphere in ms:
        walls = [v.Wall(v.WALL_ID_MAX, v.SphereGeometry(sphere[0], sphere[1]))] if sphere else []
        b.add(v.BoundingBox([0, 0, 0], list(edge)), grid, pts, walls)
    b.commit()
    setup_s = time.perf_counter() - t0
    n_in = sum(len(m[2]) for m in ms)
    cells = b.total_cells()
    calc = []
    for _ in range(1 + calc_steps):
        b.calculate()
        calc.append(b.timing_ms())
    calc_ms = statistics.mean(calc[1:])
    b.lloyd(1)  # captures the step graph
    b.lloyd(lloyd_steps)
    lloyd_ms = b.timing_ms()
    cells_after = b.total_cells()
    b.close()
    return {"value": cells / (calc_ms / 1e3), "unit": "cells/s", "ms_per_calculate": calc_ms,
            "calculates_timed": calc_steps,
            "config": {"tessellations": ntess, "generators_in": n_in, "cells": cells,
                       "sizes": "log-uniform [64, 65536]", "box_edges": "U[1,10]",
                       "walls": "even members: centred sphere r = 0.5 min(edge)",
                       "grid": "bins per axis ~ edge * (N/V)^(1/3) at the autotuner's density"},
            "lloyd": {"steps": lloyd_steps, "ms_total": lloyd_ms, "ms_per_step": lloyd_ms / lloyd_steps,
                      "cells_per_s": cells_after * lloyd_steps / (lloyd_ms / 1e3),
                      "cells_after": cells_after, "note": "each step = relax + wall filter + re-bin + calculate, "
                      "replayed from one CUDA graph"},
            "setup_s": setup_s, "timing": "CUDA events on the batch's stream (device time)"}


def run_batched(args):
    import torch
    torch.cuda.set_device(0)
    res = batched_leg(args, args.ntess, args.steps, args.lloyd_steps)
    line = {"metric": "3D cells/s, batched tessellations", "workload": "batched", "unit": "cells/s",
            "value": res["value"], "n_gpus": 1, "steps": args.steps, "warmup": 1, "higher_is_better": True,
            "dtype": "f64", "precision": args.precision, "data": "synthetic (seeded PCG64)"}
    line.update(res)
    print(json.dumps(line), flush=True)
    return 0


def serving_requests(count: int, seed: int = 0, sizes=(1e3, 1e6)):
    from vorothree_b200.workloads import serving_requests as make
    return make(count, seed, sizes)


def serve_at_rate(srv, reqs, rate: float, seed: int = 1):
    """Submit reqs at Poisson arrival times of the given rate (req/s) from one
    thread, collect them from another; returns p50/p99 latency and cells/s."""
    import threading
    rng = np.random.Generator(np.random.PCG64(seed))
    gaps = rng.exponential(1.0 / rate, size=len(reqs))
    tickets = [None] * len(reqs)
    ready = [threading.Event() for _ in reqs]
    srv.reset_stats()
    t0 = time.perf_counter()

    def submitter():
        due = t0
        for k, r in enumerate(reqs):
            due += gaps[k]
            delay = due - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            tickets[k] = srv.submit(*r)
            ready[k].set()
    th = threading.Thread(target=submitter)
    th.start()
    cells = 0
    for k in range(len(reqs)):
        ready[k].wait()
        n, _ = srv.wait(tickets[k])
        srv.take(tickets[k])
        cells += n
    th.join()
    wall = time.perf_counter() - t0
    st = srv.stats()
    return {"rate_req_s": rate, "requests": len(reqs), "p50_ms": 1e3 * st["p50_s"], "p99_ms": 1e3 * st["p99_s"],
            "cells": cells, "cells_per_s": cells / wall, "wall_s": wall, "peak_admitted_bytes": st["peak_bytes"]}


def serving_leg(args, nreq: int, rates) -> dict:
    import vorothree_b200 as v
    reqs = serving_requests(nreq)
    srv = v.TessellationServer(slots=args.serve_slots, hbm_budget_bytes=args.serve_budget_gb << 30,
                               precision=args.precision)
    # warm every slot's buffers on the whole request set (the sweep measures
    # the steady state, not the first growth of a slot's buffers)
    for t in [srv.submit(*r) for r in reqs]:
        srv.take(t)
    sweep = [serve_at_rate(srv, reqs, rate) for rate in rates]
    srv.close()
    return {"config": {"slots": args.serve_slots, "hbm_budget_gb": args.serve_budget_gb, "requests": nreq,
                       "sizes": "log-uniform [1e3, 1e6]", "mix": "half uniform, half 8-blob clustered",
                       "walls": "0-2 of plane / centred sphere", "arrivals": "Poisson"},
            "sweep": sweep, "latency": "submit-to-result wall clock per request"}


def burst_leg(args, nreq: int = 256) -> dict:
    """A burst of small requests (sizes log-uniform in [1e3, 3.2e4], the
    serving mix otherwise) submitted at once, served with the merging of small
    requests into batches (up to 64 or 8 a batch) and without it: wall time from the first submit to
    the last result, cells/s, p50/p99 latency and the batches formed."""
    import vorothree_b200 as v
    reqs = serving_requests(nreq, seed=5, sizes=(1e3, 3.2e4))
    out = {"config": {"requests": nreq, "sizes": "log-uniform [1e3, 3.2e4]", "slots": args.serve_slots,
                      "arrivals": "all at once"}}
    for mode, members in (("merged", 64), ("merged_8", 8), ("alone", 0)):
        srv = v.TessellationServer(slots=args.serve_slots, hbm_budget_bytes=args.serve_budget_gb << 30,
                                   precision=args.precision)
        if members:
            srv.set_merging(max_members=members)
        for _ in range(3):  # warm the slots' buffers and batches twice, measure the third pass
            srv.reset_stats()
            t0 = time.perf_counter()
            tickets = [srv.submit(*r) for r in reqs]
            cells = sum(srv.wait(t)[0] for t in tickets)
            for t in tickets:
                srv.take(t)
            wall = time.perf_counter() - t0
        st = srv.stats()
        ms = srv.merge_stats()
        srv.close()
        out[mode] = {"wall_ms": 1e3 * wall, "cells": cells, "cells_per_s": cells / wall,
                     "p50_ms": 1e3 * st["p50_s"], "p99_ms": 1e3 * st["p99_s"], **ms}
    return out


def run_serving(args):
    import torch
    torch.cuda.set_device(0)
    res = serving_leg(args, args.serve_requests, args.serve_rates)
    res["burst"] = burst_leg(args)
    line = {"metric": "serve p50/p99 latency", "workload": "serving", "unit": "ms", "n_gpus": 1,
            "higher_is_better": False, "value": res["sweep"][0]["p99_ms"], "precision": args.precision,
            "data": "synthetic (seeded PCG64)"}
    line.update(res)
    print(json.dumps(line), flush=True)
    return 0


def blob_classes(t, pts, nb, kept, args):
    """Time and count the blob cells and the background cells apart: the wall
    filter keeps the input order, so the kept blob generators are cell ids
    [0, nbk) and the background ones [nbk, kept).  Per-cell event counts come
    from the instrumented kernel over the same range."""
    d = pts[:nb] - 0.5
    nbk = int(((d * d).sum(1) <= 0.45 ** 2).sum())
    out = {}
    for name, (b, e) in (("blob", (0, nbk)), ("background", (nbk, kept))):
        times = []
        for _ in range(max(3, args.steps)):
            t.calculate_range(b, e)
            tm = t.timings()
            times.append(tm["clip_ms"] + tm["fallback_ms"])
        t.set_instrumentation(True)
        t.calculate_range(b, e)
        c = t.counters()
        t.set_instrumentation(False)
        n = max(1, e - b)
        out[name] = {"cells": e - b, "ms": min(times), "ns_per_cell": 1e6 * min(times) / n,
                     "per_cell": {k: round(c[k] / n, 2) for k in ("offsets", "candidates", "clips", "modifying")}}
    return out


def run_suite(args):
    """The grid cases of the reference's criterion benches on one B200, with
    the oracle (the C restatement of calculate) timed on the host cores on the
    same generators: benches/scaling.rs (N = 10 .. 1 M in a 100^3 box,
    ceil(N^(1/3)) bins per axis), benches/capacity.rs (100 k generators, 0.25
    to 20 per bin) and benches/distributions.rs (uniform, axes, central box,
    sphere surface at 1 k and 10 k; the trefoil-knot wall is not built).  A
    case's time is calculate() as a caller sees it (host wall clock, launches
    and synchronisation included) after warm-up; device time beside it."""
    import torch
    import vorothree_b200 as v
    from oracle.oracle import OracleTessellation
    from vorothree_b200.workloads import bench_distribution
    torch.cuda.set_device(0)
    nthreads = os.cpu_count() or 1
    box = ([0.0, 0.0, 0.0], [100.0, 100.0, 100.0])

    from vorothree_b200 import autotune

    def case(group, label, n, g, pts=None, seed=0):
        t = v.Tessellation(v.BoundingBox(*box), v.Algorithm3DGrid(g, g, g))
        if pts is None:
            t.random_generators(n, seed)
        else:
            t.set_generators(pts)
        # the library's tuned launch settings for this input's class and size
        # (the grid stays the bench's own heuristic)
        cls = autotune.distribution_class(t.generators(), v.BoundingBox(*box))
        tun = autotune.input_tuning(t.generators(), v.BoundingBox(*box))
        t.set_tuning(tun)
        t.calculate()
        one = t.timings()["total_ms"]
        reps = max(1, min(args.steps, int(2000.0 / max(one, 1e-3))))
        wall, dev = [], []
        for _ in range(reps):
            t0 = time.perf_counter()
            t.calculate()
            wall.append(1e3 * (time.perf_counter() - t0))
            tm = t.timings()
            dev.append(tm["clip_ms"] + tm["fallback_ms"])
        row = {"group": group, "case": label, "n": n, "grid": g, "gpu_ms": statistics.mean(wall),
               "gpu_device_ms": statistics.mean(dev), "fallback_cells": t.fallback_counts(),
               "class": cls, "tuning": tun}
        if n <= 100_000:
            gens = t.generators()
            o = OracleTessellation(*box, g, g, g)
            o.set_generators(gens)
            o.calculate(nthreads)
            cw = []
            for _ in range(3):
                t0 = time.perf_counter()
                o.calculate(nthreads)
                cw.append(1e3 * (time.perf_counter() - t0))
            row["cpu_ms"] = statistics.mean(cw)
            row["speedup"] = row["cpu_ms"] / row["gpu_ms"]
            gv, _, gn = t.summaries()
            ov, _, on = o.summaries()
            row["bitwise_equal"] = bool(np.array_equal(gv, ov) and np.array_equal(gn, on))
        t.close()
        return row

    rows = []
    for n in (10, 100, 1000, 10_000, 100_000, 1_000_000):
        rows.append(case("scaling", "uniform", n, max(1, int(np.ceil(n ** (1.0 / 3.0)))), seed=n))
    for cap in (0.25, 0.5, 1.0, 2.0, 3.0, 4.0, 6.0, 8.0, 12.0, 20.0):
        g = max(1, int(np.ceil((100_000 / cap) ** (1.0 / 3.0))))
        rows.append(case("capacity", f"{cap} per bin", 100_000, g, seed=7))
    for n in (1000, 10_000):
        g = max(1, int(np.ceil(n ** (1.0 / 3.0))))
        for kind in ("uniform", "axes", "central", "sphere"):
            rows.append(case("distributions", kind, n, g, pts=bench_distribution(kind, n, 11, *box)))
    line = {"metric": "calculate() time on the reference's criterion bench cases", "workload": "suite",
            "unit": "ms", "n_gpus": 1, "higher_is_better": False, "dtype": "f64",
            "data": "synthetic (seeded: random_generators / PCG64)",
            "cpu": {"kind": "port", "cores": nthreads,
                    "note": "the oracle, a C restatement of the reference's calculate(), N <= 100 k"},
            "rows": rows}
    print(json.dumps(line), flush=True)
    return 0


def blobs_leg(args, n: int, precision: str, steps: int, extra_grids=()) -> dict:
    """Config: n generators (4,194,304), 70% in 64 isotropic Gaussian blobs
    (sigma 0.01, centres uniform) + 30% uniform background, clipped by a
    sphere wall r = 0.45 at the centre of the unit cube, on the autotuner's
    grid.  A step is calculate() on the resident, binned generators."""
    import vorothree_b200 as v
    from vorothree_b200 import autotune
    from vorothree_b200.workloads import clustered_blobs
    pts, nb = clustered_blobs(n, 0)
    bounds = v.BoundingBox([0, 0, 0], [1, 1, 1])
    tuned = autotune.choose_grid(pts, bounds)
    grids = [tuned] + [(g, g, g) for g in extra_grids if (g, g, g) != tuned]
    res = []
    for g in grids:
        t = v.Tessellation(bounds, v.Algorithm3DGrid(*g))
        t.set_precision(precision)
        t.add_wall(v.Wall(v.WALL_ID_MAX, v.SphereGeometry([0.5, 0.5, 0.5], 0.45)))
        kept = t.set_generators(pts)
        times, fall = [], []
        for _ in range(3 + steps):
            t.calculate()
            tm = t.timings()
            times.append(tm["clip_ms"] + tm["fallback_ms"])
            fall.append(tm["fallback_ms"])
        ms = statistics.mean(times[3:])
        res.append({"grid": list(g), "kept": kept, "ms": ms, "cells_per_s": kept / (ms / 1e3),
                    "fallback_cells": t.fallback_counts(), "fallback_ms": statistics.mean(fall[3:])})
        if g == tuned:
            res[-1]["classes"] = blob_classes(t, pts, nb, kept, args)
        t.close()
    return {"value": res[0]["cells_per_s"], "unit": "cells/s", "precision": precision,
            "config": {"generators": n, "blobs": 64, "sigma": 0.01, "blob_fraction": 0.7,
                       "wall": "sphere r=0.45 at (0.5,0.5,0.5)", "grid": list(tuned),
                       "grid_source": "autotuner table (vorothree_b200/autotune_table.json)",
                       "distribution_class": autotune.distribution_class(pts, bounds)},
            "timing": "CUDA events on the tessellation's stream (clip passes incl. fallback tiers)",
            "per_grid": res}


def run_blobs(args):
    import torch
    torch.cuda.set_device(0)
    res = blobs_leg(args, args.blob_n, args.precision, args.steps, args.blob_grids)
    line = {"metric": "3D cells/s, clustered generators", "workload": "blobs", "unit": "cells/s",
            "value": res["value"], "n_gpus": 1, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic (seeded PCG64)"}
    line.update(res)
    print(json.dumps(line), flush=True)
    return 0


def run_sealed(args):
    """Config: the 1,048,576 uniform generators with a sphere wall r = 0.45 at
    the centre, computed by calculate and by calculate_sealed (the second pass
    re-clips the cells on the curved wall with their neighbours' tangent
    planes, tessellation.rs:234-318); the oracle times the same on the host."""
    import torch
    import vorothree_b200 as v
    torch.cuda.set_device(0)
    pts = uniform(N_GEN, 0)
    wall = v.Wall(v.WALL_ID_MAX, v.SphereGeometry([0.5, 0.5, 0.5], 0.45))
    t = v.Tessellation(v.BoundingBox([0, 0, 0], [1, 1, 1]), v.Algorithm3DGrid(GRID, GRID, GRID))
    t.add_wall(wall)
    kept = t.set_generators(pts)
    res = {}
    for name, fn in (("calculate", t.calculate), ("calculate_sealed", t.calculate_sealed)):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ms.append(1e3 * (time.perf_counter() - t0))
        res[name] = statistics.mean(ms)
    nseal = len(t.seal_log) // 3
    t0 = time.perf_counter()
    t.prune_boundaries()
    prune_ms = 1e3 * (time.perf_counter() - t0)
    nprune = len(t.prune_log) // 4
    t.close()
    line = {"metric": "3D cells/s, calculate_sealed", "workload": "sealed", "unit": "cells/s",
            "value": kept / (res["calculate_sealed"] / 1e3), "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "dtype": "f64", "data": "synthetic (seeded PCG64)",
            "config": {"generators": N_GEN, "kept": kept, "grid": [GRID] * 3, "wall": "sphere r=0.45 at the centre",
                       "timing": "host wall clock around each call with a device synchronize"},
            "ms": {"calculate": res["calculate"], "calculate_sealed": res["calculate_sealed"],
                   "seal_pass": res["calculate_sealed"] - res["calculate"], "prune_boundaries": prune_ms},
            "seal_clips": nseal, "prune_entries": nprune}
    if not args.no_cpu_baseline:
        from oracle.oracle import OracleTessellation
        o = OracleTessellation([0, 0, 0], [1, 1, 1], GRID, GRID, GRID)
        o.add_wall_sphere([0.5, 0.5, 0.5], 0.45, v.WALL_ID_MAX)
        o.set_generators(pts)
        nthreads = os.cpu_count() or 1
        t0 = time.perf_counter()
        o.calculate_sealed(nthreads)
        cdt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": kept / cdt, "unit": "cells/s", "cores": nthreads, "kind": "port",
                                "sample": f"all {kept} cells; calculate on {nthreads} threads, the seal pass "
                                          f"on one ({cdt:.2f} s wall)"}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["uniform", "batched", "blobs", "serving", "sealed", "suite"],
                    default="uniform",
                    help="uniform: 1M uniform generators (the headline); batched: many tessellations "
                         "+ Lloyd steps; blobs: 4M clustered generators with a sphere wall")
    ap.add_argument("--ntess", type=int, default=4096)
    ap.add_argument("--blob-n", type=int, default=4_194_304,
                    help="generators of the blobs workload (profiling runs use a smaller case)")
    ap.add_argument("--serve-requests", type=int, default=48)
    ap.add_argument("--serve-slots", type=int, default=4)
    ap.add_argument("--serve-budget-gb", type=int, default=32)
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[10.0, 30.0, 60.0])
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-autotuned", action="store_true", help="skip the autotuned-grid leg (uniform workload)")
    ap.add_argument("--lloyd-steps", type=int, default=20)
    ap.add_argument("--blob-grids", type=int, nargs="*", default=[],
                    help="cubic grids timed beside the autotuned one (blobs workload)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="cells of the CPU baseline (0 = every cell of the workload)")
    ap.add_argument("--ref-sample", type=int, default=0,
                    help="cells per step of the reference arm (0 = every cell of the workload)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fast-layout", choices=["slots", "full"], default=None,
                    help="first-tier polytope layout (default: the library's)")
    ap.add_argument("--fast-blocks", type=int, choices=[5, 6, 7], default=None,
                    help="first-tier blocks per SM, slot layout (default: the library's)")
    ap.add_argument("--no-side-configs", action="store_true",
                    help="skip the clustered, batched and serving-sweep keys of the default line")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--n", type=int, default=N_GEN, help="generators (profiling runs use a smaller case)")
    ap.add_argument("--grid", type=int, default=GRID)
    args = ap.parse_args()
    set_workload(args.n, args.grid)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "suite":
        return run_suite(args)
    if args.workload == "blobs":
        return run_blobs(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "sealed":
        return run_sealed(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
