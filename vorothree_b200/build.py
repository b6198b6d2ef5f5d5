"""Build the CUDA library in-tree: vorothree_b200/libvoronoid_b200.so (sm_100a).

    python -m vorothree_b200.build          # or vorothree_b200.build.build()

Every translation unit that does FP64 work is compiled with -fmad=false: the
FP64 arithmetic must round exactly like the reference, which never fuses a
multiply and an add (the mixed path's FP32 classification uses explicit fmaf).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvoronoid_b200.so")
BUILD_DIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
          "-Xptxas", "-warn-spills"]
# (source, fused multiply-add allowed)
SOURCES = [
    ("vd_kernels_fp64.cu", False),
    ("vd_kernels_mixed.cu", False),
    ("vd_kernels_sparse.cu", False),
    ("vd_host.cu", False),
    ("vd_measure.cu", True),
    ("vd_noalloc.cu", False),
    ("vd_batch.cu", False),
    ("vd_server.cu", False),
    ("vd_cell.cu", False),
    ("vd_seal.cu", False),
    ("vd_text.cpp", False),
    ("vd_export.cu", False),
]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "voronoid_b200.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD_DIR, exist_ok=True)
    objs, procs = [], []
    # translation units compile in parallel; any failure fails the build
    for src, fma in SOURCES:
        obj = os.path.join(BUILD_DIR, os.path.splitext(src)[0] + ".o")
        if os.path.exists(obj):
            os.unlink(obj)
        cmd = [nvcc(), *ARCH, *COMMON, "-fmad=" + ("true" if fma else "false"),
               "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd)))
        objs.append(obj)
    failed = [src for src, p in procs if p.wait() != 0]
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(failed))
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
