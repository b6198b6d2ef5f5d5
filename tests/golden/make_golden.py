"""Convert the reference's Voro++ golden data into committed fixtures.

Reads the reference crate's tests/data/{face_counts,vertex_positions}/
{generators,output}.txt (generated by Voro++, see the code.txt beside them)
and writes JSON fixtures next to this script.  Run once in a checkout that has
the reference mounted:

    python tests/golden/make_golden.py /path/to/reference

The fixtures, not the reference, are what the tests read.
"""
import json
import os
import sys


def read_generators(path):
    out = []
    with open(path) as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            # Tessellation::import_generators: id then x y z; missing -> 0.0
            xyz = []
            for k in range(3):
                try:
                    xyz.append(float(parts[1 + k]))
                except (IndexError, ValueError):
                    xyz.append(0.0)
            out.append([int(parts[0])] + xyz)
    return out


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    fc_dir = os.path.join(ref, "tests", "data", "face_counts")
    gens = read_generators(os.path.join(fc_dir, "generators.txt"))
    counts = {}
    with open(os.path.join(fc_dir, "output.txt")) as f:
        for line in f:
            p = line.split()
            if len(p) == 2:
                counts[int(p[0])] = int(p[1])
    with open(os.path.join(here, "voro_face_counts.json"), "w") as f:
        json.dump({
            "source": "reference tests/data/face_counts (Voro++ output)",
            "bounds_min": [-10.0, -10.0, -10.0], "bounds_max": [10.0, 10.0, 10.0],
            "grid": [6, 6, 6], "walls": [],
            "generators": gens, "face_counts": counts}, f, indent=0)

    vp_dir = os.path.join(ref, "tests", "data", "vertex_positions")
    gens = read_generators(os.path.join(vp_dir, "generators.txt"))
    cells = {}
    cur = None
    with open(os.path.join(vp_dir, "output.txt")) as f:
        for line in f:
            line = line.strip()
            if not line:
                continue
            if line.startswith("Cell"):
                cur = int(line.split()[1].rstrip(":"))
                cells[cur] = []
            elif cur is not None:
                c = [float(x) for x in line.split()]
                if len(c) == 3:
                    cells[cur].append(c)
    with open(os.path.join(here, "voro_vertex_positions.json"), "w") as f:
        json.dump({
            "source": "reference tests/data/vertex_positions (Voro++ output)",
            "bounds_min": [-10.0, -10.0, -10.0], "bounds_max": [10.0, 10.0, 10.0],
            "grid": [6, 6, 6],
            "walls": [{"kind": "sphere", "center": [0.0, 0.0, 0.0], "radius": 8.0, "id": -1000}],
            "generators": gens, "cells": cells}, f, indent=0)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference checkout>")
    main(sys.argv[1])
