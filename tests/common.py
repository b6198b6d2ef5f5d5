"""Shared helpers for the tests: seeded inputs and oracle/GPU comparisons."""
import json
import os

import numpy as np

from vorothree_b200.workloads import bench_distribution  # noqa: F401  (re-exported for the tests)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def uniform(n, lo, hi, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.uniform(lo, hi, size=(n, 3))


def blobs(n, nblobs, sigma, frac_blob, seed):
    """frac_blob of the points from isotropic Gaussian blobs (centres uniform in
    the unit cube, points assigned round-robin), the rest uniform."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nb = int(round(frac_blob * n))
    centres = rng.uniform(0.0, 1.0, size=(nblobs, 3))
    pts_b = centres[np.arange(nb) % nblobs] + rng.normal(0.0, sigma, size=(nb, 3))
    pts_u = rng.uniform(0.0, 1.0, size=(n - nb, 3))
    return np.concatenate([pts_b, pts_u])


def csr_lists(off, vals):
    return [vals[off[i]:off[i + 1]] for i in range(len(off) - 1)]

