"""Seeded synthetic inputs: the generator sets of the benchmark configurations
(1 M uniform, 4 M clustered with a sphere wall, 4096-member batches, serving
request streams) and the shapes of the reference's criterion benchmarks
(benches/distributions.rs).  Used by the benchmark driver and the parity
tests, so both see the same inputs; not part of the tessellation path."""
import numpy as np


def uniform_cube(n, seed=0):
    """n generators i.i.d. uniform in the unit cube (numpy PCG64(seed))."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.uniform(0.0, 1.0, size=(n, 3))


def clustered_blobs(n=4_194_304, seed=0, nblobs=64, sigma=0.01, frac=0.7):
    """frac of n generators from nblobs isotropic Gaussian blobs (sigma, centres
    uniform in the unit cube, points assigned round-robin), then the rest
    uniform in the unit cube, blobs first.  Returns (points, blob count).  With
    the defaults and a sphere wall r = 0.45 at the cube's centre this is the
    clustered benchmark configuration."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nb = int(round(frac * n))
    centres = rng.uniform(0.0, 1.0, size=(nblobs, 3))
    pts = np.concatenate([centres[np.arange(nb) % nblobs] + rng.normal(0.0, sigma, size=(nb, 3)),
                          rng.uniform(0.0, 1.0, size=(n - nb, 3))])
    return pts, nb


def batch_members(ntess=4096, seed=0):
    """Members of the batched configuration: N log-uniform in [64, 65536], box
    edges U[1,10] from the origin, even members with a centred sphere wall of
    radius 0.5 min(edge); near-cubic bins at the autotuner's density for
    uniform input of the member's size.  Each member is (edge[3], grid[3],
    points, (centre, radius) or None)."""
    from . import autotune
    from .tessellation import BoundingBox
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k in range(ntess):
        n = int(round(np.exp(rng.uniform(np.log(64), np.log(65536)))))
        edge = rng.uniform(1.0, 10.0, size=3)
        grid = list(autotune.grid_for(n, BoundingBox([0, 0, 0], list(edge)), autotune.lookup("uniform", n)))
        pts = rng.uniform(0.0, 1.0, size=(n, 3)) * edge
        sphere = (list(edge / 2.0), 0.5 * float(edge.min())) if k % 2 == 0 else None
        out.append((edge, grid, pts, sphere))
    return out


def serving_requests(count, seed=0, sizes=(1e3, 1e6)):
    """Requests of the serving configuration: sizes log-uniform in [1e3, 1e6]
    (or the given range);
    half uniform, half clustered (8 Gaussian blobs, sigma 0.03, 70% of the
    points); 0-2 walls drawn from {plane through the centre with a random
    normal, centred sphere of radius U[0.3, 0.5]}; grid from the autotuner.
    Each request is (bounds, grid, points, walls)."""
    from . import autotune
    from .tessellation import WALL_ID_MAX, BoundingBox, PlaneGeometry, SphereGeometry, Wall
    bounds = BoundingBox([0, 0, 0], [1, 1, 1])
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k in range(count):
        n = int(round(np.exp(rng.uniform(np.log(sizes[0]), np.log(sizes[1])))))
        clustered = rng.uniform() < 0.5
        if clustered:
            nb = int(0.7 * n)
            c = rng.uniform(0.1, 0.9, size=(8, 3))
            pts = np.concatenate([c[np.arange(nb) % 8] + rng.normal(0.0, 0.03, size=(nb, 3)),
                                  rng.uniform(0.0, 1.0, size=(n - nb, 3))])
        else:
            pts = rng.uniform(0.0, 1.0, size=(n, 3))
        grid = autotune.choose_grid(pts, bounds)
        walls = []
        for w in range(int(rng.integers(0, 3))):
            if rng.uniform() < 0.5:
                walls.append(Wall(WALL_ID_MAX - w, PlaneGeometry([0.5, 0.5, 0.5], list(rng.normal(size=3)))))
            else:
                walls.append(Wall(WALL_ID_MAX - w, SphereGeometry([0.5, 0.5, 0.5], float(rng.uniform(0.3, 0.5)))))
        out.append((bounds, grid, pts, walls))
    return out


def bench_distribution(kind, n, seed, lo=(0.0, 0.0, 0.0), hi=(100.0, 100.0, 100.0)):
    """The generator distributions of the reference's criterion benches
    (benches/distributions.rs), seeded: "axes" (each coordinate 0.5 + 4 (u -
    0.5)^3 of the extent, crowding the three mid-planes), "central" (uniform in
    a centred box of a tenth of the volume), "sphere" (the centre, then points
    on a sphere of radius min(extent) / 3, from directions rejection-sampled in
    the unit ball with 1e-4 < |v|^2 <= 1), or "uniform"."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    ext = hi - lo
    c = (lo + hi) / 2.0
    if kind == "uniform":
        return lo + rng.uniform(0.0, 1.0, size=(n, 3)) * ext
    if kind == "axes":
        u = rng.uniform(0.0, 1.0, size=(n, 3))
        return lo + (0.5 + 4.0 * (u - 0.5) ** 3) * ext
    if kind == "central":
        s = 0.1 ** (1.0 / 3.0)
        return c + (rng.uniform(0.0, 1.0, size=(n, 3)) - 0.5) * ext * s
    if kind == "sphere":
        r = ext.min() / 3.0
        out = [c]
        while len(out) < n:
            v = rng.uniform(-1.0, 1.0, size=(2 * n, 3))
            l2 = (v * v).sum(1)
            v = v[(l2 > 1e-4) & (l2 <= 1.0)]
            out.extend(c + v / np.sqrt((v * v).sum(1))[:, None] * r)
        return np.asarray(out[:n])
    raise ValueError(kind)
