"""Synthetic generator sets shaped like the inputs of the reference's criterion
benchmarks (benches/distributions.rs), seeded so runs repeat.  Used by the
benchmark driver and the parity tests; not part of the tessellation path."""
import numpy as np


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
