"""The bin-density autotuner: host-side classification and table logic on
CPU; one tuning pass on the GPU."""
import numpy as np
import pytest

from common import blobs, uniform


def test_grid_for_density():
    import vorothree_b200 as v
    from vorothree_b200.autotune import grid_for
    b = v.BoundingBox([0, 0, 0], [1, 1, 1])
    assert grid_for(1_000_000, b, 1.0) == (100, 100, 100)
    assert grid_for(1_000_000, b, 2.0) == (200, 200, 200)
    b2 = v.BoundingBox([0, 0, 0], [8, 1, 1])
    assert grid_for(8000, b2, 1.0) == (80, 10, 10)
    assert grid_for(0, b, 1.0) == (1, 1, 1)


def test_distribution_class():
    import vorothree_b200 as v
    from vorothree_b200.autotune import distribution_class
    b = v.BoundingBox([0, 0, 0], [1, 1, 1])
    assert distribution_class(uniform(200_000, 0, 1, 1), b) == "uniform"
    assert distribution_class(blobs(200_000, 64, 0.01, 0.7, 2), b) == "clustered"
    assert distribution_class(uniform(10, 0, 1, 3), b) == "uniform"


def test_table_roundtrip_and_lookup(tmp_path):
    from vorothree_b200 import autotune as at
    entries = {at.key("clustered", 1 << 20): {"factor": 2.0}, at.key("uniform", 1 << 20): {"factor": 1.25},
               at.key("uniform", 1 << 10): {"factor": 0.8}}
    p = str(tmp_path / "t.json")
    at.record(entries, p, device="test")
    back = at.load_table(p)
    assert back == entries
    assert at.lookup("uniform", 1 << 20, back) == 1.25
    assert at.lookup("uniform", 1500, back) == 0.8          # nearest bucket
    assert at.lookup("clustered", 1 << 12, back) == 2.0
    assert at.lookup("clustered", 100, {}) == at.DEFAULT_FACTOR["clustered"]


def test_committed_table_is_well_formed():
    from vorothree_b200 import autotune as at
    for k, e in at.load_table().items():
        cls, b = k.split("/2^")
        assert cls in ("uniform", "clustered") and int(b) % 2 == 0
        assert e["factor"] in at.FACTORS


@pytest.mark.gpu
def test_tune_on_gpu(oracle_mod):
    import vorothree_b200 as v
    from vorothree_b200 import autotune as at
    b = v.BoundingBox([0, 0, 0], [1, 1, 1])
    pts = blobs(40_000, 8, 0.02, 0.7, 5)
    entries = at.tune(pts, b, factors=(0.8, 1.6, 3.2), reps=1, entries={})
    (k, e), = entries.items()
    assert k == at.key("clustered", len(pts)) and e["factor"] in (0.8, 1.6, 3.2)
    assert len(e["trials"]) == 3 and all(t["ms"] > 0 for t in e["trials"])
    # the chosen grid computes the oracle's cells on that grid
    g = at.choose_grid(pts, b, entries)
    t = v.Tessellation(b, v.Algorithm3DGrid(*g))
    t.set_generators(pts)
    t.calculate()
    o = oracle_mod.OracleTessellation([0, 0, 0], [1, 1, 1], *g)
    o.set_generators(pts)
    o.calculate()
    assert np.array_equal(t.summaries()[0], o.summaries()[0])
