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
        if k == at.HANDOFF_KEY:
            assert set(e["tuning"]) == set(at.DEFAULT_HANDOFF)
            continue
        cls, b = k.split("/2^")
        assert cls in ("uniform", "clustered") and int(b) % 2 == 0
        assert e["factor"] in at.FACTORS
        t = e.get("tuning", at.DEFAULT_TUNING)
        assert t["fast_layout"] in at.LAYOUTS and t["fast_blocks_per_sm"] in at.BLOCKS_PER_SM


def test_lookup_tuning_defaults_and_overrides():
    from vorothree_b200 import autotune as at
    d = at.lookup_tuning("uniform", 1 << 20, {})
    assert d == dict(at.DEFAULT_TUNING, **at.DEFAULT_HANDOFF)
    entries = {at.key("uniform", 1 << 20): {"factor": 1.6, "tuning": {"fast_layout": "full", "fast_blocks_per_sm": 6}},
               at.key("clustered", 1 << 20): {"factor": 2.5, "tuning": {"fast_layout": "slots",
                                                                         "fast_blocks_per_sm": 5}},
               at.HANDOFF_KEY: {"tuning": {"huge_direct_max": 16, "huge_blocks_max": 64, "huge_narrow_max": 5000}}}
    u = at.lookup_tuning("uniform", 1 << 19, entries)
    assert u["fast_layout"] == "full" and u["huge_direct_max"] == 16 and u["huge_narrow_max"] == 5000
    c = at.lookup_tuning("clustered", 1 << 21, entries)
    assert c["fast_blocks_per_sm"] == 5 and c["fast_layout"] == "slots"


@pytest.mark.gpu
def test_tune_on_gpu(oracle_mod):
    import vorothree_b200 as v
    from vorothree_b200 import autotune as at
    b = v.BoundingBox([0, 0, 0], [1, 1, 1])
    pts = blobs(40_000, 8, 0.02, 0.7, 5)
    entries = at.tune(pts, b, factors=(0.8, 1.6, 3.2), reps=1, entries={}, layouts=("slots", "full"),
                      blocks=(6, 7))
    (k, e), = entries.items()
    assert k == at.key("clustered", len(pts)) and e["factor"] in (0.8, 1.6, 3.2)
    # three densities, then slots at 7 blocks per SM and the full layout
    assert len(e["trials"]) == 5 and all(t["ms"] > 0 for t in e["trials"])
    assert e["tuning"]["fast_layout"] in ("slots", "full")
    # the chosen grid computes the oracle's cells on that grid
    g = at.choose_grid(pts, b, entries)
    t = v.Tessellation(b, v.Algorithm3DGrid(*g))
    t.set_generators(pts)
    t.calculate()
    o = oracle_mod.OracleTessellation([0, 0, 0], [1, 1, 1], *g)
    o.set_generators(pts)
    o.calculate()
    assert np.array_equal(t.summaries()[0], o.summaries()[0])


@pytest.mark.gpu
def test_every_tuning_choice_gives_the_oracles_cells(oracle_mod):
    """Each setting the tuner can choose -- first-tier layout, blocks per SM,
    the block tier's hand-off thresholds and width -- computes the same cells,
    bit for bit, as the oracle; on a clustered input and on the sphere-surface
    distribution (whose centre cell takes the block tier)."""
    import itertools
    import vorothree_b200 as v
    from vorothree_b200.workloads import bench_distribution
    cases = [([0, 0, 0], [1, 1, 1], (14, 14, 14), np.clip(blobs(8000, 5, 0.03, 0.7, 61), 0, 1)),
             ([0, 0, 0], [100, 100, 100], (10, 10, 10), bench_distribution("sphere", 1000, 62))]
    for bmin, bmax, grid, pts in cases:
        o = oracle_mod.OracleTessellation(bmin, bmax, *grid)
        o.set_generators(pts)
        o.calculate()
        ov, oc, on = o.summaries()
        oids = o.neighbors()[1]
        choices = [dict(fast_layout=l, fast_blocks_per_sm=nb) for l, nb in
                   (("slots", 5), ("slots", 6), ("slots", 7), ("full", 6))]
        handoffs = [dict(huge_direct_max=dm, huge_narrow_max=nm, huge_blocks_max=hb)
                    for dm, nm, hb in itertools.product((1, 256), (500, 5000), (2, 64))]
        for tun in choices + [dict(choices[1], **h) for h in handoffs]:
            t = v.Tessellation(v.BoundingBox(bmin, bmax), v.Algorithm3DGrid(*grid))
            t.set_tuning(tun)
            got = t.get_tuning()
            assert all(got[k] == tun[k] for k in tun)
            t.set_generators(pts)
            t.calculate()
            gv, gc, gn = t.summaries()
            assert np.array_equal(gn, on) and np.array_equal(gv, ov) and np.array_equal(gc, oc), tun
            assert np.array_equal(t.neighbors()[1], oids), tun
            t.close()

def test_hollow_inputs_get_batched_plane_tests():
    """A dense central box or generators on a sphere leave most of the box
    empty: the per-input settings turn the walk's batched plane tests on for
    them and leave them off for uniform, plane-crowded and blob inputs."""
    from vorothree_b200 import autotune as at
    from vorothree_b200.tessellation import BoundingBox
    from vorothree_b200.workloads import bench_distribution
    box = BoundingBox([0, 0, 0], [100, 100, 100])
    for kind, want in (("central", True), ("sphere", True), ("uniform", False), ("axes", False)):
        pts = bench_distribution(kind, 5000, 3)
        assert at.hollow(pts, box) == want, kind
        assert at.input_tuning(pts, box, {})["noop_run"] == (at.NOOP_RUN_HOLLOW if want else -1), kind
    unit = BoundingBox([0, 0, 0], [1, 1, 1])
    assert not at.hollow(at.synthetic("clustered", 1 << 14, 1), unit)
    assert at.choose(bench_distribution("central", 2000, 4), box, {})[1]["noop_run"] == at.NOOP_RUN_HOLLOW
