"""The autotuner: table installation and per-bucket knob resolution (host
only), and on the GPU a tuning pass that must leave the tet set unchanged."""
import json
import os

import pytest

import fixtures as fx


@pytest.fixture()
def at(wt):
    from wtet_b200 import autotune

    saved = autotune.installed()
    yield autotune
    autotune.install(saved)


def test_resolution_by_bucket_and_kind(at):
    at.install([
        {"max_points": 1000, "batched": 0, "block_size": 128, "rounds_per_graph": 4, "overlap_shift": 2,
         "candidate_filter": 2, "pool_factor": 12},
        {"max_points": 2**64 - 1, "batched": 0, "rounds_per_graph": 16},
        {"max_points": 2**64 - 1, "batched": 1, "overlap_shift": 5},
    ])
    small = at.resolve(500)
    assert small == {"overlap_shift": 2, "rounds_per_graph": 4, "block_size": 128, "candidate_filter": 2,
                     "pool_factor": 12}
    big = at.resolve(10**6)
    assert big["rounds_per_graph"] == 16 and big["block_size"] == 256 and big["overlap_shift"] == 3
    batch = at.resolve(10**6, num_clouds=8)
    assert batch["overlap_shift"] == 5 and batch["rounds_per_graph"] == 8
    # a knob set by the caller wins over the table
    from wtet_b200 import Config

    assert at.resolve(500, config=Config(block_size=512))["block_size"] == 512
    # order of installation does not matter: buckets are sorted
    t = at.installed()
    assert [e["max_points"] for e in t if e["batched"] == 0] == [1000, 2**64 - 1]


def test_defaults_without_table(at):
    at.install([])
    assert at.resolve(123456) == at.DEFAULTS


def test_rejects_out_of_range_knobs(at):
    with pytest.raises(ValueError):
        at.install([{"max_points": 10, "batched": 0, "block_size": 96}])
    with pytest.raises(ValueError):
        at.install([{"max_points": 10, "batched": 2}])


def test_packaged_table_is_well_formed(wt):
    from wtet_b200 import autotune

    assert os.path.exists(autotune.DEFAULT_TABLE)
    with open(autotune.DEFAULT_TABLE) as f:
        table = json.load(f)["table"]
    kinds = {e["batched"] for e in table}
    assert kinds == {0, 1}
    for e in table:
        for k in autotune.KNOBS:
            assert e[k] in autotune.CHOICES[k], (k, e[k])


@pytest.mark.gpu
def test_tuning_keeps_the_triangulation(gpu, at):
    clouds = [fx.mixture(20_000, 5)]
    r = at.tune_bucket(clouds, repeats=1, verbose=False)   # raises if any knob changes the tet set
    for k in at.KNOBS:
        assert r[k] in at.CHOICES[k]
    assert r["device_ms"] > 0
