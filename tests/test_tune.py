"""The autotuner's host side (no GPU): the coordinate search finds the
fastest setting of a synthetic cost model and measures each setting once;
a stored setting round-trips per device and the environment overrides it."""

from __future__ import annotations

import json

from gpjson_b200 import tune


def test_search_finds_the_minimum_of_a_separable_cost():
    best_of = {"index_ctas_per_sm": 3, "query_ctas_per_sm": 2, "long_line_bytes": 262144, "chunk_tiles": 2048}
    calls = []

    def cost(setting):
        calls.append(json.dumps(setting, sort_keys=True))
        return sum(0 if setting[k] == v else 1 + abs(hash((k, setting[k]))) % 7 for k, v in best_of.items())

    best, seen = tune.search(cost)
    assert best == best_of
    assert len(calls) == len(set(calls)) == len(seen)  # every setting timed once
    assert seen[json.dumps(best, sort_keys=True)] == 0


def test_search_keeps_the_start_when_nothing_is_faster():
    best, seen = tune.search(lambda s: 1.0 + 0.0 * len(s))
    assert best == {k: 0 for k in tune.KNOBS}
    assert len(seen) == 1 + sum(len(v) - 1 for v in tune.CANDIDATES.values())


def test_store_round_trip_and_environment_override(tmp_path, monkeypatch):
    monkeypatch.setenv("GPJSON_TUNING_DIR", str(tmp_path))
    for var in tune.ENV.values():
        monkeypatch.delenv(var, raising=False)
    key = tune.device_key("NVIDIA B200", 148)
    assert key == "NVIDIA_B200_148sm"
    assert tune.load(key) == {}
    p = tune.save(key, {"index_ctas_per_sm": 3, "query_ctas_per_sm": 0, "long_line_bytes": -1}, {"x": 1.0}, "tweets")
    assert p.parent == tmp_path and json.loads(p.read_text())["workload"] == "tweets"
    assert tune.load(key) == {"index_ctas_per_sm": 3, "query_ctas_per_sm": 0, "long_line_bytes": -1}
    monkeypatch.setenv("GPJSON_LONG_LINE_BYTES", "4096")
    assert tune.load(key)["long_line_bytes"] == 4096
    assert tune.load(tune.device_key("other", 1)) == {"long_line_bytes": 4096}
