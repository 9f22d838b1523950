"""CPU tests of the autotuner's search and persistence (no GPU: the cost
function is a stand-in with a known minimum)."""

import json

from sparkalog_b200 import autotune

START = {"dir_rows_log2": 6, "group_lanes": 8, "group_candidates": 1 << 17, "sparse_candidates": 1 << 26,
         "fused_rows_cap": 672, "level_ratio": 4, "levels": 3, "merge_items": 11, "bloom_bits": 0,
         "merge_anti_ratio": 0, "sparse_items": 3, "compact_index": 1}


def bowl(target):
    """A separable cost with its minimum at `target` (index distance per field)."""
    def measure(t):
        return sum(abs(autotune.SPACE[k].index(t[k]) - autotune.SPACE[k].index(target[k])) for k in target) + 1.0
    return measure


def test_descent_finds_the_minimum_of_a_separable_cost():
    target = {"dir_rows_log2": 2, "group_lanes": 4, "group_candidates": 1 << 19, "sparse_candidates": 1 << 24,
              "fused_rows_cap": 512, "level_ratio": 8, "levels": 4, "merge_items": 15, "bloom_bits": 12,
              "merge_anti_ratio": 4, "sparse_items": 2, "compact_index": 0}
    best, cost, trials = autotune.coordinate_descent(bowl(target), START)
    assert best == target
    assert cost == 1.0
    # No configuration is measured twice, and the start is measured first.
    keys = [tuple(sorted(t.items())) for t, _ in trials]
    assert len(keys) == len(set(keys))
    assert trials[0][0] == START


def test_descent_skips_invalid_combinations():
    seen = []

    def measure(t):
        seen.append(t)
        return 1.0 if t["group_candidates"] > t["sparse_candidates"] else 2.0

    autotune.coordinate_descent(measure, START)
    assert all(autotune.valid(t) for t in seen)


def test_descent_keeps_the_start_on_ties():
    best, cost, _ = autotune.coordinate_descent(lambda t: 5.0, START)
    assert best == START and cost == 5.0


def test_saved_tuning_reads_the_named_file(tmp_path, monkeypatch):
    path = tmp_path / "t.json"
    autotune.save({"dir_rows_log2": 3}, path, {"device": "test"})
    monkeypatch.setenv("SPARKALOG_TUNING", str(path))
    assert autotune.saved_tuning() == {"dir_rows_log2": 3}
    assert json.loads(path.read_text())["device"] == "test"
    path.write_text("not json")
    assert autotune.saved_tuning() is None


def test_library_defaults_are_inside_the_search_space():
    d = autotune.defaults()
    assert set(autotune.SPACE) <= set(d)
    assert autotune.valid(d)


def test_shipped_tunings_are_points_of_the_search_space():
    from sparkalog_b200 import _native

    fields = {name for name, _ in _native.TuningC._fields_}
    shipped = sorted(autotune.SHIPPED_DIR.glob("*.json"))
    assert shipped
    for path in shipped:
        t = json.loads(path.read_text())["tuning"]
        assert set(t) <= fields, path.name
        merged = {**autotune.defaults(), **t}
        assert autotune.valid(merged), path.name
        for name, values in autotune.SPACE.items():
            assert merged[name] in values, (path.name, name, merged[name])
