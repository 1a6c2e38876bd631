"""The launch-shape autotuner's search and its record (host logic; the
device measurement is covered by the GPU tests)."""
import json
import os

import pytest

from lgbm_b200 import autotune

BASE = {"partition_ctas": 444, "hist_ctas": 264, "hist_rows_per_block": 512}


def test_candidates_around_the_built_in_shape():
    assert autotune.candidates(BASE, "partition_ctas") == [9, 18, 37, 74, 148, 296, 444]
    assert autotune.candidates(BASE, "hist_ctas") == [33, 66, 132, 264]
    assert autotune.candidates(BASE, "hist_rows_per_block") == [128, 256, 512, 1024, 2048]
    assert autotune.candidates(dict(BASE, hist_rows_per_block=100), "hist_rows_per_block") == [100, 128, 256, 512,
                                                                                                 1024, 2048]
    assert autotune.candidates({"partition_ctas": 3, "hist_ctas": 1, "hist_rows_per_block": 512},
                               "partition_ctas") == [1, 2, 3]
    with pytest.raises(ValueError):
        autotune.candidates(BASE, "tiles")


class FakeLearner:
    """Stands in for lgbm_b200.Learner: a known cost per shape, and the
    C side's rounding of hist_ctas to clusters of 8."""

    def __init__(self, cost):
        self.shape = dict(BASE)
        self.cost = cost
        self.calls = []

    @property
    def launch_shape(self):
        return dict(self.shape)

    @launch_shape.setter
    def launch_shape(self, s):
        self.shape = dict(s, hist_ctas=(s["hist_ctas"] + 7) // 8 * 8)

    def time_shapes(self, shapes, reps=3):
        self.calls.append([dict(s) for s in shapes])
        ms = [self.cost(s) for s in shapes]
        i = min(range(len(ms)), key=ms.__getitem__)
        self.launch_shape = shapes[i]
        return i, ms


def test_tune_is_a_coordinate_search():
    def cost(s):  # separable, minimum at (148, 132, 1024)
        return abs(s["partition_ctas"] - 148) + abs(s["hist_ctas"] - 132) / 10 + abs(s["hist_rows_per_block"] - 1024) / 100

    fl = FakeLearner(cost)
    best, best_ms, default_ms, trials = autotune.tune(fl)
    assert best == {"partition_ctas": 148, "hist_ctas": 132, "hist_rows_per_block": 1024}
    assert fl.shape == {"partition_ctas": 148, "hist_ctas": 136, "hist_rows_per_block": 1024}  # rounded
    assert default_ms == pytest.approx(cost(BASE)) and best_ms == pytest.approx(cost(best))
    assert len(fl.calls) == 4 and len(trials) == 7 + 4 + 5 + 2
    assert fl.calls[3] == [BASE, best]  # the winner confirmed against the start
    # each pass varies one knob from the best so far
    assert all(s["hist_ctas"] == 264 and s["hist_rows_per_block"] == 512 for s in fl.calls[0])
    assert all(s["partition_ctas"] == 148 and s["hist_rows_per_block"] == 512 for s in fl.calls[1])
    assert all(s["partition_ctas"] == 148 and s["hist_ctas"] == 132 for s in fl.calls[2])


def test_tune_keeps_the_start_when_the_winner_is_not_faster():
    seen = {}

    def cost(s):  # every other shape looks faster only the first time it is measured
        if s == BASE:
            return 6.0
        k = tuple(sorted(s.items()))
        seen[k] = seen.get(k, 0) + 1
        return 5.0 if seen[k] == 1 else 7.0

    fl = FakeLearner(cost)
    best, best_ms, default_ms, trials = autotune.tune(fl)
    assert best == BASE and fl.shape == BASE and best_ms == default_ms


def test_record_and_lookup(tmp_path):
    path = str(tmp_path / "shapes.json")
    assert autotune.lookup("c2/quantized", 148, path) is None
    trials = [dict(BASE, ms_per_tree=8.0), dict(BASE, partition_ctas=296, ms_per_tree=7.5)]
    best = dict(BASE, partition_ctas=296)
    autotune.record("c2/quantized", best, 7.5, BASE, 8.0, trials, "B200", 148, path)
    autotune.record("c3/quantized", BASE, 60.0, BASE, 60.0, [dict(BASE, ms_per_tree=60.0)], "B200", 148, path)
    assert autotune.lookup("c2/quantized", 148, path) == best
    assert autotune.lookup("c2/quantized", 132, path) is None  # another device
    e = json.load(open(path))["c2/quantized"]
    assert e["ms_per_tree"] == 7.5 and e["default_ms_per_tree"] == 8.0 and e["device"] == "B200"
    assert sorted(json.load(open(path))) == ["c2/quantized", "c3/quantized"]


def test_recorded_shapes_are_valid():
    """The committed record: every shape within the C ABI's ranges, and
    never slower than the built-in shape measured beside it."""
    if not os.path.exists(autotune.SHAPES_FILE):
        pytest.skip("no shapes recorded")
    data = autotune.load()
    for key, e in data.items():
        s = e["shape"]
        assert set(s) == set(autotune.KNOBS), key
        assert 1 <= s["partition_ctas"] <= 65535 and 1 <= s["hist_ctas"] <= 65535, key
        assert 32 <= s["hist_rows_per_block"] <= 1 << 24, key
        assert e["ms_per_tree"] <= e["default_ms_per_tree"], key
        assert any(all(t[k] == s[k] for k in autotune.KNOBS) for t in e["trials"]), key
