"""The measured-choice helper behind ``PolygonP2Plan.autotune`` (no GPU needed)."""

import json

import numpy as np
import pytest

from pymhm_b200 import autotune as at


def test_choose_picks_the_fastest_and_reports_every_timing():
    times = {(16, 1): 5.0, (32, 1): 3.0, (32, 4): 2.5, (64, 4): 4.0}
    best, info = at.choose(times, lambda c: times[c])
    assert best == (32, 4)
    assert not info["cached"]
    assert {tuple(json.loads(k)): v for k, v in info["timings_ms"].items()} == times


def test_cache_records_and_replays_the_choice(tmp_path):
    cache = tmp_path / "tune.json"
    key = at.shape_key("B200", np.arange(5), np.array([3, 4]))
    calls = []

    def measure(c):
        calls.append(c)
        return {(16, 1): 2.0, (32, 4): 1.0}[c]

    best, info = at.choose([(16, 1), (32, 4)], measure, key=key, cache=cache)
    assert best == (32, 4) and len(calls) == 2 and not info["cached"]
    best2, info2 = at.choose([(16, 1), (32, 4)], measure, key=key, cache=cache)
    assert best2 == (32, 4) and len(calls) == 2 and info2["cached"]
    # a recorded choice that is no longer a candidate is measured again
    best3, _ = at.choose([(16, 1)], measure, key=key, cache=cache)
    assert best3 == (16, 1) and len(calls) == 3
    # another shape signature does not hit
    other = at.shape_key("B200", np.arange(6), np.array([3, 4]))
    assert other != key


def test_failed_measurement_and_empty_candidates_raise():
    with pytest.raises(ValueError):
        at.choose([], lambda c: 1.0)
    with pytest.raises(RuntimeError):
        at.choose([(8, 1)], lambda c: float("nan"))
