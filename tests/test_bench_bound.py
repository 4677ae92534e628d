"""The serving bound bench.py reports (host arithmetic only)."""
import numpy as np
import pytest

import bench


def test_serving_bound_rule():
    # rates (visits / time): 3.33e10, 6e9, 1e10, 5e9; R = 3.33e10 and only request 0 is
    # within 20 % of it, so it keeps its 30 ms and the others cost visits / R
    t = [0.03, 0.05, 0.01, 0.002]
    v = [1e9, 0.3e9, 0.1e9, 0.01e9]
    b = bench.serving_bound(t, v, [4e7, 3e7, 1e6, 1e4])
    R = 1e9 / 0.03
    floor_ = 0.03 + (0.3e9 + 0.1e9 + 0.01e9) / R
    assert b["peak_rate_edge_visits_per_s"] == pytest.approx(R)
    assert b["saturating_requests"] == 1
    assert b["min_served_seconds"] == pytest.approx(floor_)
    assert b["max_speedup"] == pytest.approx(sum(t) / floor_)
    assert "by_family" not in b


def test_serving_bound_by_family():
    # family 1 peaks at 6e9 (request 1, which keeps its time); request 3 (5e9) is
    # within 20 % of that too, so the per-family floor is 0.03 + 0.1e9/R0 + 0.05 + 0.002
    t = [0.03, 0.05, 0.01, 0.002]
    v = [1e9, 0.3e9, 0.1e9, 0.01e9]
    b = bench.serving_bound(t, v, [4e7, 3e7, 1e6, 1e4], kinds=[0, 1, 0, 1])
    f = b["by_family"]
    R0 = 1e9 / 0.03
    assert f["peak_rate_edge_visits_per_s"] == {"rgg": pytest.approx(R0),
                                               "ba": pytest.approx(6e9)}
    assert f["saturating_requests"] == 3
    assert f["min_served_seconds"] == pytest.approx(0.03 + 0.1e9 / R0 + 0.05 + 0.002)
    # a per-family floor is never below the family-blind one
    assert f["min_served_seconds"] >= b["min_served_seconds"]
    assert f["max_speedup"] == pytest.approx(sum(t) / f["min_served_seconds"])
    assert np.isfinite(f["max_speedup"])
