"""The serving bound bench.py reports (host arithmetic only)."""
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
