"""bench.py host logic: the serving bound, the Vite file it writes for the reference, the
level-parity verdicts and the request-size inversion (no GPU)."""
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


def test_write_vite_file_round_trip(tmp_path):
    import vite_b200
    from oracle import vite_oracle as vo

    rp = np.array([0, 2, 3, 3, 5], np.int64)
    ed = np.zeros(5, vite_b200.EDGE_DTYPE)
    ed["tail"] = [1, 3, 0, 0, 2]
    ed["weight"] = [0.5, 1.25, 0.5, 1.25, 3.0]
    path = str(tmp_path / "g.bin")
    bench.write_vite_file(path, rp, ed)
    g = vo.read_vite_binary(path)
    assert g.nv == 4 and g.ne == 5
    np.testing.assert_array_equal(g.rowptr, rp)
    np.testing.assert_array_equal(g.tail, ed["tail"])
    np.testing.assert_array_equal(g.weight, ed["weight"])
    # the header and the records are exactly Vite's layout: 16 + 8 (nv + 1) + 16 ne bytes
    assert (tmp_path / "g.bin").stat().st_size == 16 + 8 * 5 + 16 * 5


def _ref_levels(mods, iters=(3, 2), nvs=(6, 2)):
    from oracle import vite_oracle as vo

    out = []
    for k, (m, it, nv) in enumerate(zip(mods, iters, nvs)):
        cv = np.arange(nv, dtype=np.int64) // 3 * 3
        out.append(vo.RefLevel(level=k, nv=nv, ne=2 * nv, iters=it, mod=m, num_colors=0,
                               seconds=0.0, cvect=cv))
    return out


def test_level_parity_verdicts():
    ref = _ref_levels([0.25, 0.5])
    ours = [{"nv": 6, "ne": 12, "iters": 3, "modularity": 0.25},
            {"nv": 2, "ne": 4, "iters": 2, "modularity": 0.5}]
    p = bench.level_parity(ours, ref, None, None, exact=True)
    assert p["pass"] and p["every_modularity_bit_identical"]
    assert p["same_levels_entries_iterations"] and p["levels"] == [2, 2]
    # one ulp off: fails the unit-weight bar, passes the real-weight one
    ours[1]["modularity"] = np.nextafter(0.5, 1.0)
    assert not bench.level_parity(ours, ref, None, None, exact=True)["pass"]
    assert bench.level_parity(ours, ref, None, None, exact=False)["pass"]
    # another iteration count fails both
    ours[1]["iters"] = 3
    assert not bench.level_parity(ours, ref, None, None, exact=False)["pass"]


def test_levels_agree():
    a = [{"nv": 10, "ne": 40, "modularity": 0.5}, {"nv": 3, "ne": 9, "modularity": 0.6}]
    b = [dict(x) for x in a]
    assert bench.levels_agree(a, b)
    b[1]["modularity"] = 0.6 * (1 + 2 * bench.REL_TOL)
    assert not bench.levels_agree(a, b)
    assert not bench.levels_agree(a, a[:1])
    b = [dict(x) for x in a]
    b[0]["ne"] = 41
    assert not bench.levels_agree(a, b)


@pytest.mark.parametrize("e", [1e3, 1e5, 3e7])
def test_rgg_vertices_for_entries(e):
    n = bench.rgg_vertices_for_entries(e)
    r = (np.sqrt(np.log(n) / (3.14159 * n)) + np.sqrt(2.0736 / n)) / 2.0
    assert n * 3.14159 * r * r * n == pytest.approx(e, rel=1e-3)
