"""Sweep launch tuning (vg_ctx_set_tuning) and the autotuner (vg_autotune): the
tuning moves vertices between degree-class kernels, which changes no result with
unit weights (bit-identical levels, modularity and communities) and with real
weights keeps every level's modularity within 1e-9 relative."""
import numpy as np
import pytest

import vite_b200 as vb

pytestmark = pytest.mark.gpu

REL = 1e-9
OTHER = {"t32": 0, "ws_max": 48, "wt_max": 200, "ct_max": 1024, "tile_grid": 8}


def fresh():
    return vb.Context(0)


def levels_equal(a, b, exact):
    assert [s["nv"] for s in a.stats] == [s["nv"] for s in b.stats]
    assert [s["ne"] for s in a.stats] == [s["ne"] for s in b.stats]
    if exact:
        assert [s["iters"] for s in a.stats] == [s["iters"] for s in b.stats]
        assert [float(s["modularity"]).hex() for s in a.stats] == \
               [float(s["modularity"]).hex() for s in b.stats]
        assert np.array_equal(a.comm, b.comm)
    else:
        for x, y in zip(a.stats, b.stats):
            assert abs(x["modularity"] - y["modularity"]) <= REL * abs(y["modularity"])


def unit_graphs(ctx):
    from conftest import multi_hub_csr
    rgg = ctx.generate_rgg(30000, 1.0, 3)
    ctx.reweight(rgg, 1)
    rp, tl, w = multi_hub_csr(20000, 3, 5000, 31, False)
    return [rgg, ctx.generate_ba(40000, 12, 5), ctx.upload(rp, tl, w)]


def test_tuning_get_set_and_ranges():
    ctx = fresh()
    d = ctx.tuning
    assert d["t32"] in (0, 1) and 32 <= d["ws_max"] <= d["wt_max"] <= d["ct_max"] <= 4096
    for bad in ({"ws_max": 16}, {"ws_max": 200}, {"wt_max": 600}, {"ct_max": 5000},
                {"t32": 2}, {"tile_grid": 0}, {"ws_max": 128, "wt_max": 100}):
        with pytest.raises(vb.VgError):
            ctx.tuning = bad
        assert ctx.tuning == d  # a rejected setting changes nothing
    ctx.tuning = OTHER
    assert ctx.tuning == OTHER
    ctx.close()


def test_other_tuning_same_results_unit_weights():
    ctx = fresh()
    gs = unit_graphs(ctx)
    ref = [ctx.run(g, want_comm=True) for g in gs]
    ctx.tuning = OTHER
    out = [ctx.run(g, want_comm=True) for g in gs]
    for a, b in zip(out, ref):
        levels_equal(a, b, exact=True)
    ctx.close()


def test_other_tuning_real_weights_within_tolerance():
    ctx = fresh()
    g = ctx.generate_ba(40000, 12, 6)
    ctx.reweight(g, 2, 99)
    ref = ctx.run(g, want_comm=True)
    ctx.tuning = OTHER
    out = ctx.run(g, want_comm=True)
    levels_equal(out, ref, exact=False)
    ctx.close()


def test_autotune_sets_a_valid_tuning_and_keeps_results():
    ctx = fresh()
    gs = unit_graphs(ctx)
    ref = [ctx.run(g, want_comm=True) for g in gs]
    r = ctx.autotune(gs, sweeps=2)
    t = r["tuning"]
    assert t == ctx.tuning
    assert 32 <= t["ws_max"] <= t["wt_max"] <= t["ct_max"] <= 4096
    assert r["start_sweep_ms"] > 0 and r["sweep_ms"] <= r["start_sweep_ms"]
    # the graphs are as they were, and the tuned runs give the same results
    out = [ctx.run(g, want_comm=True) for g in gs]
    for a, b in zip(out, ref):
        levels_equal(a, b, exact=True)
    ctx.close()


def test_batch_under_other_tuning_matches_plain():
    ctx = fresh()
    ctx.tuning = OTHER
    gs = unit_graphs(ctx)
    ref = [ctx.run(g, want_comm=True) for g in gs]
    out = ctx.run_batch(gs, want_comm=True)
    for a, b in zip(out, ref):
        levels_equal(a, b, exact=True)
    ctx.close()
