"""Batched and served runs (vg_batch_*): every graph of a batch gets what a run of
its own (vg_louvain_run) gives it. Unit weights: identical levels, modularity bits
and communities. Real weights: the same levels with per-level modularity within
1e-9 relative (FP64 atomics make even two plain runs differ in the last bits)."""
import ctypes as C

import numpy as np
import pytest

import vite_b200 as vb

pytestmark = pytest.mark.gpu

REL = 1e-9


def unit(ctx, g):
    ctx.reweight(g, 1)
    return g


def plain(ctx, g, **kw):
    return ctx.run(g, want_comm=True, **kw)


def assert_same(a, b, exact):
    assert len(a.stats) == len(b.stats)
    for x, y in zip(a.stats, b.stats):
        assert (x["nv"], x["ne"]) == (y["nv"], y["ne"])
        if exact:
            assert x["iters"] == y["iters"]
            assert x["modularity"] == y["modularity"]
        else:
            assert abs(x["modularity"] - y["modularity"]) <= REL * abs(y["modularity"])
    if exact:
        assert np.array_equal(a.comm, b.comm)


def mixed_unit(ctx):
    return [unit(ctx, ctx.generate_rgg(1000, 0.0, 0)),
            ctx.generate_er(5000, 16.0, 3),
            unit(ctx, ctx.generate_rgg(20000, 1.0, 5)),
            ctx.generate_ba(4000, 4, 7),
            unit(ctx, ctx.generate_rgg(3000, 0.0, 0)),
            ctx.generate_er(1200, 16.0, 11)]


def test_batch_unit_weights_identical_to_plain(ctx):
    gs = mixed_unit(ctx)
    ref = [plain(ctx, g) for g in gs]
    out = ctx.run_batch(gs, want_comm=True)
    for a, b in zip(out, ref):
        assert_same(a, b, exact=True)
    for g in gs:
        g.free()


def test_batch_real_weights_match_plain(ctx):
    gs = [ctx.generate_rgg(2000, 0.0, 0), ctx.generate_rgg(50000, 1.0, 9),
          ctx.generate_er(10000, 16.0, 4)]
    ctx.reweight(gs[2], 2, 77)
    ref = [plain(ctx, g) for g in gs]
    out = ctx.run_batch(gs, want_comm=True)
    for a, b in zip(out, ref):
        assert_same(a, b, exact=False)
        # the final partition: same community count
        assert len(np.unique(a.comm)) == len(np.unique(b.comm))
    for g in gs:
        g.free()


def test_batch_with_hub_graph(ctx):
    """A graph whose hubs take the multi-CTA hub class, batched with small graphs
    (unit weights: identical to its own run)."""
    from conftest import multi_hub_csr
    rp, tl, w = multi_hub_csr(40000, 6, 6000, 23, False)
    hub = ctx.upload(rp, tl, w)
    gs = [ctx.generate_er(3000, 16.0, 5), hub, unit(ctx, ctx.generate_rgg(5000, 0.0, 0))]
    ref = [plain(ctx, g) for g in gs]
    out = ctx.run_batch(gs, want_comm=True)
    for a, b in zip(out, ref):
        assert_same(a, b, exact=True)
    for g in gs:
        g.free()


def test_batch_with_locality_layout_graph(ctx):
    # n >= 2^18 takes the BFS locality layout in the plain path and in the batch
    big = unit(ctx, ctx.generate_rgg(1 << 18, 1.0, 13))
    small = ctx.generate_er(3000, 16.0, 5)
    ref = [plain(ctx, big), plain(ctx, small)]
    out = ctx.run_batch([small, big], want_comm=True)
    assert_same(out[0], ref[1], exact=True)
    assert_same(out[1], ref[0], exact=True)
    big.free()
    small.free()


def test_batch_budget_admission_and_continuous_joins(ctx):
    gs = mixed_unit(ctx)
    ref = [plain(ctx, g) for g in gs]
    est = [40 * g.ne + 200 * g.nv + (1 << 20) for g in gs]
    budget = sorted(est)[-1] + sorted(est)[-2]
    with ctx.batch(budget) as b:
        ids = {}
        # three graphs now, the rest while the first ones are running
        for k in range(3):
            ids[b.submit(gs[k], want_comm=True)] = k
        finished = []
        steps = 0
        while True:
            if steps == 2:
                for k in range(3, len(gs)):
                    ids[b.submit(gs[k], want_comm=True)] = k
            r, q = b.step()
            steps += 1
            st = b.stats()
            assert st["running_bytes"] <= budget
            finished += b.poll()
            if r == 0 and q == 0 and steps > 2:
                break
            assert steps < 500
        assert sorted(finished) == sorted(ids)
        for j, k in ids.items():
            assert_same(b.result(j, want_comm=True), ref[k], exact=True)
        st = b.stats()
        assert st["completed"] == len(gs) and st["admitted"] == len(gs)
    for g in gs:
        g.free()


def test_batch_one_phase_and_take(ctx):
    g1 = unit(ctx, ctx.generate_rgg(5000, 0.0, 0))
    g2 = ctx.generate_er(4000, 16.0, 2)
    ref1 = plain(ctx, g1, one_phase=True)
    ref2 = plain(ctx, g2)
    with ctx.batch() as b:
        j1 = b.submit(g1, one_phase=True, want_comm=True, take=True)
        j2 = b.submit(g2, want_comm=True)
        assert g1.handle is None  # handed over
        b.run_all()
        assert_same(b.result(j1, want_comm=True), ref1, exact=True)
        assert_same(b.result(j2, want_comm=True), ref2, exact=True)
        assert len(b.result(j1).stats) == 1
    g2.free()


def test_batch_same_graph_many_times(ctx):
    g = unit(ctx, ctx.generate_rgg(8000, 0.0, 0))
    ref = plain(ctx, g)
    out = ctx.run_batch([g] * 5, want_comm=True)
    for a in out:
        assert_same(a, ref, exact=True)
    g.free()


def test_batch_rejects_what_it_does_not_run(ctx):
    g = ctx.generate_er(1000, 16.0, 1)
    with ctx.batch() as b:
        jid = C.c_int64()
        for p in (vb.RunParams(1e-6, 1, 0, 8, 0, 0, 1.0, 0, 0, 2),   # coloring
                  vb.RunParams(1e-6, 0, 0, 8, 0, 2, 0.25, 0, 0, 2),  # early termination
                  vb.RunParams(1e-6, 0, 0, 8, 0, 0, 1.0, 1, 0, 2),   # threshold cycling
                  vb.RunParams(0.0, 0, 0, 8, 0, 0, 1.0, 0, 0, 2)):   # no threshold
            st = vb.lib().vg_batch_submit(b.handle, g.handle, C.byref(p), 0, C.byref(jid))
            assert st == vb.VG_ERR_ARG
        j = b.submit(g)
        with pytest.raises(vb.VgError, match="not finished"):
            b.result(j)
        b.run_all()
        assert b.result(j).stats
        with pytest.raises(vb.VgError, match="without VG_BATCH_COMM"):
            b.result(j, want_comm=True)
        b.forget(j)
        with pytest.raises(vb.VgError, match="unknown batch job"):
            b.result(j)
    empty = ctx.upload(np.zeros(4, np.int64), np.zeros(0, np.int64), np.zeros(0))
    with ctx.batch() as b:
        with pytest.raises(vb.VgError, match="needs vertices and edges"):
            b.submit(empty)
    with ctx.batch(1 << 20) as b:
        with pytest.raises(vb.VgError, match="more than the batch budget"):
            b.submit(g)
    g.free()
    empty.free()


def test_batch_captured_and_direct_iterations_agree(ctx):
    # without profiling the batch replays captured CUDA graphs of one iteration;
    # with it, every launch is issued directly: both give the same results
    gs = mixed_unit(ctx)[:4]
    graph_path = ctx.run_batch(gs, want_comm=True)
    ctx.profile(True, reset=True)
    try:
        direct = ctx.run_batch(gs, want_comm=True)
    finally:
        ctx.profile(False, reset=True)
    for a, b in zip(graph_path, direct):
        assert_same(a, b, exact=True)
    for g in gs:
        g.free()
