"""The serving loop (vite_b200.serve): requests that arrive while others run join the
running batch, finished ones are handed back and dropped, and every request's
result is the one it gets alone (vg_louvain_run)."""
import numpy as np
import pytest

from vite_b200 import serve as sv

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lanes", [(), (20000,)])
def test_served_results_equal_alone(ctx, lanes):
    gs = []
    for k in range(10):
        if k % 2:
            g = ctx.generate_ba(500 + 300 * k, 4, 100 + k)
        else:
            g = ctx.generate_rgg(800 + 900 * k, 0.0, 0)
            ctx.reweight(g, 1)
        gs.append(g)
    alone = [ctx.run(g, want_comm=True) for g in gs]
    # arrivals spread over a few rounds, so later requests join a running batch
    reqs = [sv.Request(g, arrival=0.002 * k, want_comm=True) for k, g in enumerate(gs)]
    rep = sv.serve(ctx, reqs, budget=1 << 30, lanes=lanes)
    assert [r.index for r in rep.results] == list(range(len(gs)))
    for r, a in zip(rep.results, alone):
        assert r.latency >= 0.0
        assert [(x["nv"], x["ne"], x["iters"], x["modularity"]) for x in r.levels] == \
               [(x["nv"], x["ne"], x["iters"], x["modularity"]) for x in a.stats]
        assert np.array_equal(r.comm, a.comm)
    assert sum(l["requests"] for l in rep.stats["lanes"]) == len(gs)
    assert len(rep.stats["lanes"]) == len(lanes) + 1
    seq = sv.sequential(ctx, reqs)
    for r, a in zip(seq.results, alone):
        assert [x["modularity"] for x in r.levels] == [x["modularity"] for x in a.stats]
    for g in gs:
        g.free()


def test_host_requests_uploaded_on_admission(ctx):
    """Requests held in host memory (Vite's CSR) are uploaded when admitted; with a
    budget that admits about two graphs at a time the others wait, and every result is
    still the one the graph gets alone."""
    import vite_b200

    start = ctx.bytes_in_use
    reqs, alone = [], []
    for k in range(8):
        g = ctx.generate_rgg(2000 + 700 * k, 0.0, 0) if k % 2 == 0 else \
            ctx.generate_ba(1500 + 400 * k, 4, 300 + k)
        ctx.reweight(g, 1)
        rp, tail, w = g.download()
        ed = np.empty(len(tail), vite_b200.EDGE_DTYPE)
        ed["tail"] = tail
        ed["weight"] = w
        alone.append(ctx.run(g, want_comm=True))
        g.free()
        reqs.append(sv.Request(None, arrival=0.001 * k, want_comm=True, rowptr=rp, edges=ed))
    budget = 2 * max(r.footprint() for r in reqs)
    rep = sv.serve(ctx, reqs, budget=budget)
    for r, a in zip(rep.results, alone):
        assert [(x["nv"], x["ne"], x["iters"], x["modularity"]) for x in r.levels] == \
               [(x["nv"], x["ne"], x["iters"], x["modularity"]) for x in a.stats]
        assert np.array_equal(r.comm, a.comm)
    seq = sv.sequential(ctx, reqs)
    for r, a in zip(seq.results, alone):
        assert [x["modularity"] for x in r.levels] == [x["modularity"] for x in a.stats]
    assert ctx.bytes_in_use == start  # every uploaded graph was released


def test_direct_lane_results_equal_alone(ctx):
    """Requests above `direct_above` entries run alone on the direct workers, the rest in
    batched lanes; every result is still the one the graph gets alone."""
    gs = [ctx.generate_rgg(1500 + 2500 * k, 0.0, 0) for k in range(6)]
    for g in gs:
        ctx.reweight(g, 1)
    alone = [ctx.run(g, want_comm=True) for g in gs]
    reqs = [sv.Request(g, arrival=0.001 * k, want_comm=True) for k, g in enumerate(gs)]
    cut = sorted(g.ne for g in gs)[2]
    rep = sv.serve(ctx, reqs, budget=1 << 30, lanes=(20000,), direct_above=cut, direct_workers=2)
    assert rep.stats["direct"]["requests"] == sum(g.ne > cut for g in gs)
    for r, a in zip(rep.results, alone):
        assert [(x["nv"], x["ne"], x["iters"], x["modularity"]) for x in r.levels] == \
               [(x["nv"], x["ne"], x["iters"], x["modularity"]) for x in a.stats]
        assert np.array_equal(r.comm, a.comm)
    for g in gs:
        g.free()
