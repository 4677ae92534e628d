"""The serving loop's host logic (vite_b200.serve) without a GPU: the device calls are
replaced by fakes that record what the loop asked for. Checked: every request is served
once and gets its own graph's result, size classes and the direct lane take the
requests they should, a lane never holds more than its memory budget, the FIFO model
of the plain path, and errors raised inside a lane reach the caller."""
import threading

import numpy as np
import pytest

from vite_b200 import serve as sv


class FakeGraph:
    def __init__(self, nv, ne):
        self.nv, self.ne = nv, ne
        self.freed = False

    def free(self):
        self.freed = True


class FakeLevels:
    def __init__(self, g):
        # a result that names its graph, so a mixed-up hand-back is visible
        self.stats = [{"nv": g.nv, "ne": g.ne, "iters": 1, "modularity": 0.25}]
        self.comm = None


class FakeContext:
    created = []
    lock = threading.Lock()

    def __init__(self, device=0):
        self.device = device
        self.closed = False
        self.runs = []
        with FakeContext.lock:
            FakeContext.created.append(self)

    def run(self, g, threshold=1e-6, want_comm=False):
        self.runs.append(g.ne)
        return FakeLevels(g)

    def upload_edges(self, rowptr, edges):
        return FakeGraph(len(rowptr) - 1, len(edges))

    def close(self):
        self.closed = True


class FakeBatch:
    """Each job finishes after 1 + (ne % 3) rounds; records the bytes in flight."""
    instances = []
    fail_on_step = False

    def __init__(self, ctx, budget=0):
        self.ctx, self.budget = ctx, budget
        self.jobs = {}      # id -> [graph, rounds left]
        self.done = []
        self.next_id = 0
        self.max_inflight = 0
        self.submitted = []
        FakeBatch.instances.append(self)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def submit(self, g, threshold=1e-6, want_comm=False, take=False):
        j = self.next_id
        self.next_id += 1
        self.jobs[j] = [g, 1 + g.ne % 3]
        self.submitted.append(g.ne)
        held = sum(sv.Request(x, 0.0).footprint() for x, _ in self.jobs.values())
        self.max_inflight = max(self.max_inflight, held)
        return j

    def step(self):
        if FakeBatch.fail_on_step:
            raise RuntimeError("step failed")
        for j, rec in list(self.jobs.items()):
            rec[1] -= 1
            if rec[1] == 0:
                self.done.append(j)
        return len([r for r in self.jobs.values() if r[1] > 0]), 0

    def poll(self):
        d, self.done = self.done, []
        return d

    def result(self, j, want_comm=False):
        return FakeLevels(self.jobs[j][0])

    def forget(self, j):
        del self.jobs[j]

    def stats(self):
        return {}


@pytest.fixture
def fakes(monkeypatch):
    FakeContext.created = []
    FakeBatch.instances = []
    FakeBatch.fail_on_step = False
    monkeypatch.setattr(sv, "Batch", FakeBatch)
    monkeypatch.setattr(sv, "Context", FakeContext)
    yield


def requests(sizes, spacing=0.0):
    return [sv.Request(FakeGraph(max(ne // 8, 1), ne), arrival=spacing * i)
            for i, ne in enumerate(sizes)]


SIZES = [50, 3000, 120, 9000, 700, 40000, 5, 2500, 60000, 999, 1000, 1001, 200000, 64]


@pytest.mark.parametrize("spacing", [0.0, 0.0005])
def test_each_request_served_once_with_its_own_result(fakes, spacing):
    reqs = requests(SIZES, spacing)
    ctx = FakeContext()
    rep = sv.serve(ctx, reqs, budget=1 << 40, lanes=(1000, 10000), direct_above=50000,
                   direct_workers=2)
    assert [r.index for r in rep.results] == list(range(len(reqs)))
    for r, q in zip(rep.results, reqs):
        assert r.levels[0]["ne"] == q.ne  # its own graph's result
        assert r.finish >= r.arrival and r.latency >= 0.0
    # classes: <= 1000, <= 10000, the rest up to 50000 batched; above 50000 direct
    lanes = rep.stats["lanes"]
    assert [l["requests"] for l in lanes] == [
        sum(1 for s in SIZES if s <= 1000),
        sum(1 for s in SIZES if 1000 < s <= 10000),
        sum(1 for s in SIZES if 10000 < s <= 50000)]
    assert rep.stats["direct"] == {"requests": 2, "workers": 2, "above_entries": 50000}
    # the direct requests ran alone (Context.run), every other one through a batch
    direct_runs = sorted(ne for c in FakeContext.created for ne in c.runs)
    assert direct_runs == [60000, 200000]
    batched = sorted(ne for b in FakeBatch.instances for ne in b.submitted)
    assert batched == sorted(s for s in SIZES if s <= 50000)
    # every context the loop made for itself is closed; the caller's is left open
    assert all(c.closed for c in FakeContext.created if c is not ctx)
    assert not ctx.closed


def test_lane_budget_holds(fakes):
    # ten requests of 10,000 entries: 400 kB + 250 kB + 1 MiB each in the batch's
    # estimate; a budget of three of them keeps at most three in flight
    reqs = requests([10000] * 10)
    one = reqs[0].footprint()
    rep = sv.serve(FakeContext(), reqs, budget=3 * one)
    assert len(rep.results) == 10
    (b,) = FakeBatch.instances
    assert 0 < b.max_inflight <= 3 * one
    assert rep.rounds >= 4  # ten jobs three at a time


def test_request_larger_than_budget_runs_alone(fakes):
    reqs = requests([10000, 10000])
    rep = sv.serve(FakeContext(), reqs, budget=reqs[0].footprint() // 2)
    assert len(rep.results) == 2
    assert FakeBatch.instances[0].max_inflight == reqs[0].footprint()


def test_lane_error_reaches_caller(fakes):
    FakeBatch.fail_on_step = True
    with pytest.raises(RuntimeError, match="step failed"):
        sv.serve(FakeContext(), requests([100, 200, 300]), lanes=(150,))


def test_fifo_finish_times():
    fin = sv.fifo([0.0, 0.1, 5.0], [1.0, 1.0, 1.0])
    assert list(fin) == [1.0, 2.0, 6.0]
    # out of arrival order: the queue follows arrivals, not list order
    fin = sv.fifo([2.0, 0.0], [1.0, 3.0])
    assert list(fin) == [4.0, 3.0]


def test_percentile():
    assert sv.percentile([1.0, 2.0, 3.0, 4.0], 50) == pytest.approx(2.5)
    assert sv.percentile(np.arange(101), 99) == pytest.approx(99.0)
