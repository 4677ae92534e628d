"""Served Louvain: a request loop over one running batch (continuous batching).

Requests arrive over time, each a graph in host memory (Vite's CSR: row offsets and
Edge records, pinned memory copies fastest) or already on the device, with its run
parameters. Whenever the device is free between rounds, the requests that have
arrived are admitted in arrival order while their estimated device footprint fits
the memory budget (a request larger than the whole budget runs alone); an admitted
host request is uploaded then, so its copy is part of its latency. The batch runs
one round (one phase for every graph in it, then the rebuild), and the graphs whose
level loop ended are handed back with their latency (finish time - arrival time),
releasing their share of the budget. Work of requests that arrive while others run
overlaps on the device in the same launches, and each result is the one a run of its
own gives.

``sequential`` is the plain path the batch is measured against: per request in
arrival order, the upload (for host requests) and one vg_louvain_run, a single FIFO
server.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import Batch, Context, Graph


@dataclass
class Request:
    graph: Graph | None         # a device graph, or None for a host request
    arrival: float              # seconds after the start of the stream
    threshold: float = 1e-6
    want_comm: bool = False
    rowptr: np.ndarray | None = None   # host request: int64 row offsets (nv + 1)
    edges: np.ndarray | None = None    # host request: Vite Edge records (EDGE_DTYPE)

    @property
    def nv(self) -> int:
        return self.graph.nv if self.graph is not None else len(self.rowptr) - 1

    @property
    def ne(self) -> int:
        return self.graph.ne if self.graph is not None else len(self.edges)

    def footprint(self) -> int:
        """The batch's own estimate of a graph's device memory: 40 bytes per CSR entry,
        200 per vertex and 1 MiB."""
        return 40 * self.ne + 200 * self.nv + (1 << 20)

    def device_graph(self, ctx: Context) -> tuple[Graph, bool]:
        """(the graph on the device, whether it was uploaded here and so is owned)."""
        if self.graph is not None:
            return self.graph, False
        return ctx.upload_edges(self.rowptr, self.edges), True


@dataclass
class Served:
    index: int
    arrival: float
    finish: float
    levels: list
    comm: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.finish - self.arrival


@dataclass
class ServeReport:
    results: list
    seconds: float              # first arrival to last finish
    rounds: int
    stats: dict = field(default_factory=dict)

    def latencies(self) -> np.ndarray:
        return np.array([r.latency for r in self.results])


def _lane_loop(ctx: Context, requests: list[Request], mine: list[int], budget: int, t0: float,
               clock, out: dict, info: dict) -> None:
    """One batch fed with the requests `mine` (sorted by arrival) in real time."""
    jobs: dict[int, int] = {}
    held: dict[int, int] = {}  # job -> its footprint while admitted
    inflight = 0
    rounds = 0
    with Batch(ctx, budget) as b:
        nxt = 0
        busy = False
        done = 0
        while done < len(mine):
            now = clock() - t0
            # admission: arrived requests in arrival order while their footprint fits
            # the budget; with nothing admitted the next one runs whatever its size
            while nxt < len(mine) and requests[mine[nxt]].arrival <= now:
                i = mine[nxt]
                r = requests[i]
                need = r.footprint()
                if budget and inflight > 0 and inflight + need > budget:
                    break
                g, owned = r.device_graph(ctx)
                j = b.submit(g, threshold=r.threshold, want_comm=r.want_comm, take=owned)
                jobs[j] = i
                held[j] = need
                inflight += need
                nxt += 1
                busy = True
            if not busy:
                if nxt >= len(mine):
                    raise RuntimeError("serve: requests outstanding with nothing queued or running")
                # nothing queued or running: wait for the next arrival
                time.sleep(max(0.0, requests[mine[nxt]].arrival - now))
                continue
            running, queued = b.step()
            rounds += 1
            t = clock() - t0
            for j in b.poll():
                i = jobs.pop(j)
                inflight -= held.pop(j)
                res = b.result(j, want_comm=requests[i].want_comm)
                out[i] = Served(i, requests[i].arrival, t, res.stats, res.comm)
                b.forget(j)
                done += 1
            busy = running > 0 or queued > 0
        info["rounds"] = rounds
        info["stats"] = b.stats()


def _direct_loop(ctx: Context, requests: list[Request], queue: list[int], lock, t0: float,
                 clock, out: dict, info: dict) -> None:
    """One worker of the direct lane: takes the earliest arrived request left in the
    shared queue, uploads it (host requests) and runs it alone (vg_louvain_run)."""
    n = 0
    while True:
        with lock:
            if not queue:
                break
            i = queue.pop(0)
        r = requests[i]
        wait = r.arrival - (clock() - t0)
        if wait > 0:
            time.sleep(wait)
        g, owned = r.device_graph(ctx)
        res = ctx.run(g, threshold=r.threshold, want_comm=r.want_comm)
        if owned:
            g.free()
        out[i] = Served(i, r.arrival, clock() - t0, res.stats, res.comm)
        n += 1
    info["rounds"] = n


def serve(ctx: Context, requests: list[Request], budget: int = 0, lanes=(),
          clock=time.perf_counter, direct_above: int | None = None,
          direct_workers: int = 2) -> ServeReport:
    """Run the request stream in real time.

    lanes: ascending CSR-entry bounds; with k bounds the requests are split into k+1
    size classes, each served by its own batch on its own stream and host thread
    (the last class keeps `ctx`), so the rounds of small graphs are not held to
    the length of the largest graphs' phases. Each lane gets the whole budget
    divided in proportion to its share of the requests' entries.

    direct_above: requests with more CSR entries than this skip batching (a graph
    that size fills the GPU alone, and a batch would repack it whenever its lane's
    membership changes): `direct_workers` host threads, each with its own context and
    stream, take them in arrival order and run each alone, so one request's upload
    overlaps another's run. Their memory is outside `budget` (one graph per worker).
    """
    import threading

    bounds = sorted(lanes)
    sizes = [r.ne for r in requests]
    direct = [direct_above is not None and s > direct_above for s in sizes]
    cls = [sum(1 for x in bounds if s > x) for s in sizes]
    nl = len(bounds) + 1
    order = sorted(range(len(requests)), key=lambda i: requests[i].arrival)
    mine = [[i for i in order if cls[i] == k and not direct[i]] for k in range(nl)]
    dqueue = [i for i in order if direct[i]]
    nd = direct_workers if dqueue else 0
    tot = max(sum(s for s, d in zip(sizes, direct) if not d), 1)
    ctxs = [ctx if k == nl - 1 else Context(ctx.device) for k in range(nl)]
    dctxs = [Context(ctx.device) for _ in range(nd)]
    out: dict[int, Served] = {}
    infos = [dict() for _ in range(nl + nd)]
    errors = []
    lock = threading.Lock()

    def run(k, t0):
        try:
            if k >= nl:
                _direct_loop(dctxs[k - nl], requests, dqueue, lock, t0, clock, out, infos[k])
            elif mine[k]:
                share = sum(sizes[i] for i in mine[k]) / tot
                # at least room for the lane's largest graph (the batch's own estimate:
                # 40 bytes per CSR entry, 200 per vertex, 1 MiB)
                big = max(requests[i].footprint() for i in mine[k])
                bud = 0 if budget == 0 else max(int(budget * share), big)
                _lane_loop(ctxs[k], requests, mine[k], bud, t0, clock, out, infos[k])
        except BaseException as e:  # re-raised in the caller
            errors.append(e)

    try:
        t0 = clock()
        threads = [threading.Thread(target=run, args=(k, t0)) for k in range(nl + nd)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    finally:
        for k in range(nl - 1):
            ctxs[k].close()
        for c in dctxs:
            c.close()
    if errors:
        raise errors[0]
    results = [out[i] for i in range(len(requests))]
    first = min(r.arrival for r in requests)
    last = max(r.finish for r in results)
    stats = {"lanes": [{"requests": len(mine[k]), "rounds": infos[k].get("rounds", 0)}
                       for k in range(nl)],
             "direct": {"requests": sum(direct), "workers": nd,
                        "above_entries": direct_above}}
    return ServeReport(results, last - first, sum(i.get("rounds", 0) for i in infos[:nl]), stats)


def fifo(arrivals, service) -> np.ndarray:
    """Finish times of a single FIFO server: start = max(arrival, previous finish)."""
    order = np.argsort(np.asarray(arrivals), kind="stable")
    fin = np.empty(len(order))
    t = -np.inf
    for i in order:
        t = max(t, arrivals[i]) + service[i]
        fin[i] = t
    return fin


def sequential(ctx: Context, requests: list[Request], repeats: int = 1) -> ServeReport:
    """The plain path: each request alone (its upload, for a host request, then
    vg_louvain_run), FIFO by arrival.

    Service times are measured back to back (the whole sequence `repeats` times, each
    request's fastest time kept); the FIFO queue (start = max(arrival, previous
    finish)) then gives each request's finish time for the same arrivals.
    """
    import torch  # device timing on the library's stream

    stream = torch.cuda.ExternalStream(ctx.stream)
    order = sorted(range(len(requests)), key=lambda i: requests[i].arrival)
    service = {}
    levels = {}
    comms = {}
    for _ in range(max(1, repeats)):
        for i in order:
            r = requests[i]
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g, owned = r.device_graph(ctx)
            res = ctx.run(g, threshold=r.threshold, want_comm=r.want_comm)
            if owned:
                g.free()
            e1.record(stream)
            e1.synchronize()
            t = e0.elapsed_time(e1) * 1e-3
            service[i] = min(t, service.get(i, t))
            levels[i] = res.stats
            comms[i] = res.comm
    arr = [r.arrival for r in requests]
    svc = [service[i] for i in range(len(requests))]
    fin = fifo(arr, svc)
    res_list = [Served(i, arr[i], float(fin[i]), levels[i], comms[i]) for i in range(len(requests))]
    return ServeReport(res_list, float(fin.max() - min(arr)), len(requests), {"service_s": svc})


def percentile(x, q: float) -> float:
    return float(np.percentile(np.asarray(x, dtype=np.float64), q))
