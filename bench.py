"""Benchmark: end-to-end multi-level Louvain on RGG n=2^24 (+1% extra U(0,1) edges) on B200.

One step = one full run of graphClustering's phase loop (every level: local-moving
sweeps, community updates, modularity, rebuild) over the graph, through
vg_louvain_run. `value` is seconds per step with the graph already resident in
HBM (device-timed with CUDA events on the library's stream); `e2e` is the same
step through the C ABI from pinned host buffers in Vite's layout, the H2D copy of
the CSR, the per-iteration read-backs and the D2H copy of the -o map (every input
vertex's final community, what distLouvainMethod's caller gets back) inside the
timed region. The reference (oracle/_ref, the unmodified Vite sources) runs once on
the same graph for the CPU baseline, and every level is compared with ours; the
skewed-degree configuration (Barabasi-Albert 4M, -c 8 -t 2 -a 0.25) follows as a
sub-record with its own reference run, then the batched and served forms.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one rank per GPU) every rank runs its own replica of the
workload (the path does not shard: one graph lives on one GPU); rank 0 prints
the max over ranks. --impl reference times the reference's own CPU code
(oracle/_ref) on the host cores on the full graph, generated on the host by the
oracle's generator, without loading the library under test.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_VERTICES = 1 << 24
EXTRA_PERCENT = 1.0
SEED = 2024
THRESHOLD = 1e-6
REF_BUDGET_S = 1500.0      # reference arm: its timed runs end within this many seconds of its start
METRIC = "Louvain e2e sec (RGG 2^24 +1% extra edges, full multi-level)"
UNIT = "s"


# batched workload: many small uneven graphs in one batch
BATCH_GRAPHS = 4096
BATCH_N = (1_000, 256_000)        # vertices, log-uniform
BATCH_SEED = 4242
BATCH_PLAIN_EVERY = 8             # plain path timed on every 8th graph
BATCH_RESERVE = 80 << 30          # device pool mapped before the timed batch
# served workload: Poisson stream of RGG / BA requests
SERVE_REQUESTS = 96
SERVE_E = (1e3, 5e7)              # CSR entries, log-uniform
SERVE_SEED = 5151
SERVE_LOAD = 8.0                  # offered load in units of the plain path's capacity
SERVE_BUDGET = 48 << 30           # device-memory budget of the serving batches
SERVE_LANES = (1 << 16, 1 << 20, 1 << 23)  # CSR-entry bounds of the batched size-class lanes
SERVE_DIRECT = 25_000_000         # larger requests run alone, two at a time (upload overlaps a run)
SERVE_DIRECT_WORKERS = 2
REL_TOL = 1e-9


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=N_VERTICES, help=argparse.SUPPRESS)
    ap.add_argument("--no-cpu-baseline", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--batch-graphs", type=int, default=BATCH_GRAPHS, help=argparse.SUPPRESS)
    ap.add_argument("--serve-requests", type=int, default=SERVE_REQUESTS, help=argparse.SUPPRESS)
    ap.add_argument("--skip-batched", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--skip-serving", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--serve-lanes", type=str, default=None, help=argparse.SUPPRESS)
    ap.add_argument("--skip-ba", action="store_true", help=argparse.SUPPRESS)
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def collectives(ws: int, device: str):
    """The replica path's two collectives: a barrier, and the max of a per-rank time
    (every rank runs its own graph; the job's time is the slowest rank's)."""
    import torch
    import torch.distributed as dist

    def barrier():
        if ws > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    return barrier, max_over_ranks


def workload_config(n: int) -> dict:
    return {"workload": f"RGG n={n} (Vite generator: LCG seed 1, r(n) radius, distance weights) "
                        f"+{EXTRA_PERCENT:g}% extra edges U(0,1) seed {SEED}; full multi-level "
                        f"Louvain, threshold {THRESHOLD:g}, 32-bit ids on device, FP64 weights",
            "n_vertices": n, "extra_edge_percent": EXTRA_PERCENT, "seed": SEED,
            "threshold": THRESHOLD, "parallelism": "replicas (one graph per GPU)",
            "l2": "inputs larger than L2 (CSR of 2^24 RGG = 2.3 GB)"}


# ---------------------------------------------------------------------------------------
# clocks during the timed region


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        # start timing only once the sampler is up (its start-up takes driver locks)
        t0 = time.time()
        while self.proc and time.time() - t0 < 5.0:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.05)
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        loaded = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------------------
# the reference's own code (oracle/_ref, the unmodified Vite sources) on the host cores


def cpu_info() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_rgg_file(path: str, n: int) -> tuple[int, int]:
    """The benchmark graph built on the host by the oracle's generator (bit-identical to
    the device generator: same LCG points, same radius test, same seeded extra edges) and
    written as a Vite binary file; returns (vertices, CSR entries)."""
    from oracle import vite_oracle as vo

    g = vo.rgg(n)
    x, _ = vo.add_random_edges(g, EXTRA_PERCENT, SEED)
    del g
    vo.write_vite_binary(path, x)
    return x.nv, x.ne


def run_reference_arm(args, rank: int, ws: int) -> None:
    """--impl reference: the reference's CPU implementation (graphClustering's phase loop
    over the unmodified Vite sources, oracle/_ref/vite_ref_harness, all host threads) on
    the full benchmark graph. The graph is generated on the host and written once; the
    harness reads it once and runs the whole level loop K times, each run on a fresh copy
    of the level-0 graph; a step is one run (clustering + rebuild of every level, as
    graphClustering reports them). Runs stop early, and the line says so, when one more
    would end past REF_BUDGET_S. This process never loads the library under test."""
    if rank != 0:
        return
    from oracle import vite_oracle as vo

    threads = os.cpu_count() or 1
    t_arm = time.perf_counter()
    if not os.path.exists(vo.HARNESS):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/vite_ref_harness was not built (reference sources absent)"}),
              flush=True)
        return
    with tempfile.TemporaryDirectory() as tmp:
        warm = os.path.join(tmp, "warm.bin")
        cpu_rgg_file(warm, 1 << 16)
        vo.run_harness(["-f", warm, "-r", str(args.warmup)], None, threads=threads, timeout=600)
        path = os.path.join(tmp, "rgg.bin")
        t0 = time.perf_counter()
        nv, ne = cpu_rgg_file(path, args.n)
        gen_s = time.perf_counter() - t0
        budget = max(REF_BUDGET_S - (time.perf_counter() - t_arm), 60.0)
        out = vo.run_harness(["-f", path, "-r", str(args.steps), "-B", f"{budget:.0f}"], None,
                             threads=threads, timeout=budget + 900)
    runs = vo.harness_totals(out)
    secs = [r["total_s"] for r in runs]
    per = statistics.mean(secs)
    sample = (f"the full workload: RGG n={nv} +{EXTRA_PERCENT:g}% extra edges, E={ne} CSR "
              f"entries, generated on the host by the oracle's generator (bit-identical to the "
              f"device generator) and read once from a Vite binary file; each step one whole "
              f"graphClustering level loop (clustering + rebuild, {runs[0]['levels']} levels, "
              f"{runs[0]['iterations']} iterations) on a fresh copy of the graph; mean of "
              f"{len(secs)} runs; {threads} OpenMP threads on {cpu_info()}")
    line = {"metric": METRIC, "value": per, "unit": UNIT, "n_gpus": ws, "steps": len(secs),
            "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args.n), "impl": "reference",
            "cpu_baseline": {"value": per, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": per, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "run_seconds": secs, "final_modularity": runs[-1]["final_mod"],
            "graph_read_s": vo.harness_read_seconds(out), "generate_s": gen_s,
            "warmup_runs": f"{args.warmup} level loops on RGG n=65536 (same generator)"}
    if len(secs) < args.steps:
        line["steps_requested"] = args.steps
        line["note"] = (f"{len(secs)} of {args.steps} runs: one more would have ended past the "
                        f"{REF_BUDGET_S:.0f} s budget of this arm")
    print(json.dumps(line), flush=True)


def reference_levels(path: str, flags: list, threads: int) -> tuple[list, dict]:
    """One reference run (oracle/_ref, all host threads) on a Vite binary file: its
    recorded levels and its totals."""
    from oracle import vite_oracle as vo

    with tempfile.TemporaryDirectory() as tmp:
        rec = os.path.join(tmp, "ref.rec")
        out = vo.run_harness(["-f", path, *flags], rec, threads=threads, timeout=3600)
        levels = vo.read_record(rec).levels
    tot = vo.harness_totals(out)[0]
    tot["read_s"] = vo.harness_read_seconds(out)
    return levels, tot


def level_parity(ours: list, ref_levels: list, our_map, ctx, exact: bool) -> dict:
    """Per level: vertices, entries, iterations and modularity, ours against the reference's;
    and the -o maps (graphClustering's final communities of every input vertex)."""
    from oracle import vite_oracle as vo

    ref = [lv for lv in ref_levels if lv.level >= 0]
    per = []
    for a, b in zip(ours, ref):
        per.append({"nv": [a["nv"], b.nv], "ne": [a["ne"], b.ne], "iters": [a["iters"], b.iters],
                    "modularity": [a["modularity"], b.mod],
                    "rel_diff": abs(a["modularity"] - b.mod) / abs(b.mod) if b.mod else 0.0,
                    "bits_equal": float(a["modularity"]).hex() == float(b.mod).hex()})
    same_shape = len(ours) == len(ref) and all(
        p["nv"][0] == p["nv"][1] and p["ne"][0] == p["ne"][1] and p["iters"][0] == p["iters"][1]
        for p in per)
    out = {"levels": [len(ours), len(ref)], "same_levels_entries_iterations": same_shape,
           "max_rel_modularity_diff": max(p["rel_diff"] for p in per) if per else None,
           "every_modularity_bit_identical": all(p["bits_equal"] for p in per),
           "per_level": per}
    ref_map = vo.output_map(ref_levels)
    if our_map is not None and ref_map is not None:
        cmp = ctx.compare_communities(ref_map, our_map)
        out["output_map"] = {"identical": bool(np.array_equal(ref_map, our_map)),
                             **{k: cmp[k] for k in ("nc1", "nc2", "precision", "recall",
                                                    "fscore")}}
    out["bar"] = ("bit-identical levels (unit weights)" if exact else
                  f"per-level modularity within {REL_TOL:g} relative (real weights)")
    out["pass"] = bool(same_shape and (out["every_modularity_bit_identical"] if exact else
                                      (out["max_rel_modularity_diff"] or 0.0) <= REL_TOL))
    return out


# ---------------------------------------------------------------------------------------
# batched and served forms


def levels_agree(a: list, b: list) -> bool:
    """Same levels (vertices, entries) and per-level modularity within REL_TOL."""
    if len(a) != len(b):
        return False
    for x, y in zip(a, b):
        if (x["nv"], x["ne"]) != (y["nv"], y["ne"]):
            return False
        if abs(x["modularity"] - y["modularity"]) > REL_TOL * abs(y["modularity"]):
            return False
    return True


def batched_workload(ctx, count: int, seed: int):
    """count graphs, n log-uniform in BATCH_N, half RGG (Vite's radius) and half
    Erdos-Renyi (average degree 16), unit or U(0,1) weights per graph."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(BATCH_N[0]), np.log(BATCH_N[1]), count)).astype(np.int64)
    kinds = rng.permutation(np.arange(count) % 2)
    real = rng.integers(0, 2, count)
    graphs = []
    for i in range(count):
        if kinds[i] == 0:
            g = ctx.generate_rgg(int(ns[i]), 0.0, 0)
        else:
            g = ctx.generate_er(int(ns[i]), 16.0, seed * 100_003 + i)
        if real[i]:
            ctx.reweight(g, 2, seed * 7_919 + i)
        else:
            ctx.reweight(g, 1)
        graphs.append(g)
    return graphs, kinds, real


def run_batched(ctx, stream, count: int) -> dict:
    import torch

    t0 = time.perf_counter()
    graphs, kinds, real = batched_workload(ctx, count, BATCH_SEED)
    gen_s = time.perf_counter() - t0
    nv = [g.nv for g in graphs]
    ne = [g.ne for g in graphs]
    # warm-up of both paths on a few small graphs
    warm = [ctx.generate_er(2000, 16.0, 1), ctx.generate_rgg(3000, 0.0, 0)]
    for g in warm:
        ctx.run(g, threshold=THRESHOLD)
    ctx.run_batch(warm, threshold=THRESHOLD)
    for g in warm:
        g.free()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return out, e0.elapsed_time(e1) * 1e-3

    # degree-class bounds and tile grid from the autotuner, on 16 of the batch's graphs
    # spread over its size range; the plain sample and the batch both run under them
    by_size = np.argsort(np.asarray(ne), kind="stable")
    tune_set = [graphs[int(by_size[k])] for k in np.linspace(0, count - 1, min(16, count)).astype(int)]
    t_tune = time.perf_counter()
    before = ctx.tuning
    tuned = ctx.autotune(tune_set, sweeps=2)
    t_tune = time.perf_counter() - t_tune
    sample = list(range(0, count, BATCH_PLAIN_EVERY))
    plain, t_plain = timed(lambda: [ctx.run(graphs[i], threshold=THRESHOLD).stats for i in sample])
    # the batch's working set is mapped once, as a long-running service would
    ctx.reserve(min(40 * sum(ne) + 200 * sum(nv), BATCH_RESERVE))

    def batch_all():
        with ctx.batch() as b:
            ids = [b.submit(g, threshold=THRESHOLD, take=True) for g in graphs]
            b.run_all()
            return [b.result(j).stats for j in ids], b.stats()

    (res, bst), t_batch = timed(batch_all)
    ctx.tuning = before  # the later legs run under the context's previous tuning
    agree = sum(levels_agree(res[i], plain[k]) for k, i in enumerate(sample))
    gps = count / t_batch
    plain_gps = len(sample) / t_plain
    return {
        "workload": f"{count} graphs, n log-uniform [{BATCH_N[0]}, {BATCH_N[1]}], half RGG "
                    f"(Vite radius) half Erdos-Renyi (avg degree 16), unit or U(0,1) FP64 "
                    f"weights per graph, seed {BATCH_SEED}; full multi-level Louvain, "
                    f"threshold {THRESHOLD:g}",
        "graphs": count, "vertices": int(sum(nv)), "csr_entries": int(sum(ne)),
        "rgg": int((kinds == 0).sum()), "real_weights": int(real.sum()),
        "graphs_per_s": gps, "seconds": t_batch, "rounds": bst["rounds"],
        "plain_graphs_per_s": plain_gps,
        "plain_sample": f"every {BATCH_PLAIN_EVERY}th graph ({len(sample)} graphs) run alone "
                        f"through vg_louvain_run back to back: {t_plain:.3f} s",
        "speedup_vs_plain": gps / plain_gps,
        "agree_with_plain": f"{agree}/{len(sample)} graphs: same levels, per-level modularity "
                            f"within {REL_TOL:g} relative",
        "generate_seconds": gen_s,
        "tuning": {**tuned["tuning"], "sweep_ms": tuned["sweep_ms"],
                   "start_sweep_ms": tuned["start_sweep_ms"], "seconds": t_tune,
                   "set": "vg_autotune on 16 of the batch's graphs spread over its size range "
                          "(first 2 sweeps of a phase each, faster of two timings)"},
    }


def rgg_vertices_for_entries(e: float) -> int:
    """n whose Vite-radius RGG has about e CSR entries (n * pi r(n)^2 * n)."""
    def entries(n):
        r = (np.sqrt(np.log(n) / (3.14159 * n)) + np.sqrt(2.0736 / n)) / 2.0
        return n * 3.14159 * r * r * n
    lo, hi = 16.0, 1e9
    for _ in range(80):
        mid = np.sqrt(lo * hi)
        if entries(mid) < e:
            lo = mid
        else:
            hi = mid
    return int(round(lo))


def serving_workload(ctx, count: int, seed: int):
    """count requests, CSR entries log-uniform in SERVE_E, RGG (distance weights) or
    Barabasi-Albert (m = 8, U(0,1) weights), unit-rate Poisson arrival times. Each
    request's graph is built on the device and moved to pinned host memory in Vite's
    layout (row offsets + Edge records): a request is uploaded when it is admitted."""
    import torch

    import vite_b200

    rng = np.random.default_rng(seed)
    es = np.exp(rng.uniform(np.log(SERVE_E[0]), np.log(SERVE_E[1]), count))
    kinds = rng.integers(0, 2, count)
    base = np.cumsum(rng.exponential(1.0, count))
    hosts = []
    for i in range(count):
        if kinds[i] == 0:
            g = ctx.generate_rgg(max(rgg_vertices_for_entries(es[i]), 64), 0.0, 0)
        else:
            g = ctx.generate_ba(max(int(es[i] / 16), 32), 8, seed * 1_000 + i)
            ctx.reweight(g, 2, seed * 31 + i)
        rp, tail, w = g.download()
        g.free()
        rp_pin = torch.empty(len(rp), dtype=torch.int64, pin_memory=True)
        ed_pin = torch.empty(2 * len(tail), dtype=torch.int64, pin_memory=True)
        rp_pin.numpy()[:] = rp
        ed = ed_pin.numpy().view(vite_b200.EDGE_DTYPE)
        ed["tail"] = tail
        ed["weight"] = w
        hosts.append((rp_pin, ed_pin, rp_pin.numpy(), ed))
    return hosts, kinds, base


def serving_bound(service: list, visits: list, ne: list) -> dict:
    """What batching can gain on this mix at most. A request's plain service time t_i
    cannot shrink below what its own edge visits (sum over levels of entries x
    iterations) cost at the best rate any request reached alone, R = max_i v_i / t_i;
    requests that already run within 20 % of R alone (the large ones: they fill the GPU
    by themselves) keep their own time. T_served >= sum_sat t_i + sum_other v_i / R, so
    served/plain throughput <= sum t_i / that."""
    t = np.asarray(service, dtype=np.float64)
    v = np.asarray(visits, dtype=np.float64)
    rate = v / t
    R = float(rate.max())
    sat = rate >= 0.8 * R
    floor_ = float(t[sat].sum() + (v[~sat] / R).sum())
    return {"peak_rate_edge_visits_per_s": R, "saturating_requests": int(sat.sum()),
            "saturating_min_entries": int(np.asarray(ne)[sat].min()) if sat.any() else None,
            "plain_time_share_of_saturating": float(t[sat].sum() / t.sum()),
            "min_served_seconds": floor_, "max_speedup": float(t.sum() / floor_),
            "rule": "T_served >= sum(t_i, requests within 20% of the best rate R alone) + "
                    "sum(visits_i / R, the others); visits = sum over levels of entries x "
                    "iterations; t_i = plain service time with the upload"}


def run_serving(ctx, count: int, lanes=SERVE_LANES) -> dict:
    from vite_b200 import serve as sv

    hosts, kinds, base = serving_workload(ctx, count, SERVE_SEED)
    reqs = [sv.Request(None, 0.0, THRESHOLD, rowptr=h[2], edges=h[3]) for h in hosts]
    ne = [r.ne for r in reqs]
    plain = sv.sequential(ctx, reqs, repeats=2)
    service = plain.stats["service_s"]
    visits = [sum(lv["ne"] * lv["iters"] for lv in r.levels) for r in plain.results]
    cap = count / sum(service)              # plain graphs/s, back to back
    rate = SERVE_LOAD * cap
    arrivals = base / base[-1] * (count / rate)
    for r, a in zip(reqs, arrivals):
        r.arrival = float(a)
    fin = sv.fifo(arrivals, service)
    plain_lat = fin - arrivals
    ctx.reserve(SERVE_BUDGET)
    served = sv.serve(ctx, reqs, budget=SERVE_BUDGET, lanes=lanes, direct_above=SERVE_DIRECT,
                      direct_workers=SERVE_DIRECT_WORKERS)
    lat = served.latencies()
    agree = sum(levels_agree(s.levels, p.levels) for s, p in zip(served.results, plain.results))
    gps = count / served.seconds
    plain_gps = count / float(fin.max() - arrivals.min())
    bound = serving_bound(service, visits, ne)
    del hosts
    return {
        "workload": f"{count} requests, CSR entries log-uniform [{SERVE_E[0]:g}, {SERVE_E[1]:g}], "
                    f"RGG (distance weights) or Barabasi-Albert m=8 (U(0,1) weights), held in "
                    f"pinned host memory in Vite's layout and uploaded on admission; Poisson "
                    f"arrivals at {SERVE_LOAD:g}x the plain path's capacity, seed {SERVE_SEED}; "
                    f"budget {SERVE_BUDGET >> 30} GiB, batched size-class lanes at "
                    f"{'/'.join(str(x) for x in lanes)} CSR entries, requests above "
                    f"{SERVE_DIRECT} entries run alone on {SERVE_DIRECT_WORKERS} streams; full "
                    f"multi-level Louvain",
        "requests": count, "csr_entries": int(sum(ne)), "rate_per_s": rate,
        "graphs_per_s": gps, "p50_s": sv.percentile(lat, 50),
        "p99_s": sv.percentile(lat, 99), "rounds": served.rounds,
        "lanes": served.stats["lanes"], "direct": served.stats["direct"],
        "plain_graphs_per_s": plain_gps,
        "speedup_vs_plain": gps / plain_gps,
        "plain_p50_s": sv.percentile(plain_lat, 50), "plain_p99_s": sv.percentile(plain_lat, 99),
        "plain": "each request alone (upload from pinned host memory + vg_louvain_run), FIFO "
                 "in arrival order; service times measured back to back on the device, the "
                 "sequence twice, each request's faster time; finish times from the FIFO "
                 "queue over those service times",
        "bound": bound,
        "fraction_of_bound": (gps / plain_gps) / bound["max_speedup"],
        "agree_with_plain": f"{agree}/{count} requests: same levels, per-level modularity within "
                            f"{REL_TOL:g} relative",
    }


def write_vite_file(path: str, rp: np.ndarray, ed: np.ndarray) -> None:
    """Vite's binary layout: nv, ne, rowptr[nv+1], Edge{int64 tail, double weight}[ne]."""
    import struct

    with open(path, "wb") as f:
        f.write(struct.pack("<qq", len(rp) - 1, len(ed)))
        np.ascontiguousarray(rp, dtype="<i8").tofile(f)
        ed.tofile(f)


# the skewed-degree configuration: Barabasi-Albert, unit weights, coloring + ET
BA_N, BA_M, BA_SEED = 4_194_304, 8, 1
BA_FLAGS = ["-c", "8", "-t", "2", "-a", "0.25"]
BA_KW = {"coloring": True, "max_colors": 8, "et_type": 2, "et_delta": 0.25}
BA_STEPS = 10


def run_ba_config(ctx, stream, args) -> dict:
    """Barabasi-Albert n=4,194,304, m=8 (seed 1), unit FP64 weights, graphClustering
    -c 8 -t 2 -a 0.25 (distance-1 coloring, early termination alpha 0.25): device-resident
    and end-to-end times, and the reference's own run on the same graph (oracle/_ref, all
    host threads) with every level compared bit for bit (unit weights: every sum is exact)."""
    import torch

    import vite_b200

    g = ctx.generate_ba(BA_N, BA_M, BA_SEED)
    nv, ne = g.nv, g.ne
    rp_h, tail_h, w_h = g.download()
    rp_pin = torch.empty(nv + 1, dtype=torch.int64, pin_memory=True)
    ed_pin = torch.empty(ne * 2, dtype=torch.int64, pin_memory=True)
    rp_pin.numpy()[:] = rp_h
    ed = ed_pin.numpy().view(vite_b200.EDGE_DTYPE)
    ed["tail"] = tail_h
    ed["weight"] = w_h
    del rp_h, tail_h, w_h
    comm_pin = torch.empty(nv, dtype=torch.int64, pin_memory=True)

    def timed(fn, k):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            out = fn()
        e1.record(stream)
        e1.synchronize()
        return out, e0.elapsed_time(e1) * 1e-3 / k

    def e2e():
        h = ctx.upload_edges(rp_pin.numpy(), ed)
        r = ctx.run(h, threshold=THRESHOLD, comm_out=comm_pin.numpy(), **BA_KW)
        h.free()
        return r

    for _ in range(3):
        ctx.run(g, threshold=THRESHOLD, **BA_KW)
    dev, t_dev = timed(lambda: ctx.run(g, threshold=THRESHOLD, **BA_KW), BA_STEPS)
    e2e()
    res, t_e2e = timed(e2e, BA_STEPS)
    out = {"workload": f"Barabasi-Albert n={nv} m={BA_M} (seed {BA_SEED}), unit FP64 weights, "
                       f"graphClustering {' '.join(BA_FLAGS)} (coloring with 4 hash rounds, "
                       f"early termination alpha 0.25), threshold {THRESHOLD:g}",
           "nv": nv, "ne": ne, "seconds": t_dev, "e2e_seconds": t_e2e, "steps": BA_STEPS,
           "e2e_bytes": {"h2d": 8 * (nv + 1) + 16 * ne,
                         "d2h": 8 * nv + 16 * sum(s["iters"] for s in res.stats)},
           "levels": [{"nv": s["nv"], "ne": s["ne"], "iters": s["iters"],
                       "modularity": s["modularity"], "colors": s["num_colors"],
                       "color_s": s["seconds_color"], "phase_s": s["seconds_phase"],
                       "rebuild_s": s["seconds_rebuild"]} for s in dev.stats]}
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, "ba.bin")
            write_vite_file(path, rp_pin.numpy(), ed)
            ref_lv, tot = reference_levels(path, BA_FLAGS, threads)
        out["reference_seconds"] = tot["total_s"]
        out["reference"] = (f"oracle/_ref/vite_ref_harness -f <graph> {' '.join(BA_FLAGS)}, "
                            f"{threads} OpenMP threads on {cpu_info()}: clustering "
                            f"{tot['clustering_s']:.2f} s + rebuild {tot['rebuild_s']:.2f} s "
                            f"(graph read {tot['read_s']:.1f} s excluded)")
        out["parity"] = level_parity(res.stats, ref_lv, comm_pin.numpy(), ctx, exact=True)
        out["e2e_speedup_vs_reference"] = tot["total_s"] / t_e2e
    g.free()
    return out


def main() -> None:
    args = parse()
    ws, rank, local = dist_env()
    assert args.warmup >= 3, "at least 3 warm-up steps"
    if args.impl == "reference":
        run_reference_arm(args, rank, ws)
        return

    import torch
    import torch.distributed as dist

    import vite_b200

    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    barrier, max_over_ranks = collectives(ws, "cuda")

    ctx = vite_b200.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    g = ctx.generate_rgg(args.n, EXTRA_PERCENT, SEED)
    nv, ne = g.nv, g.ne

    # pinned host copy of the CSR in Vite's layout for the end-to-end leg
    rp_h, tail_h, w_h = g.download()
    rp_pin = torch.empty(nv + 1, dtype=torch.int64, pin_memory=True)
    ed_pin = torch.empty(ne * 2, dtype=torch.int64, pin_memory=True)
    rp_pin.numpy()[:] = rp_h
    ed = ed_pin.numpy().view(vite_b200.EDGE_DTYPE)
    ed["tail"] = tail_h
    ed["weight"] = w_h
    del rp_h, tail_h, w_h
    # the -o map (final community of every input vertex) comes back here in the e2e leg
    comm_pin = torch.empty(nv, dtype=torch.int64, pin_memory=True)

    def step_device():
        return ctx.run(g, threshold=THRESHOLD)

    def step_e2e():
        h = ctx.upload_edges(rp_pin.numpy(), ed)
        res = ctx.run(h, threshold=THRESHOLD, comm_out=comm_pin.numpy())
        h.free()
        return res

    # the working set of a run (graph, its layout copy, phase state, rebuild
    # temporaries) is reserved once so that no step maps new memory mid-run
    ctx.reserve(int(64 * ne + 256 * nv))
    step_e2e()
    for _ in range(args.warmup):
        res = step_device()

    # device-resident leg
    barrier()
    torch.cuda.synchronize()
    ctx.profile(False, reset=True)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        barrier()
        runs = [None] * args.steps
        # the NVTX range lets a profiler select the timed launches (--nvtx-include bench_timed/)
        torch.cuda.nvtx.range_push("bench_timed")
        evs[0].record(stream)
        for k in range(args.steps):
            runs[k] = step_device()
            evs[k + 1].record(stream)
        torch.cuda.nvtx.range_pop()
        evs[-1].synchronize()
        torch.cuda.synchronize()
        barrier()
    _, launches = ctx.profile(False, reset=True)
    step_s = [evs[k].elapsed_time(evs[k + 1]) * 1e-3 for k in range(args.steps)]
    t_dev = max_over_ranks(evs[0].elapsed_time(evs[-1]) * 1e-3)
    clocks = clk.summary()

    # end-to-end leg through the C ABI from pinned host buffers
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        res_e2e = step_e2e()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    t_e2e = max_over_ranks(e0.elapsed_time(e1) * 1e-3)

    per_step = t_dev / args.steps
    per_e2e = t_e2e / args.steps
    last = runs[-1].stats
    lv0 = last[0]
    sweep_total = sum(s["seconds_sweep"] for s in last)
    edges_total = sum(s["edges_swept"] for s in last)
    # roofline of the local-moving sweep at level 0: algorithmic bytes 16*E + 48*V per sweep
    sweep_bytes = 16 * lv0["ne"] + 48 * lv0["nv"]
    t_sweep = lv0["seconds_sweep"] / max(lv0["iters"], 1)
    achieved = sweep_bytes / t_sweep / 1e9
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = json.load(open(peaks_path))["hbm_gbs"]
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "sweep_traffic.json")
    if os.path.exists(tpath):
        tj = json.load(open(tpath))
        traffic = tj.get("dram_bytes_per_sweep_level0")

    cpu, parity = None, None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        # the reference (oracle/_ref, all host threads) once on the whole benchmark graph,
        # read from a Vite binary file: its time is the CPU baseline, its levels and -o map
        # are compared with ours
        threads = os.cpu_count() or 1
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, "rgg.bin")
            write_vite_file(path, rp_pin.numpy(), ed)
            ref_lv, tot = reference_levels(path, [], threads)
        cpu = {"value": tot["total_s"], "unit": UNIT, "cores": threads, "kind": "reference",
               "sample": f"the full workload once (E={ne}): graphClustering's level loop over "
                         f"the unmodified Vite sources (oracle/_ref), clustering "
                         f"{tot['clustering_s']:.2f} s + rebuild {tot['rebuild_s']:.2f} s, "
                         f"{tot['levels']} levels; graph read from a Vite binary file "
                         f"({tot['read_s']:.1f} s, excluded); {threads} OpenMP threads on "
                         f"{cpu_info()}"}
        parity = level_parity(res_e2e.stats, ref_lv, comm_pin.numpy(), ctx, exact=False)
        del ref_lv

    line = {
        "metric": METRIC, "value": per_step, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.n),
        "levels": [{"nv": s["nv"], "ne": s["ne"], "iters": s["iters"],
                    "modularity": s["modularity"], "sweep_s": s["seconds_sweep"],
                    "phase_s": s["seconds_phase"], "rebuild_s": s["seconds_rebuild"]}
                   for s in last],
        "final_modularity": max(s["modularity"] for s in last),
        "step_seconds": step_s,
        "layout_s": lv0_layout if (lv0_layout := last[0].get("seconds_layout")) else 0.0,
        "local_move_gteps": edges_total / sweep_total / 1e9 if sweep_total else None,
        "graphs_per_s_total": ws * args.steps / t_dev,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": "local-moving sweep (all degree-class launches of one iteration), "
                               f"level 0; algorithmic bytes 16*E+48*V = {sweep_bytes}; "
                               f"peak {peak_src}"},
        # D2H per step: the -o map (8 B per input vertex) and the modularity +
        # frozen-count read-back (16 B) of every iteration
        "e2e": {"value": per_e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * (nv + 1) + 16 * ne,
                "d2h_bytes_per_step": 8 * nv + 16 * sum(s["iters"] for s in res_e2e.stats)},
        "gpu_launches": launches,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if parity is not None:
        line["reference_parity"] = parity
    g.free()
    del rp_pin, ed_pin, ed, comm_pin
    if ws == 1 and not args.skip_ba:
        line["ba_config"] = run_ba_config(ctx, stream, args)
    if ws == 1 and not args.skip_batched:
        line["batched"] = run_batched(ctx, stream, args.batch_graphs)
    if ws == 1 and not args.skip_serving:
        lanes = (tuple(int(x) for x in args.serve_lanes.split(",") if x)
                 if args.serve_lanes is not None else SERVE_LANES)
        line["serving"] = run_serving(ctx, args.serve_requests, lanes)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
