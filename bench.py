"""Benchmark: end-to-end multi-level Louvain on RGG n=2^24 (+1% extra U(0,1) edges) on B200.

One step = one full run of graphClustering's phase loop (every level: local-moving
sweeps, community updates, modularity, rebuild) over the graph, through
vg_louvain_run. `value` is seconds per step with the graph already resident in
HBM (device-timed with CUDA events on the library's stream); `e2e` is the same
step through the C ABI from pinned host buffers in Vite's layout, the H2D copy of
the CSR and the D2H read of the per-level results inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one rank per GPU) every rank runs its own replica of the
workload (the path does not shard: one graph lives on one GPU); rank 0 prints
the max over ranks. --impl reference times the reference's own CPU code
(oracle/_ref, built from the reference sources) on the host cores.
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
SAMPLE_VERTICES = 1 << 20  # CPU-baseline sample (same generator, same seed)
METRIC = "Louvain e2e sec (RGG 2^24 +1% extra edges, full multi-level)"
UNIT = "s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=N_VERTICES, help=argparse.SUPPRESS)
    ap.add_argument("--no-cpu-baseline", action="store_true", help=argparse.SUPPRESS)
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


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
# CPU baseline: the reference's own code (oracle/_ref) on a bounded sample


def reference_sample_seconds(ctx, threads: int, n_sample: int) -> tuple[float, int, str]:
    """Run the reference binary on an RGG sample written in Vite's binary format;
    returns (seconds of clustering + rebuild, CSR entries of the sample, kind)."""
    from oracle import vite_oracle as vo

    g = ctx.generate_rgg(n_sample, EXTRA_PERCENT, SEED)
    rp, tail, w = g.download()
    g.free()
    sample = vo.Graph(rp, tail, w)
    if os.path.exists(vo.HARNESS):
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, "sample.bin")
            vo.write_vite_binary(path, sample)
            out = vo.run_harness(["-f", path], os.path.join(tmp, "s.rec"), threads=threads,
                                 timeout=600)
        tot = [l for l in out.splitlines() if l.startswith("HARNESS total_clustering_s")][0].split()
        return float(tot[6]), sample.ne, "reference"
    r = vo.run(sample)  # restatement (single thread) when the reference build is absent
    return r.seconds, sample.ne, "port"


def run_reference_arm(args, rank: int, ws: int) -> None:
    """--impl reference: the reference's CPU implementation on the host cores."""
    if rank != 0:
        return
    import vite_b200
    threads = os.cpu_count() or 1
    ctx = vite_b200.Context(int(os.environ.get("LOCAL_RANK", "0")))
    full = ctx.generate_rgg(args.n, EXTRA_PERCENT, SEED)
    e_full = full.ne
    full.free()
    for _ in range(args.warmup):
        reference_sample_seconds(ctx, threads, 1 << 14)
    secs = []
    kind, e_s = "reference", 1
    for _ in range(args.steps):
        s, e_s, kind = reference_sample_seconds(ctx, threads, SAMPLE_VERTICES)
        secs.append(s)
    ctx.close()
    per = statistics.mean(secs) * e_full / e_s
    sample = (f"RGG n={SAMPLE_VERTICES} +{EXTRA_PERCENT:g}% (E={e_s}) full multi-level Louvain "
              f"(clustering + rebuild, graph load excluded), mean of {len(secs)} runs "
              f"({statistics.mean(secs):.3f} s), scaled by CSR entries to E={e_full}")
    line = {"metric": METRIC, "value": per, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args.n), "impl": "reference",
            "cpu_baseline": {"value": per, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": per, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------


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

    def barrier():
        if ws > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

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

    def step_device():
        return ctx.run(g, threshold=THRESHOLD)

    def step_e2e():
        h = ctx.upload_edges(rp_pin.numpy(), ed)
        res = ctx.run(h, threshold=THRESHOLD)
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
        step_e2e()
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

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        s, e_s, kind = reference_sample_seconds(ctx, threads, SAMPLE_VERTICES)
        cpu = {"value": s * ne / e_s, "unit": UNIT, "cores": threads if kind == "reference" else 1,
               "kind": kind,
               "sample": f"RGG n={SAMPLE_VERTICES} +{EXTRA_PERCENT:g}% (E={e_s}), full multi-level "
                         f"Louvain measured {s:.3f} s, scaled by CSR entries to E={ne}"}

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
        # D2H per step: the modularity + frozen-count read-back (16 B) of every iteration
        "e2e": {"value": per_e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * (nv + 1) + 16 * ne,
                "d2h_bytes_per_step": 16 * sum(s["iters"] for s in last)},
        "gpu_launches": launches,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.free()
    ctx.close()
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
