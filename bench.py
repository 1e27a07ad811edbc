#!/usr/bin/env python
"""Throughput of exact Pareto-frontier enumeration on B200.

Workload (one "step"): the batched stream -- 512 knapsack BDDs (3 objectives,
n ~ U{20..60}) + 256 set-packing independent-set BDDs (3 objectives, n ~ U{60..100},
20 constraints), seeds 0..767, all enumerated top-down (method 1) through one engine
run whose every launch covers every instance still running.

  value   solves/s with the DDs already resident in HBM (pmdd_resident_*), device time
          from CUDA events on the engine stream, summed over the K timed steps;
          L2 flushed (256 MiB write) between timed steps.
  e2e     solves/s through pmdd_enumerate_batch with host DD buffers: DD upload and
          frontier download inside the timed region (host clock around the call).
Extra keys: one-at-a-time solves/s of the same stream through pmdd_enumerate, the
served loop (Poisson arrivals at 50/200/800 req/s, KP/SP method 1 + TSP method 3, and
the same mix submitted at once for the server's capacity),
the config-1 filter roofline (1024 x KP d=3 n=40), the reference CPU baseline.

Multi-GPU: one process per GPU (torchrun); every rank enumerates its own stream
(seeds offset by rank), no data-path collective ("replicas", weak scaling); the
timed region is bracketed by barriers and the max over ranks is reported.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s + p50/p99 latency, batched vs one-at-a-time on B200; filter % HBM"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ------------------------------------------------------------------ helpers
def build_dds(specs, threads=16):
    """specs: list of (problem_type, text, tag) -> DecisionDiagrams (built in parallel;
    ctypes releases the GIL inside the C++ constructors)."""
    from pmdd_b200 import DecisionDiagram

    def one(s):
        return DecisionDiagram.from_text(s[1], s[0], 3)

    with cf.ThreadPoolExecutor(threads) as ex:
        return list(ex.map(one, specs))


def kp_arrays_from_text(text):
    """(profits (d, n), weights (n,), capacity) of a one-constraint knapsack instance text."""
    tok = list(map(int, text.split()))
    n, m, d = tok[0], tok[1], tok[2]
    assert m == 1
    prof = np.array(tok[3:3 + d * n], dtype=np.int32).reshape(d, n)
    w = np.array(tok[3 + d * n:3 + d * n + n], dtype=np.int32)
    return prof, w, tok[3 + d * n + n]


def dd_bytes(dd):
    v = dd.view
    n = (v.num_layers + 1) + (v.num_nodes + 1) + 2 * v.num_arcs + v.num_weights * v.nobjs
    if v.min_weight:
        n += v.num_nodes
    if v.node_state:
        n += 2 * v.num_nodes * v.state_words
    return 4 * n


def read_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for name, val in zip(names, parts[5:9]):
                    if val.lower() in ("active", "1", "yes"):
                        reasons.add(name)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------- reference CPU arm
def cpu_reference_sample(specs, workers, budget_s=25.0, max_items=96):
    """Reference binary (oracle/_ref) on a bounded sample of the stream, `workers`
    concurrent single-threaded processes; returns (solves/s, sample size, kind)."""
    import oracle

    sample = specs[:: max(1, len(specs) // max_items)][:max_items]
    if not oracle.have_ref(3):
        return None
    tmp = tempfile.mkdtemp()
    paths = []
    for i, (ptype, text, tag) in enumerate(sample):
        p = os.path.join(tmp, f"{i}.dat")
        with open(p, "w") as f:
            f.write(text)
        paths.append((ptype, p))
    lock = threading.Lock()
    per_worker = [0.0] * workers
    done = [0]
    t_start = time.time()

    def work(w):
        for k in range(w, len(paths), workers):
            if time.time() - t_start > budget_s * 4:
                break
            ptype, p = paths[k]
            r = oracle.run_ref(p, ptype, 1, 3, threads=1)
            with lock:
                per_worker[w] += float(r["stats"]["timing"]["wall"]["wall_enumeration_s"])
                done[0] += 1

    with cf.ThreadPoolExecutor(workers) as ex:
        list(ex.map(work, range(workers)))
    makespan = max(per_worker) if per_worker else 0.0
    return (done[0] / makespan if makespan > 0 else None), done[0]


def single_instances(P, instances, device, with_ref):
    """The single-instance configurations (seed 0): 3-objective knapsack n=40, 4-objective
    knapsack n=60, 7-objective knapsack n=25, 3-objective set packing n=100 (m=20), each by
    methods 1 and 3.  GPU: device time of one pmdd_enumerate after a warm-up call, and the
    wall time of the call from host buffers.  Reference CPU (when built): its own binary
    with every host thread, wall_enumeration_s of its stats record (DD build excluded)."""
    import oracle  # reference CPU leg only

    cases = [("kp3_n40", 1, 3, instances.knapsack_text(40, 3, 0)),
             ("kp4_n60", 1, 4, instances.knapsack_text(60, 4, 0)),
             ("kp7_n25", 1, 7, instances.knapsack_text(25, 7, 0)),
             ("sp3_n100_m20", 2, 3, instances.setpacking_text(100, 20, 3, 0))]
    threads = os.cpu_count() or 1
    out = []
    tmp = tempfile.mkdtemp()
    for name, ptype, d, text in cases:
        dd = P.DecisionDiagram.from_text(text, ptype, d)
        path = os.path.join(tmp, name + ".dat")
        with open(path, "w") as f:
            f.write(text)
        for method in (1, 3):
            P.enumerate_dd(dd, method=method, device=device)
            st = {}
            t0 = time.perf_counter()
            pts = P.enumerate_dd(dd, method=method, stats=st, device=device)
            wall = time.perf_counter() - t0
            rec = {"instance": name, "method": method, "solutions": int(len(pts)),
                   "gpu_device_s": st["device_elapsed_s"], "gpu_call_s": wall,
                   "candidates": int(st["work_candidates_total"]), "join_products": int(st["work_join_products_total"]),
                   "candidates_filtered_per_s": st["work_candidates_total"] / st["device_elapsed_s"]}
            if with_ref and oracle.have_ref(d):
                r = oracle.run_ref(path, ptype, method, d, threads=threads)
                rec["ref_cpu_s"] = float(r["stats"]["timing"]["wall"]["wall_enumeration_s"])
                rec["ref_cpu_threads"] = threads
                rec["ref_solutions"] = int(r["stats"]["outputs"]["num_solutions"])
            out.append(rec)
    return out


# --------------------------------------------------------------- served loop
def served_loop(rate, n_req, seed, P, instances, device=0, detail=None):
    """Poisson arrivals at `rate` req/s (rate 0: every request at once, so that solves/s is
    the server's capacity on the mix); KP (n~U{20..60}) / SP (n~U{60..100}) method 1 and
    TSP (n~U{9..13}, method 3); latency = finish - arrival on the host clock.  Afterwards
    every request runs alone on an idle server (submit -> result); the slowdown of a
    request is its served latency over its lone one.  Knapsack
    and set-packing DDs are built on the host before the loop; a TSP request goes in by
    its cost matrices (the server's shared n-city MDD on the device).  Every
    result's frontier CSV.gz and stats record are handed to the asynchronous writer as it
    is polled (the reference's per-request output); the writer's tail after the last
    result is reported beside the latencies.  The TSP sizes' shared structures are built
    in both servers before any request (a server's warm-up), so that neither latency
    includes a first request's build."""
    from pmdd_b200.writer import FrontierWriter

    mix = instances.served_mix(n_req, seed)
    specs = [(p, instances.tsp_arrays_from_tag(tag) if p == 3 else text, m) for p, text, m, tag in mix]
    built = iter(build_dds([(p, t, "") for p, t, _ in specs if p != 3]))
    dds = [t if p == 3 else next(built) for p, t, _ in specs]
    rng = np.random.default_rng(seed + 1)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_req)) if rate > 0 else np.zeros(n_req)
    srv = P.Server(device=device)
    tsp_sizes = sorted({int(tag.split("_")[1][1:]) for p, _, _, tag in mix if p == 3})
    for n in tsp_sizes:  # the shared n-city structures, built before the clock starts
        srv.prepare_tsp(n)
    outdir = tempfile.mkdtemp(prefix="pmdd_served_")
    writer = FrontierWriter()
    t0 = time.perf_counter()
    t0_mono = time.monotonic()
    nxt = 0
    lat = []
    finished = 0
    while finished < n_req:
        now = time.perf_counter() - t0
        while nxt < n_req and arrivals[nxt] <= now:
            if specs[nxt][0] == 3:
                srv.submit_tsp(dds[nxt], nxt, method=specs[nxt][2])
            else:
                srv.submit(dds[nxt], nxt, method=specs[nxt][2])
            nxt += 1
        if srv.pending() == 0:
            if nxt < n_req:
                time.sleep(max(0.0, min(0.002, arrivals[nxt] - now)))
            continue
        srv.run(1)
        while True:
            r = srv.poll()
            if r is None:
                break
            if r.status != 0:
                raise RuntimeError(f"served request {r.req_id} failed: {r.error}")
            # finish_s is the engine's steady clock; arrival is relative to t0
            lat.append((r.req_id, (r.finish_s - (t0_mono + arrivals[r.req_id])) * 1e3))
            finished += 1
            rec = json.dumps({"request": int(r.req_id), "problem_type": specs[r.req_id][0],
                              "method": specs[r.req_id][2], "num_solutions": int(len(r.frontier))})
            writer.submit(r.frontier, os.path.join(outdir, f"r{r.req_id}.frontier.csv.gz"),
                          os.path.join(outdir, "stats.jsonl"), rec)
    wall = time.perf_counter() - t0
    info = srv.info()
    srv.close()
    tw = time.perf_counter()
    written = writer.flush()
    tail_ms = (time.perf_counter() - tw) * 1e3
    writer.close()
    shutil.rmtree(outdir, ignore_errors=True)
    # each request alone: a server with nothing else to do, submit -> result
    alone = np.zeros(n_req)
    lone = P.Server(device=device)
    for n in tsp_sizes:
        lone.prepare_tsp(n)
    for i in range(n_req):
        if specs[i][0] == 3:
            lone.submit_tsp(dds[i], i, method=specs[i][2])
        else:
            lone.submit(dds[i], i, method=specs[i][2])
        while lone.pending() > 0:
            lone.run(0)
        r = lone.poll()
        alone[i] = (r.finish_s - r.submit_s) * 1e3
    lone.close()
    ids = np.array([i for i, _ in lat])
    lat = np.array([x for _, x in lat])
    slow = lat / np.maximum(alone[ids], 1e-3)
    if detail is not None:  # per request: tag, method, served and lone latency (profiling aid)
        served_ms = dict(zip(ids.tolist(), lat.tolist()))
        detail.extend({"tag": mix[i][3], "method": mix[i][2], "served_ms": served_ms[i], "alone_ms": float(alone[i]),
                       "arrival_s": float(arrivals[i])} for i in range(n_req))
    return {"rate_rps": rate if rate > 0 else None, "arrivals": "poisson" if rate > 0 else "all at once",
            "requests": n_req, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "solves_per_s": n_req / wall,
            "alone_p50_ms": float(np.percentile(alone, 50)), "alone_p99_ms": float(np.percentile(alone, 99)),
            "slowdown_p50": float(np.percentile(slow, 50)), "slowdown_p99": float(np.percentile(slow, 99)),
            "outputs_written": written, "writer_tail_ms": tail_ms,
            "admission": {k: int(info[k]) for k in ("admitted", "completed", "rejected", "failed", "queued_peak",
                                                     "running_peak", "budget_bytes", "peak_used_bytes")}}


def config1_filter(P, dds, device, peak, flush=None):
    """One resident enumeration of a set of config-1 DDs (after the caller's warm-up):
    the tile kernel's and the whole filter's algorithmic bytes over their kernel time."""
    import torch

    r1 = P.ResidentSet(dds, device=device)
    try:
        r1.enumerate(method=1, keep=False)
        st1 = {}
        if flush is not None:
            flush.zero_()
        torch.cuda.synchronize()
        r1.enumerate(method=1, stats=st1, keep=False)
    finally:
        r1.close()
    b1 = (st1["work_tile_candidates_total"] + st1["work_tile_survivors_total"]) * 3 * 4
    a1 = b1 / st1["kernel_expand_td_s"] / 1e9
    bf = (st1["work_candidates_total"] + st1["work_frontier_survivors_total"]) * 3 * 4
    tf = st1["kernel_expand_td_s"] + st1["kernel_dominance_s"]
    af = bf / tf / 1e9
    return {"instances": len(dds), "solves_per_s": len(dds) / st1["device_elapsed_s"],
            "achieved_gbs": a1, "frac_of_peak": a1 / peak,
            "kernel_s": st1["kernel_expand_td_s"], "algorithmic_bytes": int(b1),
            "tile_launches": int(st1["tile_launches"]),
            "filter_achieved_gbs": af, "filter_frac_of_peak": af / peak,
            "filter_kernel_s": tf, "filter_algorithmic_bytes": int(bf),
            "device_s": st1["device_elapsed_s"]}


SINGLE_CASES = {
    "kp3_n40": (1, 3, lambda I: I.knapsack_text(40, 3, 0)),
    "kp4_n60": (1, 4, lambda I: I.knapsack_text(60, 4, 0)),
    "kp7_n25": (1, 7, lambda I: I.knapsack_text(25, 7, 0)),
    "sp3_n100_m20": (2, 3, lambda I: I.setpacking_text(100, 20, 3, 0)),
    "tsp5_n13": (3, 5, lambda I: I.tsp_text(13, 5, 0)),
}


def instance_only(args):
    """`--instance NAME --method M`: one single-instance configuration (seed 0) through
    pmdd_enumerate, `--warmup` untimed runs then `--steps` timed ones; one JSON line with
    the device time and work counters of each timed run.  The command the committed
    single-instance profiles run under ncu."""
    import torch

    import pmdd_b200 as P
    from pmdd_b200 import instances

    torch.cuda.set_device(0)
    ptype, d, make = SINGLE_CASES[args.instance]
    dd = P.DecisionDiagram.from_text(make(instances), ptype, d)
    for _ in range(args.warmup):
        P.enumerate_dd(dd, method=args.method)
    runs = []
    for _ in range(max(1, args.steps)):
        st = {}
        t0 = time.perf_counter()
        pts = P.enumerate_dd(dd, method=args.method, stats=st)
        wall = time.perf_counter() - t0
        runs.append({"device_s": st["device_elapsed_s"], "wall_s": wall, "solutions": int(len(pts)),
                     "chained_layers": int(st["work_chained_layers"]),
                     "candidates": int(st["work_candidates_total"]), "join_products": int(st["work_join_products_total"]),
                     "launches": int(st["gpu_launches"])})
    print(json.dumps({"instance": args.instance, "method": args.method, "runs": runs}))


def config1_only(args):
    """`--config1 N`: the config-1 filter leg alone (N x KP d=3 n=40, seeds 0..N-1,
    method 1), `--warmup` untimed resident enumerations then `--steps` timed ones; one
    JSON line.  This is the command the committed tile-kernel profiles run under ncu."""
    import torch

    import pmdd_b200 as P
    from pmdd_b200 import instances

    torch.cuda.set_device(0)
    peak, peak_kind = read_peaks()
    dds = build_dds([(1, instances.knapsack_text(40, 3, s), "") for s in range(args.config1)])
    res = P.ResidentSet(dds, device=0)
    for _ in range(args.warmup):
        res.enumerate(method=1, keep=False)
    res.close()
    runs = [config1_filter(P, dds, 0, peak) for _ in range(max(1, args.steps))]
    best = max(runs, key=lambda r: r["achieved_gbs"])
    best["peak_gbs"] = peak
    best["peak_kind"] = peak_kind
    best["runs"] = len(runs)
    print(json.dumps({"config1_filter": best}))


# ------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("native", "reference"), default="native")
    ap.add_argument("--quick", action="store_true", help="smaller side measurements (development)")
    ap.add_argument("--no-extras", action="store_true", help="skip one-at-a-time, served, config-1 and CPU legs")
    ap.add_argument("--subset", type=int, default=0,
                    help="profile a subset: every k-th instance of the stream (k = value); not a bench line")
    ap.add_argument("--config1", type=int, default=0,
                    help="only the config-1 filter leg on this many KP d=3 n=40 instances (profiling aid; "
                         "prints its own JSON line, not a bench line)")
    ap.add_argument("--instance", default="",
                    help="only one single-instance configuration (kp3_n40, kp4_n60, kp7_n25, sp3_n100_m20, tsp5_n13) by "
                         "--method, `--warmup` untimed then `--steps` timed runs (profiling aid; own JSON line)")
    ap.add_argument("--method", type=int, default=1)
    ap.add_argument("--served", action="store_true",
                    help="only the served-loop legs (profiling aid; prints its own JSON line, not a bench line)")
    ap.add_argument("--served-rates", default="50,200,800,0",
                    help="with --served: arrival rates in req/s (0: every request at once)")
    ap.add_argument("--served-detail", default="",
                    help="with --served: write every request's tag and served / lone latency to this JSON file")
    args = ap.parse_args()
    if args.config1 > 0:
        config1_only(args)
        return
    if args.instance:
        instance_only(args)
        return
    if args.served:
        import torch

        import pmdd_b200 as P
        from pmdd_b200 import instances

        torch.cuda.set_device(0)
        rates = [int(x) for x in args.served_rates.split(",") if x]
        detail = {}
        legs = []
        for rate in rates:
            detail[str(rate)] = []
            legs.append(served_loop(rate, {50: 100, 200: 200}.get(rate, 400), rate, P, instances, 0, detail[str(rate)]))
        if args.served_detail:
            with open(args.served_detail, "w") as f:
                json.dump(detail, f)
        print(json.dumps({"served": legs}))
        return

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    from pmdd_b200 import instances, replicas

    n_kp, n_sp = 512, 256
    specs = replicas.rank_stream(rank, n_kp, n_sp, 3)
    if args.subset > 1:
        specs = specs[:: args.subset]
    config = {"workload": "batched stream: 512 knapsack BDDs (d=3, n~U{20..60}) + 256 set-packing BDDs "
                          "(d=3, n~U{60..100}, m=20), seeds 0..767, method 1",
              "instances_per_gpu": n_kp + n_sp, "nobjs": 3, "method": 1,
              "l2": "256 MiB buffer written between timed steps",
              "parallelism": f"replicas x{args.gpus} (independent instances per GPU, no collective)"}

    if args.impl == "reference":
        if rank != 0:
            return
        cores = os.cpu_count() or 1
        vals = []
        n_done = 0
        for s in range(args.warmup + args.steps):
            r = cpu_reference_sample(specs, cores, budget_s=10.0, max_items=48)
            if r is None:
                print(json.dumps({"impl": "reference", "unavailable": "reference CPU binary oracle/_ref/multiobj_nobjs3 "
                                                                      "not built (make -C oracle REF=...)"}))
                return
            if s >= args.warmup:
                vals.append(r[0])
                n_done = r[1]
        v = float(np.median(vals))
        sample = f"{n_done} stream instances per step, {cores} concurrent single-threaded reference processes"
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * n_done / v,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
                          "data": "synthetic", "config": config,
                          "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "reference",
                                           "sample": sample},
                          "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    import torch

    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta

        dist = dist_mod
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    device = local
    torch.cuda.set_device(device)

    import pmdd_b200 as P

    lib = P._native.gpu_lib()
    t = time.time()
    dds = build_dds(specs)
    log(f"[rank {rank}] built {len(dds)} DDs in {time.time() - t:.1f}s")
    h2d_bytes = sum(dd_bytes(d) for d in dds)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{device}")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, dist, f"cuda:{device}")

    # ---------------------------------------------- device-resident (value)
    res = P.ResidentSet(dds, device=device)
    sizes = None
    for _ in range(args.warmup):
        sizes = res.enumerate(method=1, keep=False)
    barrier()
    dev_time = 0.0
    k_expand = 0.0
    k_big = 0.0
    k_total = 0.0
    launches = 0
    cand = surv = tile_launches = all_cand = 0
    stats_last = {}
    with ClockSampler(device) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            st = {}
            res.enumerate(method=1, stats=st, keep=False)
            dev_time += st["device_elapsed_s"]
            k_expand += st["kernel_expand_td_s"]
            k_big += st["kernel_dominance_s"]
            k_total += st["kernel_total_s"]
            launches += st["gpu_launches"]
            cand += st["work_tile_candidates_total"]
            surv += st["work_tile_survivors_total"]
            tile_launches += st["tile_launches"]
            all_cand += st["work_candidates_total"]
            stats_last = st
    barrier()
    clocks = clk.summary()
    t_max = max_over_ranks(dev_time)
    n_inst = len(dds)
    value = n_inst * args.steps * world / t_max
    ms_per_step = 1e3 * t_max / args.steps
    res.close()

    # roofline of the fused expand+filter tile kernel: algorithmic bytes of a launch =
    # (candidates it filters, read as parent points + survivors it writes) x d x 4 B;
    # achieved = those bytes / its CUDA-event time (sums over the K timed steps, i.e.
    # per-launch bytes over the average launch duration)
    peak, peak_kind = read_peaks()
    alg_bytes = (cand + surv) * 3 * 4
    achieved = alg_bytes / k_expand / 1e9 if k_expand > 0 else 0.0
    alg_per_launch = alg_bytes / max(1, tile_launches)
    traffic = None
    issue = None
    lex = os.environ.get("PMDD_LEX_TILES", "1") != "0"  # three objectives: the lexicographic tiles
    kname = "expand_tile_lex_kernel" if lex else "expand_tile_kernel"
    tpath = os.path.join(ROOT, "profiles", f"{kname}_stream_traffic.json")
    if os.path.exists(tpath):
        try:
            tj = json.load(open(tpath))
            ratio = tj.get("dram_bytes_per_algorithmic_byte")
            if ratio is not None:
                traffic = ratio * alg_per_launch
            issue = tj.get("issue")
        except Exception:
            traffic = None

    # ---------------------------------------------------------------- e2e
    barrier()
    e2e_wall = 0.0
    d2h = 0
    for s in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        outs = P.enumerate_batch(dds, method=1, device=device)
        t1 = time.perf_counter()
        if s >= args.warmup:
            e2e_wall += t1 - t0
            d2h = sum(o.nbytes for o in outs)
    e2e_max = max_over_ranks(e2e_wall)
    e2e_value = n_inst * args.steps * world / e2e_max

    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generators, reference text formats)",
        "config": config,
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(h2d_bytes),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if peak else None, "traffic": traffic,
                     "kernel": (f"{kname}<int32> (fused expand + lexicographic merge + staircase filter)" if lex
                                else f"{kname}<3,int32> (fused expand + pairwise dominance filter)"),
                     "traffic_source": os.path.relpath(tpath, ROOT) if traffic is not None else None,
                     "peak_kind": peak_kind,
                     "launches": int(tile_launches),
                     "algorithmic_bytes_per_launch": int(alg_per_launch),
                     "avg_launch_s": k_expand / max(1, tile_launches),
                     "tile_candidates_per_step": int(cand / max(1, args.steps)),
                     "all_candidates_per_step": int(all_cand / max(1, args.steps)),
                     "issue": issue},
        "step_breakdown_s": {"device": t_max / args.steps, "tiles": k_expand / args.steps,
                             "oversized": k_big / args.steps, "kernels_total": k_total / args.steps},
    }
    if args.subset > 1:
        line["config"]["subset"] = f"every {args.subset}th instance (profiling run, not a bench line)"

    if rank == 0 and not args.no_extras:
        # one-at-a-time through the C ABI (same stream, e2e style)
        sub = dds if not args.quick else dds[::8]
        t0 = time.perf_counter()
        for d in sub:
            P.enumerate_dd(d, method=1, device=device)
        oat = len(sub) / (time.perf_counter() - t0)
        line["one_at_a_time"] = {"value": oat, "unit": "solves/s", "instances": len(sub),
                                 "batched_e2e_over_one_at_a_time": e2e_value / world / oat}
        # served loop
        served = []
        for rate in (50, 200, 800, 0):
            n_req = {50: 100, 200: 200, 800: 400, 0: 400}[rate] // (4 if args.quick else 1)
            served.append(served_loop(rate, n_req, rate, P, instances, device))
        line["served"] = served
        # config-1 filter roofline: 1024 x KP d=3 n=40
        # (tile kernel alone, and the whole filter: tiles + oversized-destination path)
        n1 = 256 if args.quick else 1024
        dd1 = build_dds([(1, instances.knapsack_text(40, 3, s), "") for s in range(n1)])
        line["config1_filter"] = config1_filter(P, dd1, device, peak, flush)
        del dd1
        # the knapsack half of the stream with DD construction inside the timed region:
        # built on the device from the instance arrays and enumerated from there, against
        # the host constructors (16 threads) + upload + enumeration
        kp_texts = [t for p_, t, _ in specs if p_ == 1]
        kp_arr = [kp_arrays_from_text(t) for t in kp_texts]
        P.ResidentSet.from_knapsack(kp_arr[:2], device=device).close()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rb = P.ResidentSet.from_knapsack(kp_arr, device=device)
        t_build = time.perf_counter() - t0
        n_b = rb.enumerate(method=1, keep=False)
        t_dev = time.perf_counter() - t0
        rb.close()
        t0 = time.perf_counter()
        kdds = build_dds([(1, t, "") for t in kp_texts])
        t_hb = time.perf_counter() - t0
        outs_h = P.enumerate_batch(kdds, method=1, device=device)
        t_host = time.perf_counter() - t0
        del kdds
        line["knapsack_with_construction"] = {
            "instances": len(kp_texts), "unit": "solves/s",
            "device_built": len(kp_texts) / t_dev, "device_build_s": t_build,
            "host_built": len(kp_texts) / t_host, "host_build_s": t_hb, "host_build_threads": 16,
            "same_frontier_sizes": list(n_b) == [len(o) for o in outs_h]}
        # reference CPU baseline on the box's cores
        if world == 1:
            cores = os.cpu_count() or 1
            r = cpu_reference_sample(specs, cores, budget_s=12.0, max_items=48)
            if r is not None and r[0]:
                line["cpu_baseline"] = {"value": r[0], "unit": "solves/s", "cores": cores, "kind": "reference",
                                        "sample": f"{r[1]} stream instances, {cores} concurrent single-threaded "
                                                  f"reference processes (wall_enumeration_s, DD build excluded)"}
        # single large instances, GPU next to the reference CPU path
        line["single_instance"] = single_instances(P, instances, device, with_ref=(world == 1 and not args.quick))
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
