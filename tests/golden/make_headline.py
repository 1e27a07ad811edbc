"""Regenerates tests/golden/headline/ -- reference results for the workloads the
throughput claims are measured on -- from the reference's own CPU binary.

    make -C oracle REF=/path/to/PMDD            # builds oracle/_ref/multiobj_nobjs{3,4}
    python tests/golden/make_headline.py

Writes
    kp4_n60_s0.m1.csv.gz, kp4_n60_s0.m3.csv.gz
                  the 4-objective knapsack n=60 (seed 0) frontier of methods 1 and 3,
                  sorted ascending, in the reference's CSV text (gzip'd)
    stream.json   for each of the 768 instances of the batched stream (512 knapsack
                  d=3 n~U{20..60} + 256 set packing d=3 n~U{60..100}, seeds 0..767,
                  method 1): its tag, solution count and the SHA-256 of its sorted
                  frontier CSV text
    served.json   the same for the served-loop request lists (instances.served_mix with
                  seeds 50 / 200 / 800 and 100 / 200 / 400 requests; knapsack and set
                  packing by method 1, TSP by method 3)
The frontier text is the reference's --frontier-out format (util/output_utils.cpp:
87-152): one point per line, objectives as %d separated by commas, rows in ascending
lexicographic order (enum/pareto_frontier.hpp:418-433).
"""
from __future__ import annotations

import concurrent.futures as cf
import gzip
import hashlib
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
OUT = os.path.join(HERE, "headline")
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from pmdd_b200 import instances  # noqa: E402

SERVED_LISTS = ((50, 100), (200, 200), (800, 400))


def frontier_text(points) -> str:
    pts = oracle.sorted_set(points)
    return "".join(",".join(str(int(x)) for x in row) + "\n" for row in pts)


def digest(points) -> str:
    return hashlib.sha256(frontier_text(points).encode()).hexdigest()


def run_one(args):
    tag, ptype, method, nobjs, text = args
    with tempfile.NamedTemporaryFile("w", suffix=".dat", delete=False) as f:
        f.write(text)
        path = f.name
    try:
        r = oracle.run_ref(path, ptype, method, nobjs, threads=1)
    finally:
        os.unlink(path)
    return {"tag": tag, "problem_type": ptype, "method": method, "num_solutions": int(len(r["frontier"])),
            "sha256": digest(r["frontier"])}


def run_all(jobs, workers):
    with cf.ThreadPoolExecutor(workers) as ex:
        return list(ex.map(run_one, jobs))


def main():
    os.makedirs(OUT, exist_ok=True)
    workers = os.cpu_count() or 1
    # 4-objective knapsack n=60, methods 1 and 3: full frontiers
    text = instances.knapsack_text(60, 4, 0)
    with tempfile.NamedTemporaryFile("w", suffix=".dat", delete=False) as f:
        f.write(text)
        path = f.name
    for m in (1, 3):
        r = oracle.run_ref(path, 1, m, 4, threads=workers)
        with gzip.open(os.path.join(OUT, f"kp4_n60_s0.m{m}.csv.gz"), "wt") as g:
            g.write(frontier_text(r["frontier"]))
        print("kp4_n60_s0 method", m, len(r["frontier"]))
    os.unlink(path)
    # the batched stream
    jobs = [(tag, pt, 1, 3, t) for pt, t, tag in instances.stream_mix(512, 256, 3, seed0=0)]
    res = run_all(jobs, workers)
    with open(os.path.join(OUT, "stream.json"), "w") as f:
        json.dump({"workload": "stream_mix(512, 256, 3, seed0=0), method 1", "instances": res}, f, indent=0)
    print("stream", len(res))
    # the served lists
    lists = {}
    for seed, n_req in SERVED_LISTS:
        jobs = [(tag, pt, m, 3, t) for pt, t, m, tag in instances.served_mix(n_req, seed)]
        lists[str(seed)] = {"requests": n_req, "results": run_all(jobs, workers)}
        print("served", seed, n_req)
    with open(os.path.join(OUT, "served.json"), "w") as f:
        json.dump({"workload": "served_mix(n_req, seed)", "lists": lists}, f, indent=0)


if __name__ == "__main__":
    main()
