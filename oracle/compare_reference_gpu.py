"""Context timings: the reference's own GPU path next to this engine, on one B200.

Runs, for each instance and method, the drop-in binary pmdd_b200/bin/multiobj_nobjs<N>
and the reference built with its GPU path (`make -C oracle ref-gpu`, binaries
oracle/_ref/multiobj_nobjs<N>_gpu), both with `--backend gpu --stats-out`, and prints a
markdown table of solution counts and `wall_enumeration_s` (DD construction excluded)
from each stats record.  Test infrastructure: nothing here is part of the engine, and the
reference is only timed, never used to check.

    python oracle/compare_reference_gpu.py [--timeout 300] [--only kp3_n40,...]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, ".."))
sys.path.insert(0, ROOT)

from pmdd_b200 import instances  # noqa: E402

KNOWN = os.path.join(ROOT, "tests", "golden", "known_counts")


def cases():
    out = [
        ("kp3_n40", 1, 3, instances.knapsack_text(40, 3, 0), (1, 3)),
        ("kp4_n60", 1, 4, instances.knapsack_text(60, 4, 0), (1, 3)),
        ("kp7_n25", 1, 7, instances.knapsack_text(25, 7, 0), (1, 3)),
        ("sp3_n100_m20", 2, 3, instances.setpacking_text(100, 20, 3, 0), (1, 3)),
        ("tsp3_n13", 3, 3, instances.tsp_text(13, 3, 0), (1, 3)),
    ]
    for seed in ("30131", "11093"):
        with open(os.path.join(KNOWN, f"tsp-nobj5-ncities15-seed{seed}.dat")) as f:
            out.append((f"tsp5_n15_seed{seed}", 3, 5, f.read(), (1,)))
    return out


def run(binary, path, ptype, method, timeout):
    with tempfile.TemporaryDirectory() as td:
        sp = os.path.join(td, "s.jsonl")
        cmd = [binary, path, str(ptype), str(method), "0", "--backend", "gpu", "--stats-out", sp]
        t0 = time.perf_counter()
        try:
            p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        except subprocess.TimeoutExpired:
            return {"status": f"timeout {timeout}s"}
        wall = time.perf_counter() - t0
        if p.returncode != 0:
            tail = (p.stdout + p.stderr).strip().splitlines()
            return {"status": "failed: " + (tail[-1][:80] if tail else f"rc {p.returncode}")}
        rec = json.loads(open(sp).read().strip().splitlines()[-1])
        return {"status": "ok", "solutions": rec["outputs"]["num_solutions"],
                "enum_s": rec["timing"]["wall"]["wall_enumeration_s"],
                "kernel_s": rec["timing"]["kernel"]["kernel_total_s"], "process_s": wall}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--timeout", type=float, default=300.0)
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    only = set(filter(None, args.only.split(",")))
    tmp = tempfile.mkdtemp()
    print("| instance | method | solutions (this / reference) | enum s, this / reference | ratio "
          "| kernel s, this / reference | ratio | process s, this / reference |")
    print("|---|---:|---|---|---:|---|---:|---|")
    for name, ptype, d, text, methods in cases():
        if only and name not in only:
            continue
        path = os.path.join(tmp, name + ".dat")
        with open(path, "w") as f:
            f.write(text)
        mine_bin = os.path.join(ROOT, "pmdd_b200", "bin", f"multiobj_nobjs{d}")
        ref_bin = os.path.join(HERE, "_ref", f"multiobj_nobjs{d}_gpu")
        for m in methods:
            a = run(mine_bin, path, ptype, m, args.timeout)
            b = run(ref_bin, path, ptype, m, args.timeout) if os.path.exists(ref_bin) else {"status": "not built"}
            sols = f"{a.get('solutions', a['status'])} / {b.get('solutions', b['status'])}"
            both = a["status"] == b["status"] == "ok"

            def pair(key):
                fa = f"{a[key]:.4f}" if a["status"] == "ok" else a["status"]
                fb = f"{b[key]:.4f}" if b["status"] == "ok" else b["status"]
                r = f"{b[key] / a[key]:.1f}x" if both and a[key] > 0 else ""
                return f"{fa} / {fb}", r

            e, er = pair("enum_s")
            k, kr = pair("kernel_s")
            pw, _ = pair("process_s")
            print(f"| {name} | {m} | {sols} | {e} | {er} | {k} | {kr} | {pw} |", flush=True)


if __name__ == "__main__":
    main()
