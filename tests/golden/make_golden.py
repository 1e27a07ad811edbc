"""Regenerates the golden fixtures in tests/golden/ from the reference's own CPU binary.

Run in a checkout where the reference sources are available (the fixtures are
committed, so the tests never need them):

    make -C oracle REF=/path/to/PMDD            # builds oracle/_ref/multiobj_nobjs{3..7}
    python tests/golden/make_golden.py /path/to/PMDD

For every fixture instance this writes
    <name>.dat           the instance (reference text format)
    <name>.json          the reference run's structure stats and solution counts, and for
                         knapsack and set packing the counters of the reference's CPU
                         enumeration run on this project's DD numbering ("same_numbering",
                         methods 1 and 3 with and without state dominance; needs
                         `make -C oracle harness`)
    <name>.m<k>.csv      the reference frontier for method k, sorted ascending
Instances are seeded synthetic ones from pmdd_b200.instances plus a few files of
the reference's own data/ directory (named ref_*).  The 5-objective 15-city TSP files
in known_counts/ are copied verbatim; their solution counts come from the reference's
published notes (kb/autoresearch/TSP_STATUS.md:26-37, kb/GPU_NOTES.md:25-28).
"""
from __future__ import annotations

import json
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from pmdd_b200 import instances  # noqa: E402

SYNTHETIC = [
    # name, problem_type, nobjs, text, methods
    ("kp3_n10_s0", 1, 3, instances.knapsack_text(10, 3, 0), (1, 3)),
    ("kp3_n20_s1", 1, 3, instances.knapsack_text(20, 3, 1), (1, 3)),
    ("kp3_n30_s2", 1, 3, instances.knapsack_text(30, 3, 2), (1, 3)),
    ("kp3_n40_s0", 1, 3, instances.knapsack_text(40, 3, 0), (1, 3)),
    ("kp4_n20_s3", 1, 4, instances.knapsack_text(20, 4, 3), (1, 3)),
    ("kp4_n30_s4", 1, 4, instances.knapsack_text(30, 4, 4), (1, 3)),
    ("kp7_n12_s5", 1, 7, instances.knapsack_text(12, 7, 5), (1, 3)),
    ("kp7_n25_s0", 1, 7, instances.knapsack_text(25, 7, 0), (1, 3)),
    ("kp5_n18_s6", 1, 5, instances.knapsack_text(18, 5, 6), (1, 3)),
    ("sp3_n30_s0", 2, 3, instances.setpacking_text(30, 20, 3, 0), (1, 3)),
    ("sp3_n60_s1", 2, 3, instances.setpacking_text(60, 20, 3, 1), (1, 3)),
    ("sp3_n100_s0", 2, 3, instances.setpacking_text(100, 20, 3, 0), (1, 3)),
    ("sp4_n40_s2", 2, 4, instances.setpacking_text(40, 10, 4, 2), (1, 3)),
    ("tsp3_n6_s0", 3, 3, instances.tsp_text(6, 3, 0), (1, 3)),
    ("tsp3_n8_s1", 3, 3, instances.tsp_text(8, 3, 1), (1, 3)),
    ("tsp3_n10_s2", 3, 3, instances.tsp_text(10, 3, 2), (1, 3)),
    ("tsp3_n13_s0", 3, 3, instances.tsp_text(13, 3, 0), (3,)),
    ("tsp4_n9_s3", 3, 4, instances.tsp_text(9, 4, 3), (1, 3)),
]

REFERENCE_FILES = [
    # name, path under the reference checkout, problem_type, nobjs, methods
    ("ref_kp3_n10_ins1", "data/3/knapsack/KP_p-3_n-10_ins-1.dat", 1, 3, (1, 3)),
    ("ref_kp3_n20_ins1", "data/3/knapsack/KP_p-3_n-20_ins-1.dat", 1, 3, (1, 3)),
    ("ref_kp3_n30_ins1", "data/3/knapsack/KP_p-3_n-30_ins-1.dat", 1, 3, (1, 3)),
    ("ref_kp4_n20_ins1", "data/4/knapsack/KP_p-4_n-20_ins-1.dat", 1, 4, (1, 3)),
    ("ref_bp3_n100", "data/3/binproblem/bp-100-20-3-10-10192.dat", 2, 3, (1, 3)),
    ("ref_tsp3_n10", "data/3/tsp/tsp-nobj3-ncities10-seed12870.dat", 3, 3, (1, 3)),
    ("ref_tsp5_n10", "data/5/tsp/tsp-nobj5-ncities10-seed15800.dat", 3, 5, (1, 3)),
]

KNOWN_COUNTS = {
    "tsp-nobj5-ncities15-seed1081.dat": 55198,
    "tsp-nobj5-ncities15-seed11093.dat": 29505,
    "tsp-nobj5-ncities15-seed13095.dat": 117171,
    "tsp-nobj5-ncities15-seed14792.dat": 77303,
    "tsp-nobj5-ncities15-seed23138.dat": 51306,
    "tsp-nobj5-ncities15-seed24645.dat": 38883,
    "tsp-nobj5-ncities15-seed30131.dat": 24381,
    "tsp-nobj5-ncities15-seed32239.dat": 78849,
    "tsp-nobj5-ncities15-seed6440.dat": 32237,
    "tsp-nobj5-ncities15-seed7702.dat": 53917,
}


def record(name, path, problem_type, nobjs, methods):
    out = {"name": name, "problem_type": problem_type, "nobjs": nobjs, "methods": {}}
    for m in methods:
        r = oracle.run_ref(path, problem_type, m, nobjs, threads=1)
        pts = oracle.sorted_set(r["frontier"])
        with open(os.path.join(HERE, f"{name}.m{m}.csv"), "w") as f:
            for row in pts:
                f.write(",".join(str(int(x)) for x in row) + "\n")
        s = r["stats"]
        out["methods"][str(m)] = {
            "num_solutions": s["outputs"]["num_solutions"],
            "layer_coupling": s["structure"]["layer_coupling"],
            "work_candidates_total": s["work"]["work_candidates_total"],
            "work_join_products_total": s["work"]["work_join_products_total"],
            "stdout_first_line": r["stdout"][0],
        }
        st = s["structure"]
        out["structure"] = {k: st[k] for k in ("original_width", "reduced_width", "original_num_nodes",
                                              "reduced_num_nodes", "max_num_nodes_per_layer", "max_num_in_arcs",
                                              "total_num_in_arcs")}
    if problem_type == 1 and 1 in methods:
        # knapsack state dominance (method 1, state_dominance 1): same frontier, fewer labels
        r = oracle.run_ref(path, problem_type, 1, nobjs, threads=1, state_dominance=1)
        s = r["stats"]
        out["state_dominance_1"] = {
            "num_solutions": s["outputs"]["num_solutions"],
            "work_candidates_total": s["work"]["work_candidates_total"],
            "work_frontier_survivors_total": s["work"]["work_frontier_survivors_total"],
            "dominance_filtered_total": s["dominance"]["dominance_filtered_total"],
        }
    if problem_type in (1, 2) and oracle.have_harness(nobjs):
        # the reference's CPU enumeration on this project's DD numbering (oracle/ref_harness.cpp):
        # counters of methods 1 and 3 with and without state dominance, comparable one to one
        from pmdd_b200 import DecisionDiagram

        dd = DecisionDiagram.from_file(path, problem_type, nobjs)
        runs = {}
        for m in (1, 3):
            for sd in (0, 1):
                r = oracle.run_harness(dd, problem_type, m, sd)
                ref_m = str(m) if str(m) in out["methods"] else None
                if ref_m is not None:
                    assert oracle.sorted_set(r["frontier"]).tolist() == oracle.sorted_set(
                        oracle.run_ref(path, problem_type, m, nobjs)["frontier"]).tolist()
                runs[f"m{m}_sd{sd}"] = r["stats"]
        out["same_numbering"] = runs
    with open(os.path.join(HERE, f"{name}.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(name, {m: out["methods"][m]["num_solutions"] for m in out["methods"]})


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ["PMDD_REFERENCE_DIR"]
    for name, pt, d, text, methods in SYNTHETIC:
        path = os.path.join(HERE, f"{name}.dat")
        with open(path, "w") as f:
            f.write(text)
        record(name, path, pt, d, methods)
    for name, rel, pt, d, methods in REFERENCE_FILES:
        path = os.path.join(HERE, f"{name}.dat")
        shutil.copyfile(os.path.join(ref_root, rel), path)
        record(name, path, pt, d, methods)
    kc = os.path.join(HERE, "known_counts")
    os.makedirs(kc, exist_ok=True)
    for fname in KNOWN_COUNTS:
        shutil.copyfile(os.path.join(ref_root, "data", "5", "tsp", fname), os.path.join(kc, fname))
    with open(os.path.join(kc, "counts.json"), "w") as f:
        json.dump(KNOWN_COUNTS, f, indent=1)


if __name__ == "__main__":
    main()
