"""The drop-in command line (pmdd_b200/bin/multiobj_nobjs<N>).

Argument handling mirrors the reference parser (src/pmdd/util/cli_parser.cpp:181-488):
the CPU tests pin every rejection message below, and, where the reference binary was
compiled into oracle/_ref, also compare message and exit code with it directly.  The GPU
tests run the binary on the golden instances and check the three stdout lines
(src/pmdd/util/output_utils.cpp:302-374), the gzip'd frontier CSV (output_utils.cpp:87-152)
and the stats JSONL record (output_utils.cpp:154-300) against the golden records.
"""
import gzip
import json
import os
import subprocess

import pytest

from conftest import GOLDEN, ROOT, golden_cases, golden_frontier

BIN = os.path.join(ROOT, "pmdd_b200", "bin")
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
KP = os.path.join(GOLDEN, "kp3_n10_s0.dat")

# (arguments after the input path, first stdout line) -- reference messages verbatim.
REJECTIONS = [
    (["5", "1", "0"], "Error - invalid problem type '5'. Valid problem types are 1 (knapsack), 2 (set packing), 3 (TSP)."),
    (["0", "1", "0"], "Error - invalid problem type '0'. Valid problem types are 1 (knapsack), 2 (set packing), 3 (TSP)."),
    (["1", "1", "0", "--backend", "gpu", "--cpu-threads", "2"], "Error - cpu thread options are not valid with backend=gpu."),
    (["1", "1", "0", "--max-cand", "12Q", "--backend", "gpu"],
     "Error - invalid --max-cand value '12Q' (expected positive integer with optional K, M, or B suffix)."),
    (["1", "1", "0", "--max-prod", "0", "--backend", "gpu"],
     "Error - invalid --max-prod value '0' (expected positive integer with optional K, M, or B suffix)."),
    (["1", "1", "0", "--max-cand", "5", "--max-cand", "6", "--backend", "gpu"],
     "Error - GPU candidate batch cap provided multiple times."),
    (["1", "1", "0", "--max-cand", "5M"], "Error - --max-cand is only valid with backend=gpu."),
    (["1", "1", "0", "gpu", "4"], "Error - gpu shorthand does not accept a kernel value; use 'gpu'."),
    (["1", "1", "0", "cpu", "0"], "Error - invalid cpu shorthand thread count '0' (expected positive integer)."),
    (["1", "1", "0", "7"], "Error - positional numeric argument '7' must immediately follow shorthand backend token cpu|gpu."),
    (["1", "1", "0", "--foo"], "Error - unrecognized optional argument '--foo'."),
    (["1", "1", "0", "--backend", "cuda"], "Error - backend token 'cuda' is unsupported; use 'gpu'."),
    (["1", "1", "0", "cuda"], "Error - backend token 'cuda' is unsupported; use 'gpu'."),
    (["1", "1", "0", "--backend", "gpu", "gpu"], "Error - cannot mix shorthand backend token with --backend."),
    (["1", "1", "0", "gpu", "--backend", "gpu"], "Error - cannot mix --backend with shorthand backend token."),
    (["1", "1", "0", "--backend"], "Error - --backend requires a value (cpu or gpu)."),
    (["1", "2", "0", "--backend", "gpu"], "Error - GPU backend is unsupported for method 2."),
    (["1", "1", "0", "--frontier-out"], "Error - --frontier-out requires a file path."),
    (["1", "1", "0", "--stats-out", ""], "Error - --stats-out path cannot be empty."),
    (["1", "1", "0", "--cpu-threads", "x"], "Error - invalid --cpu-threads value 'x' (expected positive integer)."),
]


@pytest.fixture(scope="module")
def cli():
    path = os.path.join(BIN, "multiobj_nobjs3")
    if not os.path.exists(path):
        subprocess.run(["make", "-C", os.path.join(ROOT, "pmdd_b200"), "cli"], check=True, capture_output=True)
    assert os.path.exists(path), "multiobj_nobjs3 not built"
    return BIN


def run(binary, args, cwd=None):
    p = subprocess.run([binary] + args, capture_output=True, text=True, timeout=300, cwd=cwd)
    return p.returncode, p.stdout, p.stderr


@pytest.mark.parametrize("args,message", REJECTIONS, ids=[" ".join(a) for a, _ in REJECTIONS])
def test_rejections_match_reference_messages(cli, args, message):
    rc, out, _ = run(os.path.join(cli, "multiobj_nobjs3"), [KP] + args)
    assert rc == 1
    assert out.splitlines()[0] == message
    ref = os.path.join(REF_BIN, "multiobj_nobjs3")
    if os.path.exists(ref):
        rrc, rout, _ = run(ref, [KP] + args)
        assert (rrc, rout.splitlines()[0]) == (rc, message)


def test_missing_input_and_short_argv(cli):
    rc, out, _ = run(os.path.join(cli, "multiobj_nobjs3"), ["/nonexistent.dat", "1", "1", "0", "--backend", "gpu"])
    assert rc == 1 and out.splitlines()[0] == "Error - file /nonexistent.dat could not be found"
    rc, out, _ = run(os.path.join(cli, "multiobj_nobjs3"), [KP, "1", "1"])
    assert rc == 1 and "Usage: multiobj_nobjs<NUM_OBJS>" in out


def test_cpu_backend_is_rejected_loudly(cli):
    rc, out, _ = run(os.path.join(cli, "multiobj_nobjs3"), [KP, "1", "1", "0"])
    assert rc == 1 and "use --backend gpu" in out


def test_nobjs_links_present(cli):
    for k in range(1, 9):
        assert os.path.exists(os.path.join(cli, f"multiobj_nobjs{k}"))


CASES = [(rec, m) for rec in golden_cases() for m in (1, 3) if str(m) in rec["methods"]]


@pytest.mark.gpu
@pytest.mark.parametrize("rec,method", CASES, ids=[f"{r['name']}-m{m}" for r, m in CASES])
def test_cli_outputs_match_golden(cli, tmp_path, rec, method):
    import numpy as np

    binary = os.path.join(cli, f"multiobj_nobjs{rec['nobjs']}")
    fr = tmp_path / "f.csv.gz"
    st = tmp_path / "s.jsonl"
    rc, out, err = run(binary, [rec["dat"], str(rec["problem_type"]), str(method), "0", "--backend", "gpu",
                                "--frontier-out", str(fr), "--stats-out", str(st)])
    assert rc == 0, out + err
    g = rec["methods"][str(method)]
    lines = out.splitlines()
    assert len(lines) == 3
    assert lines[0] == g["stdout_first_line"]
    float(lines[1])
    third = lines[2].split("\t")
    if rec["problem_type"] == 3:
        assert len(third) == 4
    else:
        s = rec["structure"]
        assert len(third) == 13
        assert [int(x) for x in third[:6]] == [method, 0, s["original_width"], s["reduced_width"],
                                              s["original_num_nodes"], s["reduced_num_nodes"]]
        layers = len(s["max_num_nodes_per_layer"])
        assert int(third[8]) == 0 if method == 1 else 0 <= int(third[8]) < layers
    with gzip.open(fr, "rt") as f:
        text = f.read()
    rows = [[int(x) for x in line.split(",")] for line in text.splitlines() if line]
    got = np.array(rows, dtype=np.int64).reshape(-1, rec["nobjs"])
    want = golden_frontier(rec, method)
    np.testing.assert_array_equal(got, want)
    assert [tuple(r) for r in rows] == sorted(tuple(r) for r in rows)
    with open(st) as f:
        recs = [json.loads(line) for line in f if line.strip()]
    assert len(recs) == 1
    j = recs[0]
    assert j["schema_version"] == 1
    assert j["identity"]["backend"] == "gpu" and j["identity"]["method"] == method
    assert j["outputs"]["num_solutions"] == g["num_solutions"]
    assert j["outputs"]["frontier_out_path"] == str(fr)
    if rec["problem_type"] != 3:
        assert j["structure"]["layer_coupling"] == int(third[8])
    if method == 1 or j["structure"]["layer_coupling"] == g["layer_coupling"]:
        # method 3 picks its cutset by the GPU rule; the golden run is the CPU's, so the
        # volumes agree when the two rules pick the same layer
        assert j["work"]["work_candidates_total"] == g["work_candidates_total"]
        assert j["work"]["work_join_products_total"] == g["work_join_products_total"]
    if "structure" in rec and rec["problem_type"] != 3:
        assert j["structure"]["max_num_nodes_per_layer"] == rec["structure"]["max_num_nodes_per_layer"]


@pytest.mark.gpu
def test_cli_default_output_names(cli, tmp_path):
    """--save-frontier / --save-stats write <input stem>.frontier.csv.gz / .stats.jsonl in the cwd."""
    rc, out, err = run(os.path.join(cli, "multiobj_nobjs3"),
                       [KP, "1", "3", "0", "--backend", "gpu", "--save-frontier", "--save-stats"], cwd=tmp_path)
    assert rc == 0, out + err
    assert (tmp_path / "kp3_n10_s0.frontier.csv.gz").exists()
    assert (tmp_path / "kp3_n10_s0.stats.jsonl").exists()
