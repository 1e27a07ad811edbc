"""Layer chaining (chain.cu): small steps expand several layers per host read-back.

Each setting runs in a child process (the engine reads PMDD_CHAIN_LAYERS and
PMDD_CHAIN_MAX_CAND at start-up): chaining off, the default (chains of 8 layers at first
for expansions of at most 2^17 candidates, growing while a request runs alone), chains
starting at one layer, and 64 layers for expansions of any size, growing in batches too
-- the last makes requests stop their chains at oversized destinations and at full
frontier buffers.  A chain's later layers are sized and planned by the count kernel of
the layer before (count.cu), the first by chain_prep_kernel and tile_plan_kernel.  In
every setting the frontiers of the golden fixtures equal the reference's, and those of
seeded knapsack (3, 4 and 7 objectives), set-packing and TSP instances, alone and in
mixed batches of two objective counts, equal the oracle's; the chained settings report
chained layers, chaining off reports none.  Method 3 chains a side only while the side
rule would pick it again and stops a layer short of the other side, so its frontiers
equal the oracle's and its cutset layer and per-side layer counts equal those of the run
without chaining.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle
import pmdd_b200 as P
from conftest import ROOT, frontier_digest
from pmdd_b200 import instances

pytestmark = pytest.mark.gpu

SINGLE = [(1, "kp", 40, 3, 11), (1, "kp", 30, 4, 12), (1, "kp", 22, 7, 13), (2, "sp", 100, 3, 14),
          (2, "sp", 70, 4, 15), (3, "tsp", 10, 3, 16)]
BATCH = [(1, "kp", 20 + 2 * i, 3 + i % 2, 100 + i) for i in range(12)]


def _text(kind, n, d, seed):
    if kind == "kp":
        return instances.knapsack_text(n, d, seed)
    if kind == "sp":
        return instances.setpacking_text(n, 20, d, seed)
    return instances.tsp_text(n, d, seed)


CHILD = r"""
import json, sys
sys.path.insert(0, {root!r})
sys.path.insert(0, {tests!r})
import numpy as np
import oracle
import pmdd_b200 as P
from conftest import golden_cases, golden_frontier, frontier_digest
from test_gpu_chain import SINGLE, BATCH, _text
out = {{"golden": 0, "single": [], "batch": [], "chained": 0, "m3": [], "m3_shape": []}}
for rec in golden_cases():
    dd = P.DecisionDiagram.from_file(rec["dat"], rec["problem_type"], rec["nobjs"])
    for m in rec["methods"]:
        st = {{}}
        got = P.enumerate_dd(dd, method=int(m), stats=st)
        assert np.array_equal(oracle.sorted_set(got), oracle.sorted_set(golden_frontier(rec, int(m)))), (rec["name"], m)
        out["chained"] += st["work_chained_layers"]
        out["golden"] += 1
for pt, kind, n, d, seed in SINGLE:
    dd = P.DecisionDiagram.from_text(_text(kind, n, d, seed), pt, d)
    st = {{}}
    got = P.enumerate_dd(dd, method=1, stats=st)
    out["single"].append(frontier_digest(got))
    out["chained"] += st["work_chained_layers"]
    st = {{}}
    got = P.enumerate_dd(dd, method=3, stats=st)
    out["m3"].append(frontier_digest(got))
    out["m3_shape"].append([st["layer_coupling"], st["layers_td"], st["layers_bu"]])
    out["chained"] += st["work_chained_layers"]
dds = [P.DecisionDiagram.from_text(_text(kind, n, d, seed), pt, d) for pt, kind, n, d, seed in BATCH]
st = {{}}
for got in P.enumerate_batch(dds, method=1, stats=st):
    out["batch"].append(frontier_digest(got))
out["chained"] += st["work_chained_layers"]
print(json.dumps(out))
"""


def _run(env):
    e = dict(os.environ)
    for k in ("PMDD_CHAIN_LAYERS", "PMDD_CHAIN_MAX_CAND", "PMDD_CHAIN_GROW", "PMDD_CHAIN_MAX_REQUESTS"):
        e.pop(k, None)
    e.update(env)
    p = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT, tests=os.path.join(ROOT, "tests"))], env=e,
                       capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stdout + p.stderr
    return json.loads(p.stdout.strip().splitlines()[-1])


@pytest.fixture(scope="module")
def want():
    single = [frontier_digest(oracle.enumerate(P.DecisionDiagram.from_text(_text(k, n, d, s), pt, d), 1))
              for pt, k, n, d, s in SINGLE]
    batch = [frontier_digest(oracle.enumerate(P.DecisionDiagram.from_text(_text(k, n, d, s), pt, d), 1))
             for pt, k, n, d, s in BATCH]
    m3 = [frontier_digest(oracle.enumerate(P.DecisionDiagram.from_text(_text(k, n, d, s), pt, d), 3))
          for pt, k, n, d, s in SINGLE]
    return single, batch, m3


@pytest.fixture(scope="module")
def unchained():
    return _run({"PMDD_CHAIN_LAYERS": "0"})


@pytest.mark.parametrize("env,chained", [({"PMDD_CHAIN_LAYERS": "0"}, False), ({}, True),
                                         ({"PMDD_CHAIN_LAYERS": "1"}, True),
                                         ({"PMDD_CHAIN_LAYERS": "64", "PMDD_CHAIN_MAX_CAND": str(1 << 40),
                                           "PMDD_CHAIN_GROW": "all"}, True)],
                         ids=["off", "default", "one-layer", "long-chains"])
def test_chained_steps_give_the_same_frontiers(env, chained, want, unchained):
    got = _run(env)
    assert got["golden"] > 10
    assert got["single"] == want[0]
    assert got["batch"] == want[1]
    assert got["m3"] == want[2]
    assert got["m3_shape"] == unchained["m3_shape"]
    assert (got["chained"] > 0) == chained
