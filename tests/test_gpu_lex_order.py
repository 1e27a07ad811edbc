"""Frontiers in lexicographic (three objectives) and objective-sum (four) order: tile_lex.cu,
big_lex.cu, stair.cuh.

* Knapsack profits with objective 1 + objective 2 the same for every item make the
  (objective 1, objective 2) projections of a frontier an antichain, so the staircase
  grows with every point: n = 18 overflows the tiles' 64 entries, n = 26 also the
  oversized path's 256.  Both fall back to checking every earlier point; the frontiers
  must equal the oracle's.
* Both ends of the pairwise / staircase crossover (PMDD_LEX_PAIR_MAX 0: every
  destination by a staircase warp; 1024: every destination pairwise), the parent runs
  staged by bulk copies or loaded directly (PMDD_LEX_BULK 1 / 0), and the pairwise tile
  kernel (PMDD_LEX_TILES=0) stay exact on the golden fixtures and seeded instances, and
  so do oversized destinations of up to 4096 runs sorted by merge rounds
  (PMDD_BIG_LEX_MAX_ARCS=4096) or none of them on the lexicographic path (0).  Four
  objectives: the pairwise tile kernel (the default) and the tiles in objective-sum order
  (PMDD_SUM_TILES=1; a candidate swept against the points before it) give the golden and
  the oracle's frontiers.  The engine reads these settings at start-up, so each runs
  in a child process.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle
import pmdd_b200 as P
from pmdd_b200 import instances

pytestmark = pytest.mark.gpu


def kp_anti(n, seed, spread=1000):
    rng = np.random.default_rng(seed)
    x = rng.integers(1, spread, size=n)
    p0 = rng.integers(1, 1001, size=n)
    w = rng.integers(1, 1001, size=n)
    lines = [f"{n} 1 3", " ".join(map(str, p0)), " ".join(map(str, x)), " ".join(map(str, spread - x)),
             " ".join(map(str, w)) + f" {int(w.sum()) // 2}"]
    return "\n".join(lines) + "\n"


@pytest.mark.parametrize("n", [18, 22, 26])
def test_staircase_overflow_falls_back_exactly(n):
    dd = P.DecisionDiagram.from_text(kp_anti(n, 3), 1, 3)
    for method in (1, 3):
        st = {}
        got = P.enumerate_dd(dd, method=method, stats=st)
        want = oracle.enumerate(dd, method)
        assert np.array_equal(oracle.sorted_set(got), oracle.sorted_set(want)), method
        assert len(np.unique(got, axis=0)) == len(got)
        if n == 26 and method == 1:
            assert st["work_candidates_peak"] > 1024  # oversized destinations took part


CHILD = r"""
import json, sys
sys.path.insert(0, {root!r})
sys.path.insert(0, {tests!r})
import numpy as np
import oracle
import pmdd_b200 as P
from pmdd_b200 import instances
from conftest import golden_cases, golden_frontier
n = 0
for rec in golden_cases():
    if rec["nobjs"] not in (3, 4):
        continue
    dd = P.DecisionDiagram.from_file(rec["dat"], rec["problem_type"], rec["nobjs"])
    for m in rec["methods"]:
        got = P.enumerate_dd(dd, method=int(m))
        assert np.array_equal(oracle.sorted_set(got), oracle.sorted_set(golden_frontier(rec, int(m)))), (rec["name"], m)
        n += 1
for text, pt, d in ((instances.knapsack_text(46, 3, 31), 1, 3), (instances.setpacking_text(90, 20, 3, 32), 2, 3),
                    (instances.tsp_text(11, 3, 33), 3, 3), (instances.knapsack_text(36, 4, 34), 1, 4),
                    (instances.setpacking_text(80, 20, 4, 35), 2, 4), (instances.tsp_text(10, 4, 36), 3, 4)):
    dd = P.DecisionDiagram.from_text(text, pt, d)
    for m in (1, 3):
        got = P.enumerate_dd(dd, method=m)
        assert np.array_equal(oracle.sorted_set(got), oracle.sorted_set(oracle.enumerate(dd, m))), (pt, m)
        n += 1
print(json.dumps({{"checked": n}}))
"""


@pytest.mark.parametrize("env", [{"PMDD_LEX_PAIR_MAX": "0"}, {"PMDD_LEX_PAIR_MAX": "1024"}, {"PMDD_LEX_TILES": "0"},
                                 {"PMDD_LEX_BULK": "1"}, {"PMDD_LEX_BULK": "0"}, {"PMDD_BIG_LEX_MAX_ARCS": "4096"},
                                 {"PMDD_BIG_LEX_MAX_ARCS": "0"}, {"PMDD_SUM_TILES": "1"}],
                         ids=["all-staircase", "all-pairwise", "pairwise-kernel", "bulk-staging", "direct-loads",
                              "merge-rounds", "no-oversized-lex", "four-objective-sum-order"])
def test_filter_paths_stay_exact(env):
    from conftest import ROOT

    e = dict(os.environ)
    for k in ("PMDD_LEX_PAIR_MAX", "PMDD_LEX_TILES", "PMDD_LEX_BULK", "PMDD_BIG_LEX_MAX_ARCS", "PMDD_SUM_TILES"):
        e.pop(k, None)
    e.update(env)
    p = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT, tests=os.path.join(ROOT, "tests"))], env=e,
                       capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stdout + p.stderr
    assert json.loads(p.stdout.strip().splitlines()[-1])["checked"] > 20
