"""Oversized destinations in crowded steps.

A batch of knapsack instances puts more destinations above the tile size into one step
than the GPU holds SFS blocks at once (three per SM).  With the built-in crossover they
all take the GPU-wide pivot/mark pass; with the crossover raised past every destination
they take one SFS block each, started largest first.  Either way the batched frontiers
must equal the lone runs', a sample must match the oracle, and a small --max-cand (passes
over the oversized destinations) must change nothing.  The engine reads the crossover at
start-up, so each setting runs in a child process.
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

CHILD = r"""
import json, sys
sys.path.insert(0, {root!r})
import numpy as np
import oracle
import pmdd_b200 as P
from pmdd_b200 import instances
dds = [P.DecisionDiagram.from_text(instances.knapsack_text(46 + i % 9, 3, 4000 + i), 1, 3) for i in range(160)]
st = {{}}
batch = P.enumerate_batch(dds, method=1, stats=st)
assert st["work_tile_candidates_total"] < st["work_candidates_total"]  # some destinations left the tiles
for i, dd in enumerate(dds):
    lone = P.enumerate_dd(dd, method=1)
    assert np.array_equal(oracle.sorted_set(batch[i]), oracle.sorted_set(lone)), i
for i in (0, 57, 159):
    assert np.array_equal(oracle.sorted_set(batch[i]), oracle.sorted_set(oracle.enumerate(dds[i], 1))), i
capped = P.enumerate_batch(dds[:120], method=1, max_cand=200_000)
for a, b in zip(batch[:120], capped):
    assert np.array_equal(oracle.sorted_set(a), oracle.sorted_set(b))
print(json.dumps({{"launches": st["gpu_launches"]}}))
"""


@pytest.mark.parametrize("mark_min", [None, 1 << 40], ids=["pivot-mark", "sfs-largest-first"])
def test_crowded_steps_match_lone_runs_and_the_oracle(mark_min, tmp_path):
    from conftest import ROOT

    env = dict(os.environ, PMDD_TUNING_FILE=str(tmp_path / "none.json"))
    env.pop("PMDD_BIG_MARK_MIN", None)
    if mark_min is not None:
        env["PMDD_BIG_MARK_MIN"] = str(mark_min)
    p = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT)], env=env, capture_output=True, text=True,
                       timeout=900)
    assert p.returncode == 0, p.stdout + p.stderr
    assert json.loads(p.stdout.strip().splitlines()[-1])["launches"] > 0
