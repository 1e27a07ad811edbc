"""Known answers held by the reference: the Pareto-frontier sizes of the ten 5-objective
15-city TSP instances (kb/autoresearch/TSP_STATUS.md:26-37 of the reference, from its own
GPU top-down and CPU coupled runs).  Run through the drop-in binary with method 1.
"""
import json
import os
import subprocess

import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

KC = os.path.join(GOLDEN, "known_counts")
COUNTS = json.load(open(os.path.join(KC, "counts.json")))


@pytest.mark.parametrize("name", sorted(COUNTS), ids=lambda n: n.replace(".dat", ""))
def test_tsp15_5obj_frontier_size(name):
    binary = os.path.join(ROOT, "pmdd_b200", "bin", "multiobj_nobjs5")
    p = subprocess.run([binary, os.path.join(KC, name), "3", "1", "0", "--backend", "gpu"], capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert int(p.stdout.splitlines()[0]) == COUNTS[name]
