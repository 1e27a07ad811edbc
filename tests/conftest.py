import glob
import json
import os
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden_cases():
    out = []
    for path in sorted(glob.glob(os.path.join(GOLDEN, "*.json"))):
        with open(path) as f:
            rec = json.load(f)
        rec["dat"] = path[:-5] + ".dat"
        out.append(rec)
    return out


def golden_frontier(rec, method):
    import numpy as np

    path = os.path.join(GOLDEN, f"{rec['name']}.m{method}.csv")
    rows = []
    with open(path) as f:
        for line in f:
            if line.strip():
                rows.append([int(x) for x in line.split(",")])
    return np.array(rows, dtype=np.int64).reshape(-1, rec["nobjs"])


@pytest.fixture(scope="session")
def golden():
    return golden_cases()
