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


HEADLINE = os.path.join(GOLDEN, "headline")


def frontier_text(points) -> str:
    """A frontier in the reference's --frontier-out text: rows in ascending
    lexicographic order, objectives as %d joined by commas, one row per line
    (src/pmdd/util/output_utils.cpp:87-152, enum/pareto_frontier.hpp:418-433)."""
    import numpy as np

    pts = np.asarray(points, dtype=np.int64)
    if pts.shape[0] > 1:
        pts = pts[np.lexsort(pts.T[::-1])]
    return "".join(",".join(str(int(x)) for x in row) + "\n" for row in pts)


def frontier_digest(points) -> str:
    import hashlib

    return hashlib.sha256(frontier_text(points).encode()).hexdigest()


def headline(name):
    with open(os.path.join(HEADLINE, name)) as f:
        return json.load(f)
