"""The headline-parity fixtures (tests/golden/headline/) and their digest rule, on CPU.

The fixtures record the reference binary's frontier of every instance of the batched
stream and of the served request lists as a SHA-256 of its sorted frontier text.  This
pins the digest rule to the reference's own files: the text this project builds from
a golden frontier is byte for byte the reference's --frontier-out CSV, and the
committed digests cover exactly the instances the workload generators produce.
"""
import gzip
import os

import numpy as np

from conftest import GOLDEN, HEADLINE, frontier_digest, frontier_text, golden_cases, golden_frontier, headline
from pmdd_b200 import instances


def test_frontier_text_is_the_reference_csv():
    for rec in golden_cases()[:8]:
        for m in rec["methods"]:
            pts = golden_frontier(rec, int(m))
            with open(os.path.join(GOLDEN, f"{rec['name']}.m{m}.csv")) as f:
                assert frontier_text(pts[::-1]) == f.read()


def test_kp4_n60_reference_frontiers_agree():
    texts = []
    for m in (1, 3):
        with gzip.open(os.path.join(HEADLINE, f"kp4_n60_s0.m{m}.csv.gz"), "rt") as f:
            texts.append(f.read())
    assert texts[0] == texts[1] and texts[0].count("\n") == 3285


def test_stream_fixture_covers_the_stream():
    rec = headline("stream.json")["instances"]
    specs = instances.stream_mix(512, 256, 3, seed0=0)
    assert [r["tag"] for r in rec] == [tag for _, _, tag in specs]
    assert all(r["method"] == 1 for r in rec)
    empty = frontier_digest(np.zeros((0, 3), dtype=np.int32))
    assert all(r["num_solutions"] > 0 and r["sha256"] != empty for r in rec)


def test_served_fixture_covers_the_served_lists():
    lists = headline("served.json")["lists"]
    for seed, n_req in ((50, 100), (200, 200), (800, 400)):
        rec = lists[str(seed)]["results"]
        mix = instances.served_mix(n_req, seed)
        assert [(r["tag"], r["problem_type"], r["method"]) for r in rec] == [(t, p, m) for p, _, m, t in mix]
