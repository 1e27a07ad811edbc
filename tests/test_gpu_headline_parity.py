"""Bit-exact parity on the workloads the throughput claims are measured on.

Every frontier of the batched stream (768 instances) and the 4-objective knapsack n=60
frontiers of methods 1 and 3 must equal the reference binary's (tests/golden/headline/,
written by tests/golden/make_headline.py), compared as sorted frontier text (the stream
by SHA-256 of that text).
"""
import concurrent.futures as cf
import gzip
import os

import pytest

from conftest import HEADLINE, frontier_digest, frontier_text, headline
import pmdd_b200 as P
from pmdd_b200 import instances

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stream_dds():
    specs = instances.stream_mix(512, 256, 3, seed0=0)
    with cf.ThreadPoolExecutor(16) as ex:
        return list(ex.map(lambda s: P.DecisionDiagram.from_text(s[1], s[0], 3), specs))


@pytest.mark.parametrize("method", [1, 3])
def test_kp4_n60_frontier_equals_reference(method):
    dd = P.DecisionDiagram.from_text(instances.knapsack_text(60, 4, 0), 1, 4)
    got = P.enumerate_dd(dd, method=method)
    with gzip.open(os.path.join(HEADLINE, f"kp4_n60_s0.m{method}.csv.gz"), "rt") as f:
        assert frontier_text(got) == f.read()


def _check_stream(outs):
    rec = headline("stream.json")["instances"]
    assert len(outs) == len(rec)
    bad = [r["tag"] for r, o in zip(rec, outs)
           if len(o) != r["num_solutions"] or frontier_digest(o) != r["sha256"]]
    assert not bad, f"{len(bad)} stream frontiers differ from the reference: {bad[:5]}"


def test_stream_resident_frontiers_equal_reference(stream_dds):
    res = P.ResidentSet(stream_dds)
    try:
        outs = res.enumerate(method=1)
    finally:
        res.close()
    _check_stream(outs)


def test_stream_batch_frontiers_equal_reference(stream_dds):
    _check_stream(P.enumerate_batch(stream_dds, method=1))
