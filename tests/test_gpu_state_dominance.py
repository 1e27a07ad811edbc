"""Knapsack state dominance on the GPU (method 1, problem type 1, state_dominance > 0).

The reference prunes, after every top-down layer, the labels of a node that a label of
one of the next two nodes in min_weight order weakly dominates
(src/pmdd/enum/gpu/topdown.cu:256-521).  The frontier does not change; the labels
removed, the candidates of later layers and the survivors do.  Bar: the frontier and all
three counts equal to the reference run (golden fixtures) and to the oracle.
"""
import itertools

import numpy as np
import pytest

import oracle
import pmdd_b200 as P
from conftest import golden_cases, golden_frontier
from pmdd_b200 import instances

pytestmark = pytest.mark.gpu

KP = [c for c in golden_cases() if "state_dominance_1" in c]


def same_set(a, b):
    return np.array_equal(oracle.sorted_set(np.asarray(a, dtype=np.int64)),
                          oracle.sorted_set(np.asarray(b, dtype=np.int64)))


@pytest.mark.parametrize("rec", KP, ids=[c["name"] for c in KP])
def test_golden_state_dominance(rec):
    dd = P.DecisionDiagram.from_file(rec["dat"], 1, rec["nobjs"])
    st = {}
    got = P.enumerate_dd(dd, method=1, state_dominance=1, stats=st)
    assert same_set(got, golden_frontier(rec, 1))
    want = rec["state_dominance_1"]
    assert st["dominance_filtered_total"] == want["dominance_filtered_total"]
    assert st["work_candidates_total"] == want["work_candidates_total"]
    assert st["work_frontier_survivors_total"] == want["work_frontier_survivors_total"]


SEEDED = [(d, n, instances.knapsack_text(n, d, 500 + 13 * n + d)) for d, n in
          itertools.product((1, 2, 3, 5, 8), (3, 9, 17, 28))]


@pytest.mark.parametrize("case", SEEDED, ids=[f"kp{d}_n{n}" for d, n, _ in SEEDED])
def test_seeded_state_dominance_against_oracle(case):
    d, n, text = case
    dd = P.DecisionDiagram.from_text(text, 1, d)
    st, ost = {}, {}
    got = P.enumerate_dd(dd, method=1, state_dominance=1, stats=st)
    want = oracle.enumerate(dd, 1, state_dominance=1, stats=ost)
    assert same_set(got, want)
    assert st["dominance_filtered_total"] == ost["dominance_filtered_total"]
    assert st["work_candidates_total"] == ost["candidates_total"]


def test_state_dominance_in_a_batch_and_resident():
    dds = [P.DecisionDiagram.from_text(instances.knapsack_text(12 + i % 20, 3, 900 + i), 1, 3) for i in range(40)]
    want = []
    for dd in dds:
        ost = {}
        want.append((oracle.enumerate(dd, 1, state_dominance=1, stats=ost), ost["dominance_filtered_total"]))
    st = {}
    got = P.enumerate_batch(dds, method=1, state_dominance=1, stats=st)
    for g, (w, _) in zip(got, want):
        assert same_set(g, w)
    assert st["dominance_filtered_total"] == sum(r for _, r in want)
    res = P.ResidentSet(dds)
    try:
        st2 = {}
        got2 = res.enumerate(method=1, state_dominance=1, stats=st2)
        for g, (w, _) in zip(got2, want):
            assert same_set(g, w)
        assert st2["dominance_filtered_total"] == st["dominance_filtered_total"]
        # the same resident set without state dominance prunes nothing
        st3 = {}
        res.enumerate(method=1, stats=st3)
        assert st3["dominance_filtered_total"] == 0
    finally:
        res.close()


@pytest.mark.parametrize("ptype,method", [(1, 3), (2, 1), (3, 1)])
def test_state_dominance_is_a_no_op_elsewhere(ptype, method):
    """Like the reference's GPU path: only method 1 on knapsack prunes states."""
    text = {1: instances.knapsack_text(20, 3, 7), 2: instances.setpacking_text(40, 12, 3, 7),
            3: instances.tsp_text(7, 3, 7)}[ptype]
    dd = P.DecisionDiagram.from_text(text, ptype, 3)
    st = {}
    got = P.enumerate_dd(dd, method=method, state_dominance=1, stats=st)
    assert same_set(got, oracle.enumerate(dd, method))
    assert st["dominance_filtered_total"] == 0
