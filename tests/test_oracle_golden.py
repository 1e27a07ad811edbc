"""The oracle (C restatement of the reference's CPU enumeration) and the host DD
constructors, pinned against fixtures produced by the reference's own binary."""
import numpy as np
import pytest

import oracle
from conftest import golden_cases, golden_frontier
from pmdd_b200 import DecisionDiagram

CASES = golden_cases()


@pytest.mark.parametrize("rec", CASES, ids=[c["name"] for c in CASES])
def test_dd_structure_matches_reference(rec):
    dd = DecisionDiagram.from_file(rec["dat"], rec["problem_type"], rec["nobjs"])
    ref = rec["structure"]
    info = dd.info()
    assert dd.layer_sizes() == ref["max_num_nodes_per_layer"]
    assert info["total_num_in_arcs"] == ref["total_num_in_arcs"]
    assert info["max_num_in_arcs"] == ref["max_num_in_arcs"]
    for k in ("original_width", "reduced_width", "original_num_nodes", "reduced_num_nodes"):
        assert info[k] == ref[k], k


@pytest.mark.parametrize("rec", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference_frontier(rec):
    dd = DecisionDiagram.from_file(rec["dat"], rec["problem_type"], rec["nobjs"])
    for m in rec["methods"]:
        m = int(m)
        want = golden_frontier(rec, m)
        st = {}
        got = oracle.enumerate(dd, m, stats=st)
        assert np.array_equal(oracle.sorted_set(got), want), f"method {m}"
        assert len(got) == rec["methods"][str(m)]["num_solutions"]
        if m == 1:
            # the CPU top-down candidate count is the reference's work_candidates_total
            assert st["candidates_total"] == rec["methods"]["1"]["work_candidates_total"]
        if m == 3:
            assert st["join_products_total"] == rec["methods"]["3"]["work_join_products_total"]
            assert st["layer_coupling"] == rec["methods"]["3"]["layer_coupling"]


@pytest.mark.parametrize("rec", [c for c in CASES if c["problem_type"] != 3][:8], ids=lambda c: c["name"])
def test_oracle_bottomup_equals_topdown(rec):
    dd = DecisionDiagram.from_file(rec["dat"], rec["problem_type"], rec["nobjs"])
    want = golden_frontier(rec, 1 if "1" in rec["methods"] else 3)
    assert np.array_equal(oracle.sorted_set(oracle.enumerate(dd, 2)), want)


@pytest.mark.parametrize("rec", [c for c in CASES if c["problem_type"] == 1], ids=lambda c: c["name"])
def test_oracle_knapsack_state_dominance_keeps_frontier(rec):
    """Knapsack state dominance prunes labels but not the frontier (single constraint)."""
    dd = DecisionDiagram.from_file(rec["dat"], 1, rec["nobjs"])
    st = {}
    got = oracle.enumerate(dd, 1, state_dominance=1, stats=st)
    assert np.array_equal(oracle.sorted_set(got), golden_frontier(rec, 1))
    # and prunes exactly the labels the reference's run with state_dominance=1 prunes
    want = rec["state_dominance_1"]
    assert st["dominance_filtered_total"] == want["dominance_filtered_total"]
    assert st["candidates_total"] == want["work_candidates_total"]
    assert st["survivors_total"] == want["work_frontier_survivors_total"]


NUMBERED = [c for c in CASES if "same_numbering" in c]


@pytest.mark.parametrize("rec", NUMBERED, ids=[c["name"] for c in NUMBERED])
def test_oracle_counters_match_reference_on_same_numbering(rec):
    """Every counter of methods 1 and 3, with and without state dominance (knapsack and
    set packing), equals the reference's CPU enumeration run on the same DD numbering."""
    dd = DecisionDiagram.from_file(rec["dat"], rec["problem_type"], rec["nobjs"])
    for key, want in rec["same_numbering"].items():
        m, sd = int(key[1]), int(key[-1])
        st = {}
        got = oracle.enumerate(dd, m, state_dominance=sd, stats=st)
        assert len(got) == want["num_solutions"], key
        assert np.array_equal(oracle.sorted_set(got), golden_frontier(rec, m if str(m) in rec["methods"] else 1)), key
        assert st["dominance_filtered_total"] == want["dominance_filtered_total"], key
        assert st["candidates_total"] == want["work_candidates_total"], key
        assert st["survivors_total"] == want["work_frontier_survivors_total"], key
        if m == 3:
            assert st["layer_coupling"] == want["layer_coupling"], key
            assert st["join_products_total"] == want["work_join_products_total"], key


def test_same_numbering_fixtures_exercise_set_packing_state_dominance():
    pruned = [c["name"] for c in NUMBERED
              if c["problem_type"] == 2 and c["same_numbering"]["m1_sd1"]["dominance_filtered_total"] > 0
              and c["same_numbering"]["m3_sd1"]["dominance_filtered_total"] > 0]
    assert len(pruned) >= 3, pruned


def test_nd_keep_rule_against_bruteforce():
    rng = np.random.default_rng(7)
    for trial in range(30):
        d = int(rng.integers(1, 6))
        n = int(rng.integers(1, 60))
        pts = rng.integers(0, 4, size=(n, d)).astype(np.int32)
        keep = oracle.nd_keep(pts)
        for i in range(n):
            dom = any(
                j != i and np.all(pts[j] >= pts[i]) and (np.any(pts[j] != pts[i]) or j < i) for j in range(n)
            )
            assert keep[i] == (not dom)
