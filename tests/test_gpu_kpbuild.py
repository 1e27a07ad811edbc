"""Knapsack BDDs built on the device (pmdd_resident_build_knapsack).

Bar: every flat array (layer and arc offsets, arc tails and weight rows, the weight table,
min_weight) equal to the host constructor's -- whose DD structure is pinned against the
reference's stats -- and the frontiers and counters of enumerations over the built set
equal to those over the host-built DDs."""
import numpy as np
import pytest

import oracle
import pmdd_b200 as P
from pmdd_b200 import _native, instances

KEYS = ("layer_offsets", "in_arc_offsets", "arc_src", "arc_weight", "weights", "min_weight")


def text_of(profits, weights, cap):
    d, n = profits.shape
    lines = [f"{n} 1 {d}"] + [" ".join(map(str, r)) for r in profits] + [" ".join(map(str, weights)) + f" {cap}"]
    return "\n".join(lines) + "\n"


def assert_same_dd(res, i, text, d):
    host = P.DecisionDiagram.from_text(text, 1, d)
    want = host.arrays()
    got = res.dd_arrays(i)
    for k in KEYS:
        w = np.asarray(want[k]).reshape(-1)
        g = np.asarray(got[k]).reshape(-1)
        assert w.shape == g.shape and np.array_equal(w, g), (i, k)
    info, hinfo = res.dd_info(i), host.info()
    for k in ("original_width", "original_num_nodes", "reduced_width", "reduced_num_nodes"):
        assert info[k] == hinfo[k], (i, k)
    return host


SEEDED = [(n, d, 7000 + 31 * n + d) for n in (1, 2, 3, 7, 16, 25, 40, 60) for d in (1, 2, 3, 4, 7, 8)]


@pytest.mark.gpu
@pytest.mark.parametrize("d", (1, 2, 3, 4, 7, 8))
def test_device_built_arrays_equal_host_built(d):
    cases = [c for c in SEEDED if c[1] == d]
    specs = [instances.knapsack_arrays(n, d, s) for n, _, s in cases]
    res = P.ResidentSet.from_knapsack(specs)
    try:
        for i, (n, _, s) in enumerate(cases):
            assert_same_dd(res, i, instances.knapsack_text(n, d, s), d)
    finally:
        res.close()


@pytest.mark.gpu
def test_edge_instances():
    """Zero weights, items heavier than the capacity, capacity 0, one item."""
    rng = np.random.default_rng(11)
    specs, texts = [], []
    for trial in range(120):
        n = int(rng.integers(1, 16))
        d = 2
        profits = rng.integers(0, 60, size=(d, n)).astype(np.int32)
        weights = rng.integers(0, 14, size=n).astype(np.int32)
        weights[rng.random(n) < 0.2] = 0
        cap = 0 if rng.random() < 0.15 else int(rng.integers(0, 40))
        weights[rng.random(n) < 0.15] = cap + int(rng.integers(1, 6))
        specs.append((profits, weights, cap))
        texts.append(text_of(profits, weights, cap))
    res = P.ResidentSet.from_knapsack(specs)
    try:
        for i, t in enumerate(texts):
            assert_same_dd(res, i, t, 2)
        got = res.enumerate(method=1)
        for i, t in enumerate(texts):
            want = oracle.enumerate(P.DecisionDiagram.from_text(t, 1, 2), 1)
            assert np.array_equal(oracle.sorted_set(got[i]), oracle.sorted_set(want)), i
    finally:
        res.close()


@pytest.mark.gpu
@pytest.mark.parametrize("method", (1, 3))
@pytest.mark.parametrize("sd", (0, 1))
def test_enumeration_over_the_built_set(method, sd):
    cases = [(int(n), 3, 9100 + i) for i, n in enumerate(np.random.default_rng(4).integers(10, 45, size=40))]
    specs = [instances.knapsack_arrays(n, d, s) for n, d, s in cases]
    dds = [P.DecisionDiagram.from_text(instances.knapsack_text(n, d, s), 1, d) for n, d, s in cases]
    built = P.ResidentSet.from_knapsack(specs)
    uploaded = P.ResidentSet(dds)
    try:
        st_b, st_u = {}, {}
        got = built.enumerate(method=method, state_dominance=sd, stats=st_b)
        ref = uploaded.enumerate(method=method, state_dominance=sd, stats=st_u)
        for g, r in zip(got, ref):
            assert np.array_equal(oracle.sorted_set(g), oracle.sorted_set(r))
        for k in ("work_candidates_total", "work_frontier_survivors_total", "dominance_filtered_total",
                  "work_join_products_total"):
            assert st_b[k] == st_u[k], k
        if sd:
            assert st_b["dominance_filtered_total"] > 0
    finally:
        built.close()
        uploaded.close()


@pytest.mark.gpu
def test_golden_fixtures_from_device_built_dds():
    from conftest import golden_cases, golden_frontier

    recs = [r for r in golden_cases() if r["problem_type"] == 1 and "1" in r["methods"]]
    specs = []
    for r in recs:
        toks = list(map(int, open(r["dat"]).read().split()))
        n, m, d_file = toks[0], toks[1], toks[2]
        assert m == 1
        prof = np.array(toks[3:3 + d_file * n], dtype=np.int32).reshape(d_file, n)[: r["nobjs"]]
        w = np.array(toks[3 + d_file * n:3 + d_file * n + n], dtype=np.int32)
        specs.append((prof, w, toks[3 + d_file * n + n]))
    res = P.ResidentSet.from_knapsack(specs)
    try:
        for method in (1, 3):
            got = res.enumerate(method=method)
            for r, g in zip(recs, got):
                assert np.array_equal(oracle.sorted_set(g), golden_frontier(r, 1)), (r["name"], method)
    finally:
        res.close()


def test_invalid_knapsack_sets_are_rejected_before_the_device():
    lib = _native.gpu_lib()
    import ctypes

    P32 = ctypes.POINTER(ctypes.c_int32)
    prof = np.ones((2, 3), dtype=np.int32)
    for n, d, w, cap, why in ((0, 2, [1, 1, 1], 5, "n must be"), (3, 9, [1, 1, 1], 5, "nobjs"),
                              (3, 2, [1, -1, 1], 5, "weights"), (3, 2, [1, 1, 1], -1, "capacity"),
                              (3, 2, [1, 1, 1], (1 << 24) + 1, "capacity")):
        wa = np.array(w, dtype=np.int32)
        spec = (_native.PmddKnapsack * 1)(_native.PmddKnapsack(n, d, prof.ctypes.data_as(P32),
                                                               wa.ctypes.data_as(P32), cap, 0))
        err = ctypes.create_string_buffer(256)
        assert not lib.pmdd_resident_build_knapsack(spec, 1, 0, err, len(err))
        assert why in err.value.decode(), err.value
