"""TSP MDDs on the device: the n-city structure built once on the GPU and shared, each
instance adding its weight table (pmdd_resident_build_tsp, pmdd_server_submit_tsp).

Bar: every flat array equal to the host constructor's (whose MDD structure is pinned
against the reference's stats), and frontiers and counters of enumerations over the
device-built set equal to those over host-built DDs and to the oracle."""
import ctypes

import numpy as np
import pytest

import oracle
import pmdd_b200 as P
from pmdd_b200 import _native, instances

KEYS = ("layer_offsets", "in_arc_offsets", "arc_src", "arc_weight", "weights")


def text_of(cost):
    d, n, _ = cost.shape
    lines = [f"{d}", f"{n}"]
    for mat in cost:
        lines += [" ".join(map(str, row)) for row in mat]
    return "\n".join(lines) + "\n"


@pytest.mark.gpu
def test_device_built_arrays_equal_host_built():
    cases = [(n, d, 300 + 7 * n + d) for n in range(2, 14) for d in (1, 3, 5)] + [(15, 5, 1)]
    costs = [instances.tsp_arrays(n, d, s) for n, d, s in cases]
    res = P.ResidentSet.from_tsp(costs)
    try:
        for i, (n, d, s) in enumerate(cases):
            host = P.DecisionDiagram.from_text(instances.tsp_text(n, d, s), 3, d).arrays()
            got = res.dd_arrays(i)
            for k in KEYS:
                w = np.asarray(host[k]).reshape(-1)
                g = np.asarray(got[k]).reshape(-1)
                assert w.shape == g.shape and np.array_equal(w, g), (n, d, k)
    finally:
        res.close()


@pytest.mark.gpu
@pytest.mark.parametrize("method", (1, 3))
def test_enumeration_over_the_built_set(method):
    cases = [(n, 3, 500 + n) for n in (4, 5, 6, 7, 8, 9, 10, 11, 12)]
    costs = [instances.tsp_arrays(n, d, s) for n, d, s in cases]
    dds = [P.DecisionDiagram.from_text(instances.tsp_text(n, d, s), 3, d) for n, d, s in cases]
    built = P.ResidentSet.from_tsp(costs)
    uploaded = P.ResidentSet(dds)
    try:
        st_b, st_u = {}, {}
        got = built.enumerate(method=method, stats=st_b)
        ref = uploaded.enumerate(method=method, stats=st_u)
        for g, r, dd in zip(got, ref, dds):
            assert np.array_equal(oracle.sorted_set(g), oracle.sorted_set(r))
            assert np.array_equal(oracle.sorted_set(g), oracle.sorted_set(oracle.enumerate(dd, method)))
        for k in ("work_candidates_total", "work_frontier_survivors_total", "work_join_products_total"):
            assert st_b[k] == st_u[k], k
    finally:
        built.close()
        uploaded.close()


@pytest.mark.gpu
def test_golden_fixtures_from_device_built_mdds():
    from conftest import golden_cases, golden_frontier

    recs = [r for r in golden_cases() if r["problem_type"] == 3]
    costs = []
    for r in recs:
        tok = list(map(int, open(r["dat"]).read().split()))
        d_file, n = tok[0], tok[1]
        costs.append(np.array(tok[2:2 + d_file * n * n], dtype=np.int32).reshape(d_file, n, n)[: r["nobjs"]])
    res = P.ResidentSet.from_tsp(costs)
    try:
        for method in (1, 3):
            got = res.enumerate(method=method)
            for r, g in zip(recs, got):
                m = method if str(method) in r["methods"] else int(next(iter(r["methods"])))
                assert np.array_equal(oracle.sorted_set(g), golden_frontier(r, m)), (r["name"], method)
    finally:
        res.close()


@pytest.mark.gpu
def test_server_takes_tsp_requests_by_their_costs():
    rng = np.random.default_rng(8)
    srv = P.Server()
    want = {}
    try:
        for k in range(24):
            n = int(rng.integers(3, 12))
            cost = instances.tsp_arrays(n, 3, 900 + k)
            method = 1 + 2 * (k % 2)
            assert srv.submit_tsp(cost, k, method=method) == 0
            want[k] = oracle.enumerate(P.DecisionDiagram.from_text(text_of(cost), 3, 3), method)
        got = {}
        while len(got) < len(want):
            srv.run(1)
            while True:
                r = srv.poll()
                if r is None:
                    break
                assert r.status == 0, r.error
                got[r.req_id] = r.frontier
        for k, w in want.items():
            assert np.array_equal(oracle.sorted_set(got[k]), oracle.sorted_set(w)), k
    finally:
        srv.close()


def test_invalid_tsp_sets_are_rejected_before_the_device():
    lib = _native.gpu_lib()
    for n, d, why in ((1, 2, "n must be"), (21, 2, "n must be"), (5, 0, "nobjs"), (5, 9, "nobjs")):
        cost = np.zeros((max(d, 1), max(n, 1), max(n, 1)), dtype=np.int32)
        spec = (_native.PmddTsp * 1)(_native.PmddTsp(n, d, cost.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        err = ctypes.create_string_buffer(256)
        assert not lib.pmdd_resident_build_tsp(spec, 1, 0, err, len(err))
        assert why in err.value.decode(), err.value
