"""Parity of the CUDA engine (through the C ABI) with the reference's frontiers:
the committed golden fixtures (made by the reference's own binary) and the oracle on
seeded instances.  Bar: bit-exact equality of the frontier as a set of integer
vectors (no floating point on this path)."""
import itertools

import numpy as np
import pytest

import oracle
import pmdd_b200 as P
from conftest import golden_cases, golden_frontier
from pmdd_b200 import instances

pytestmark = pytest.mark.gpu

CASES = golden_cases()


def same_set(a, b):
    return np.array_equal(oracle.sorted_set(np.asarray(a, dtype=np.int64)), oracle.sorted_set(np.asarray(b, dtype=np.int64)))


@pytest.mark.parametrize("rec", CASES, ids=[c["name"] for c in CASES])
def test_golden_fixtures(rec):
    dd = P.DecisionDiagram.from_file(rec["dat"], rec["problem_type"], rec["nobjs"])
    for m in rec["methods"]:
        st = {}
        got = P.enumerate_dd(dd, method=int(m), stats=st)
        assert same_set(got, golden_frontier(rec, int(m))), f"method {m}"
        if int(m) == 1:
            assert st["work_candidates_total"] == rec["methods"]["1"]["work_candidates_total"]
        elif st["layer_coupling"] == rec["methods"]["3"]["layer_coupling"]:
            # same cutset layer as the reference CPU run -> same join volume
            assert st["work_join_products_total"] == rec["methods"]["3"]["work_join_products_total"]


SEEDED = (
    [(1, d, instances.knapsack_text(n, d, 100 + 7 * n + d), f"kp{d}_n{n}") for d, n in
     itertools.product((1, 2, 3, 4, 6, 8), (1, 2, 7, 16, 22))]
    + [(2, d, instances.setpacking_text(n, m, d, 200 + n), f"sp{d}_n{n}_m{m}") for d, n, m in
       ((3, 12, 4), (3, 50, 15), (2, 80, 20), (5, 35, 10), (1, 20, 5))]
    + [(3, d, instances.tsp_text(n, d, 300 + n), f"tsp{d}_n{n}") for d, n in
       ((3, 2), (3, 3), (3, 5), (2, 9), (4, 8), (6, 7), (5, 9))]
)


@pytest.mark.parametrize("case", SEEDED, ids=[c[3] for c in SEEDED])
@pytest.mark.parametrize("method", (1, 3))
def test_seeded_against_oracle(case, method):
    ptype, d, text, _ = case
    dd = P.DecisionDiagram.from_text(text, ptype, d)
    got = P.enumerate_dd(dd, method=method)
    want = oracle.enumerate(dd, method)
    assert same_set(got, want)
    # a frontier is an antichain without duplicates
    assert len(np.unique(got, axis=0)) == len(got)


def test_seam_mirror_functions():
    bdd = P.DecisionDiagram.from_text(instances.knapsack_text(20, 3, 5), 1, 3)
    mdd = P.DecisionDiagram.from_text(instances.tsp_text(7, 3, 5), 3, 3)
    want_b = oracle.enumerate(bdd, 1)
    want_m = oracle.enumerate(mdd, 1)
    assert same_set(P.topdown_cuda_enumerate(bdd, True, 1, 0), want_b)
    assert same_set(P.coupled_bdd_cuda_enumerate(bdd, True, 1, 0), want_b)
    assert same_set(P.topdown_mdd_cuda_enumerate(mdd), want_m)
    assert same_set(P.coupled_cuda_enumerate(mdd), want_m)


def test_batch_equals_one_at_a_time():
    texts = [(1, instances.knapsack_text(15 + (i % 10), 3, 1000 + i)) for i in range(24)]
    texts += [(2, instances.setpacking_text(40 + i, 12, 3, 2000 + i)) for i in range(8)]
    dds = [P.DecisionDiagram.from_text(t, p, 3) for p, t in texts]
    for method in (1, 3):
        batch = P.enumerate_batch(dds, method=method)
        for dd, got in zip(dds, batch):
            assert same_set(got, P.enumerate_dd(dd, method=method))
            assert same_set(got, oracle.enumerate(dd, method))


def brute_force_knapsack(profits, weights, cap):
    """All feasible subsets (int64 sums) -> their Pareto-maximal distinct vectors."""
    d, n = profits.shape
    vals = []
    for mask in range(1 << n):
        sel = np.array([(mask >> i) & 1 for i in range(n)], dtype=np.int64)
        if int(sel @ weights) <= cap:
            vals.append(profits.astype(np.int64) @ sel)
    pts = np.unique(np.array(vals, dtype=np.int64), axis=0)
    keep = [not any(np.all(q >= p) and np.any(q != p) for q in pts) for p in pts]
    return pts[np.array(keep)]


def test_wide_objectives_use_int64():
    """Profits near 2^30 push path sums past int32: the engine switches to int64 points."""
    rng = np.random.default_rng(42)
    n, d = 9, 3
    profits = rng.integers(1, 1 << 30, size=(d, n))
    weights = rng.integers(1, 100, size=n)
    cap = int(weights.sum()) // 2
    text = f"{n} 1 {d}\n" + "\n".join(" ".join(map(str, r)) for r in profits) + "\n" + \
        " ".join(map(str, weights)) + f" {cap}\n"
    dd = P.DecisionDiagram.from_text(text, 1, d)
    want = brute_force_knapsack(profits, weights, cap)
    for method in (1, 3):
        got = P.enumerate_dd(dd, method=method)
        assert got.dtype == np.int64
        assert same_set(got, want)


def test_oversized_destinations_path():
    """A 5-objective TSP drives destinations past one tile into the global-memory path."""
    dd = P.DecisionDiagram.from_text(instances.tsp_text(10, 5, 77), 3, 5)
    st = {}
    got = P.enumerate_dd(dd, method=1, stats=st)
    assert st["work_candidates_peak"] > 1024
    assert same_set(got, oracle.enumerate(dd, 1))


def test_duplicate_heavy_instances():
    """Identical and near-identical items create many equal candidates across arcs:
    exactly one copy of each frontier point must survive, on every path."""
    for n, d, spread in ((24, 3, 1), (30, 2, 2), (16, 4, 3)):
        rng = np.random.default_rng(n + d)
        profits = rng.integers(1, 1 + spread, size=(d, n))
        weights = rng.integers(1, 1 + spread, size=n)
        cap = int(weights.sum()) // 2
        text = f"{n} 1 {d}\n" + "\n".join(" ".join(map(str, r)) for r in profits) + "\n" + \
            " ".join(map(str, weights)) + f" {cap}\n"
        dd = P.DecisionDiagram.from_text(text, 1, d)
        for method in (1, 3):
            got = P.enumerate_dd(dd, method=method)
            assert same_set(got, oracle.enumerate(dd, method))
            assert len(np.unique(got, axis=0)) == len(got)


def test_high_fan_in_knapsack():
    """A 3-objective knapsack with n=48: the last layers' destinations gather thousands
    of parents and take the oversized path with large candidate sets."""
    dd = P.DecisionDiagram.from_text(instances.knapsack_text(48, 3, 4), 1, 3)
    st = {}
    got = P.enumerate_dd(dd, method=1, stats=st)
    assert st["work_candidates_peak"] > 100_000
    assert same_set(got, oracle.enumerate(dd, 1))


SFS_VARIANT = r"""
import sys
sys.path.insert(0, {root!r})
import numpy as np
import oracle
import pmdd_b200 as P
from pmdd_b200 import instances
rng = np.random.default_rng(1)
ties = ["5", "10"]  # 5-objective 10-city TSP with costs 0..2: equal candidates from different arcs
for _ in range(5):
    m = rng.integers(0, 3, size=(10, 10))
    np.fill_diagonal(m, 0)
    ties += [" ".join(str(int(x)) for x in row) for row in m]
cases = [(3, 5, instances.tsp_text(10, 5, 77)), (1, 3, instances.knapsack_text(48, 3, 4)),
         (1, 3, instances.knapsack_text(30, 3, 9)), (3, 5, "\n".join(ties) + "\n"), (3, 7, instances.tsp_text(9, 7, 3))]
for ptype, d, text in cases:
    dd = P.DecisionDiagram.from_text(text, ptype, d)
    for method in (1, 3):
        got = oracle.sorted_set(np.asarray(P.enumerate_dd(dd, method=method), dtype=np.int64))
        want = oracle.sorted_set(np.asarray(oracle.enumerate(dd, method), dtype=np.int64))
        assert np.array_equal(got, want), (ptype, d, method)
print("ok")
"""


def test_oversized_destinations_through_the_gpu_wide_pass():
    """With PMDD_BIG_MARK_MIN lowered, every oversized destination goes through the
    GPU-wide mark/write pass instead of a single-block sort-filter-skyline: same
    frontiers."""
    import os
    import subprocess
    import sys

    from conftest import ROOT

    env = dict(os.environ, PMDD_BIG_MARK_MIN="1025")
    p = subprocess.run([sys.executable, "-c", SFS_VARIANT.format(root=ROOT)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0 and p.stdout.strip().endswith("ok"), p.stdout + p.stderr


@pytest.mark.parametrize("method", (1, 3))
def test_max_cand_bounds_the_oversized_scratch(method):
    """--max-cand (the reference's destination batching, topdown.cu:671-860) caps the
    candidates materialised at once: oversized destinations are filtered in passes of
    whole destinations.  Same frontier, less device memory at the peak."""
    dd = P.DecisionDiagram.from_text(instances.tsp_text(10, 5, 77), 3, 5)
    st_all, st_cap = {}, {}
    whole = P.enumerate_dd(dd, method=method, stats=st_all)
    capped = P.enumerate_dd(dd, method=method, max_cand=3000, stats=st_cap)
    assert same_set(whole, capped)
    assert same_set(capped, oracle.enumerate(dd, method))
    assert st_cap["work_candidates_total"] == st_all["work_candidates_total"]
    if method == 1:
        assert st_cap["gpu_mem_peak_used_bytes"] < st_all["gpu_mem_peak_used_bytes"]
    else:  # the cutset join's buffers may set the peak instead
        assert st_cap["gpu_mem_peak_used_bytes"] <= st_all["gpu_mem_peak_used_bytes"]


def test_invalid_dd_is_rejected_not_run():
    dd = P.DecisionDiagram.from_text(instances.knapsack_text(5, 3, 1), 1, 3)
    with pytest.raises(P.CudaEnumerationError):
        P.enumerate_dd(dd, method=2)


def test_standalone_pareto_filter_against_oracle():
    """pmdd_pareto_filter keeps exactly the maximal points, one copy of each."""
    rng = np.random.default_rng(11)
    for n, d, hi in ((1, 3, 5), (2, 1, 3), (700, 3, 40), (5000, 4, 60), (20000, 3, 2000), (3000, 8, 6),
                     (40000, 2, 100000)):
        pts = rng.integers(-hi, hi, size=(n, d)).astype(np.int32)
        keep = oracle.nd_keep(pts) if n <= 5000 else None
        got = P.pareto_filter(pts)
        if keep is not None:
            assert same_set(got, pts[keep])
        # properties that hold at any size: an antichain without duplicates that covers the set
        assert len(np.unique(got, axis=0)) == len(got)
        g = got.astype(np.int64)
        sample = pts[rng.choice(n, size=min(n, 300), replace=False)].astype(np.int64)
        for p in sample:
            assert np.any(np.all(g >= p, axis=1))
        for i in range(min(len(g), 200)):
            dom = np.all(g >= g[i], axis=1) & np.any(g != g[i], axis=1)
            assert not dom.any()
