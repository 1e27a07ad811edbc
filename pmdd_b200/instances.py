"""Seeded synthetic instances in the reference's text formats.

One fixed generator (numpy PCG64 via `default_rng(seed)`) per problem type, written
so that the reference's parsers and this package's read the same files:

* knapsack (knapsack_instance.cpp:17-47): profits ~ U[1,1000] per objective and item,
  one weight row ~ U[1,1000], capacity = floor(sum of weights / 2);
* set packing (setpacking_instance.hpp:49-80): objective coefficients ~ U[1,100];
  m constraints, each a uniform random subset of size U{2..20} (1-based indices);
* TSP (tsp_instance.cpp:11-32): per objective an n x n cost matrix ~ U[1,1000] with a
  zero diagonal.
"""
from __future__ import annotations

import numpy as np


def knapsack_arrays(n: int, nobjs: int, seed: int):
    """(profits (nobjs, n), weights (n,), capacity) of the instance knapsack_text writes."""
    rng = np.random.default_rng(seed)
    profits = rng.integers(1, 1001, size=(nobjs, n)).astype(np.int32)
    weights = rng.integers(1, 1001, size=n).astype(np.int32)
    return profits, weights, int(weights.sum()) // 2


def knapsack_text(n: int, nobjs: int, seed: int) -> str:
    profits, weights, cap = knapsack_arrays(n, nobjs, seed)
    lines = [f"{n} 1 {nobjs}"]
    lines += [" ".join(str(int(x)) for x in row) for row in profits]
    lines.append(" ".join(str(int(x)) for x in weights) + f" {cap}")
    return "\n".join(lines) + "\n"


def setpacking_text(n: int, m: int, nobjs: int, seed: int) -> str:
    rng = np.random.default_rng(seed)
    objs = rng.integers(1, 101, size=(nobjs, n))
    lines = [f"{n} {m} {nobjs}"]
    lines += [" ".join(str(int(x)) for x in row) for row in objs]
    for _ in range(m):
        k = int(rng.integers(2, 21))
        k = min(k, n)
        vars_ = rng.choice(n, size=k, replace=False) + 1
        lines.append(f"{k} " + " ".join(str(int(v)) for v in vars_))
    return "\n".join(lines) + "\n"


def tsp_arrays(n: int, nobjs: int, seed: int) -> np.ndarray:
    """Cost matrices (nobjs, n, n) of the instance tsp_text writes."""
    rng = np.random.default_rng(seed)
    cost = np.empty((nobjs, n, n), dtype=np.int32)
    for o in range(nobjs):
        mat = rng.integers(1, 1001, size=(n, n))
        np.fill_diagonal(mat, 0)
        cost[o] = mat
    return cost


def tsp_text(n: int, nobjs: int, seed: int) -> str:
    cost = tsp_arrays(n, nobjs, seed)
    lines = [f"{nobjs}", f"{n}"]
    for mat in cost:
        lines += [" ".join(str(int(x)) for x in row) for row in mat]
    return "\n".join(lines) + "\n"


def stream_mix(num_knapsack: int = 512, num_setpacking: int = 256, nobjs: int = 3, seed0: int = 0):
    """The batched-stream workload: knapsack n ~ U{20..60} and set packing n ~ U{60..100}
    (m = 20), one seed per instance.  Returns (problem_type, text, tag) triples."""
    out = []
    rng = np.random.default_rng(10_000 + seed0)
    for i in range(num_knapsack):
        n = int(rng.integers(20, 61))
        out.append((1, knapsack_text(n, nobjs, seed0 + i), f"kp{nobjs}_n{n}_s{seed0 + i}"))
    for j in range(num_setpacking):
        n = int(rng.integers(60, 101))
        s = seed0 + num_knapsack + j
        out.append((2, setpacking_text(n, 20, nobjs, s), f"sp{nobjs}_n{n}_s{s}"))
    return out


def served_mix(n_req: int, seed: int):
    """The served-loop request list: each request is knapsack (d=3, n ~ U{20..60},
    method 1), set packing (d=3, n ~ U{60..100}, m = 20, method 1) or TSP (d=3,
    n ~ U{9..13} cities, method 3) with equal odds, instance seeds 50000 + 10000*seed + i.
    Returns (problem_type, text, method, tag) tuples; a TSP request's cost matrices are
    tsp_arrays(n, 3, instance seed), the same instance its text describes."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_req):
        kind = rng.integers(0, 3)
        s = 50_000 + seed * 10_000 + i
        if kind == 0:
            n = int(rng.integers(20, 61))
            out.append((1, knapsack_text(n, 3, s), 1, f"kp3_n{n}_s{s}"))
        elif kind == 1:
            n = int(rng.integers(60, 101))
            out.append((2, setpacking_text(n, 20, 3, s), 1, f"sp3_n{n}_s{s}"))
        else:
            n = int(rng.integers(9, 14))
            out.append((3, tsp_text(n, 3, s), 3, f"tsp3_n{n}_s{s}"))
    return out


def tsp_arrays_from_tag(tag: str) -> np.ndarray:
    """Cost matrices of a served-mix TSP request from its tag (tsp3_n<n>_s<seed>)."""
    _, n, s = tag.split("_")
    return tsp_arrays(int(n[1:]), 3, int(s[1:]))
