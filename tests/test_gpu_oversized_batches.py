"""Oversized destinations in crowded steps.

A batch of knapsack instances puts more destinations above the tile size into one step
than the GPU holds SFS blocks at once (three per SM), so their blocks are started largest
first; a lone instance sends its few oversized destinations down the GPU-wide mark pass
instead.  The two paths must give the same frontiers, and a sample must match the oracle.
"""
import numpy as np
import pytest

import oracle
import pmdd_b200 as P
from pmdd_b200 import instances

pytestmark = pytest.mark.gpu


def test_crowded_steps_match_lone_runs_and_the_oracle():
    dds = [P.DecisionDiagram.from_text(instances.knapsack_text(46 + i % 9, 3, 4000 + i), 1, 3) for i in range(160)]
    st = {}
    batch = P.enumerate_batch(dds, method=1, stats=st)
    assert st["work_tile_candidates_total"] < st["work_candidates_total"]  # some destinations left the tiles
    for i, dd in enumerate(dds):
        lone = P.enumerate_dd(dd, method=1)
        assert np.array_equal(oracle.sorted_set(batch[i]), oracle.sorted_set(lone)), i
    for i in (0, 57, 159):
        want = oracle.enumerate(dds[i], 1)
        assert np.array_equal(oracle.sorted_set(batch[i]), oracle.sorted_set(want)), i


def test_crowded_steps_with_a_small_scratch_cap():
    """--max-cand passes over the oversized destinations while they are ordered by size."""
    dds = [P.DecisionDiagram.from_text(instances.knapsack_text(48 + i % 5, 3, 4500 + i), 1, 3) for i in range(120)]
    full = P.enumerate_batch(dds, method=1)
    capped = P.enumerate_batch(dds, method=1, max_cand=200_000)
    for a, b in zip(full, capped):
        assert np.array_equal(oracle.sorted_set(a), oracle.sorted_set(b))
