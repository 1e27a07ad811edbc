"""The rule behind the oversized path's pivot prefilter, restated on the CPU.

The GPU-wide pass for destinations above a tile drops every candidate that some pivot
dominates (a pivot q dominates candidate p when q >= p on every objective and q differs
from p or comes before it), packs the remaining candidates in candidate order, and runs
the pairwise filter over those alone.  That is exact for any pivot set, because whatever
dominates a remaining candidate is itself remaining: a pivot dominating the dominator
would dominate the candidate too, equal points included.  These tests check the claim
against the oracle's filter (the GPU filter rule: of equal points the first is kept) on
seeded sets with many duplicates, for the engine's pivot choice (largest objective sums)
and for arbitrary ones.
"""
import numpy as np
import pytest

import oracle


def dominated_by_pivots(pts: np.ndarray, piv: np.ndarray) -> np.ndarray:
    """True where some pivot (positions `piv`) dominates the candidate."""
    out = np.zeros(len(pts), dtype=bool)
    P = pts[piv]
    for a in range(0, len(pts), 1024):
        x = pts[a:a + 1024]
        ge = np.all(P[None, :, :] >= x[:, None, :], axis=2)
        eq = np.all(P[None, :, :] == x[:, None, :], axis=2)
        earlier = piv[None, :] < np.arange(a, a + len(x))[:, None]
        out[a:a + 1024] = np.any(ge & (~eq | earlier), axis=1)
    return out


def two_stage_keep(pts: np.ndarray, piv: np.ndarray) -> np.ndarray:
    rest = np.flatnonzero(~dominated_by_pivots(pts, piv))
    keep = np.zeros(len(pts), dtype=bool)
    keep[rest[oracle.nd_keep(pts[rest])]] = True
    return keep


def largest_sum_pivots(pts: np.ndarray, k: int) -> np.ndarray:
    s = pts.astype(np.int64).sum(axis=1)
    return np.sort(np.argsort(-s, kind="stable")[:k])


@pytest.mark.parametrize("n,d,hi,seed", [(3000, 3, 12, 0), (2500, 5, 4, 1), (2000, 2, 40, 2), (1500, 7, 3, 3),
                                         (4000, 4, 1000, 4), (1200, 1, 5, 5)])
def test_pivot_prefilter_is_exact(n, d, hi, seed):
    rng = np.random.default_rng(seed)
    pts = rng.integers(-hi, hi + 1, size=(n, d)).astype(np.int32)
    pts[rng.integers(0, n, n // 5)] = pts[rng.integers(0, n, n // 5)]  # plant duplicates
    want = oracle.nd_keep(pts)
    for piv in (largest_sum_pivots(pts, 512), largest_sum_pivots(pts, n // 64 + 1),
                np.sort(rng.choice(n, 97, replace=False)), np.arange(n), np.zeros(0, dtype=np.int64)):
        assert np.array_equal(two_stage_keep(pts, piv), want)


def test_equal_points_keep_the_first_copy():
    """Copies of one maximal point: a pivot that is a later copy must not remove the first."""
    pts = np.array([[5, 5, 5], [1, 9, 0], [5, 5, 5], [5, 5, 5], [0, 0, 0]], dtype=np.int32)
    for piv in (np.array([2]), np.array([3]), np.array([0, 3]), np.array([4])):
        keep = two_stage_keep(pts, piv)
        assert keep.tolist() == [True, True, False, False, False]
