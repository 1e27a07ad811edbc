"""The staircase rule of the three-objective filters (stair.cuh), on CPU.

A line-by-line Python rendering of one warp walking a destination's candidates in
descending lexicographic order, 32 at a time: staircase lookup by binary search, the
chunk's survivors checked against each other lane by lane, and the staircase rebuilt
from its surviving entries and the chunk's new maxima at the positions the kernel
computes (asserting the staircase stays strictly ordered and no two entries collide).
Its keep flags must give the oracle's frontier (the reference GPU filter's keep rule,
src/pmdd/enum/gpu/dominance_utils.cuh:10-23) on seeded sets with duplicates, with
anti-correlated objectives, and with a staircase capacity small enough to force the
fallback to checking every earlier point.  The tile kernel's split of a large
destination into segments walked by separate warps, joined by looking each survivor up
in the earlier segments' final staircases, must give the same keep flags.
"""
import numpy as np
import pytest

import oracle


def stair_walk(P, cap, save=False):
    """Keep flags of one warp's walk; with `save` also the final staircase (None if it
    outgrew cap)."""
    n = len(P)
    keep = np.zeros(n, bool)
    stair = []          # (objective 1, objective 2), objective 1 descending
    overflow = False
    for c0 in range(0, n, 32):
        lanes = range(32)
        valid = [c0 + l < n for l in lanes]
        q1 = [int(P[c0 + l, 1]) if valid[l] else 0 for l in lanes]
        q2 = [int(P[c0 + l, 2]) if valid[l] else 0 for l in lanes]
        dom = [not v for v in valid]
        if overflow:
            for l in lanes:
                if valid[l]:
                    p = c0 + l
                    dom[l] = any(P[j, 1] >= q1[l] and P[j, 2] >= q2[l] for j in range(p))
                    keep[p] = not dom[l]
            continue
        m = len(stair)
        cnt = [0] * 32
        for l in lanes:
            if valid[l] and m > 0:
                a, b = 0, m
                while a < b:
                    mid = (a + b) // 2
                    if stair[mid][0] >= q1[l]:
                        a = mid + 1
                    else:
                        b = mid
                cnt[l] = a
                dom[l] = a > 0 and stair[a - 1][1] >= q2[l]
        alive = [not d for d in dom]
        rem = [False] * 32
        for j in lanes:
            if alive[j]:
                for l in lanes:
                    ge = q1[j] >= q1[l] and q2[j] >= q2[l]
                    dom[l] |= ge and j < l
                    rem[l] |= ge and j > l and (q1[j], q2[j]) != (q1[l], q2[l])
        for l in lanes:
            if valid[l]:
                keep[c0 + l] = not dom[l]
        if c0 + 32 >= n and not save:
            break
        fresh = [l for l in lanes if not dom[l] and not rem[l]]
        kill = [any(q1[j] >= e1 and q2[j] >= e2 for j in fresh) for e1, e2 in stair]
        gt = [sum(q1[j] > e1 for j in fresh) for e1, _ in stair]
        surv = [i for i in range(m) if not kill[i]]
        if len(surv) + len(fresh) > cap:
            overflow = True
            continue
        new = [None] * (len(surv) + len(fresh))
        for r, i in enumerate(surv):
            pos = r + gt[i]
            assert new[pos] is None
            new[pos] = stair[i]
        for l in fresh:
            pos = sum(1 for i in surv if i < cnt[l]) + sum(q1[j] > q1[l] for j in fresh)
            assert new[pos] is None
            new[pos] = (q1[l], q2[l])
        for x, y in zip(new, new[1:]):
            assert x[0] > y[0] and x[1] < y[1]
        stair = new
    if save:
        return keep, (None if overflow else stair)
    return keep


def segmented_walk(P, seg, cap):
    """The tile kernel's split of a large destination (tile_lex.cu): segments of equal
    length at most `seg`, each walked from an empty staircase by its own warp, the final
    staircases of all but the last kept; then every survivor of segment g is looked up in
    the staircases of segments 0..g-1 (or compared with their points where one was not
    kept)."""
    n = len(P)
    nseg = (n + seg - 1) // seg
    ln = (n + nseg - 1) // nseg
    keep = np.zeros(n, bool)
    stairs = []
    for g in range(nseg):
        a, b = g * ln, min(n, (g + 1) * ln)
        assert a < b
        k, st = stair_walk(P[a:b], cap, save=True)
        keep[a:b] = k
        stairs.append(st)
    for q in range(n):
        if not keep[q]:
            continue
        q1, q2 = P[q, 1], P[q, 2]
        for t in range(q // ln):
            st = stairs[t]
            if st is None:
                dom = any(P[j, 1] >= q1 and P[j, 2] >= q2 for j in range(t * ln, (t + 1) * ln))
            else:
                lo, hi = 0, len(st)
                while lo < hi:
                    mid = (lo + hi) // 2
                    if st[mid][0] >= q1:
                        lo = mid + 1
                    else:
                        hi = mid
                dom = lo > 0 and st[lo - 1][1] >= q2
            if dom:
                keep[q] = False
                break
    return keep


@pytest.mark.parametrize("cap", [64, 256, 5])
def test_staircase_walk_keeps_the_oracle_frontier(cap):
    rng = np.random.default_rng(cap)
    for t in range(60):
        n = int(rng.integers(1, 200))
        hi = int(rng.choice([4, 10, 50, 1000, 100000]))
        pts = rng.integers(0, hi, size=(n, 3)).astype(np.int64)
        if t % 4 == 0:
            pts[n // 3:2 * n // 3] = pts[:2 * n // 3 - n // 3]
        if t % 5 == 1:
            x = rng.integers(0, 1000, size=n)
            y = rng.integers(0, 1000, size=n)
            pts = np.stack([x, y, 2000 - x - y + rng.integers(0, 5, size=n)], 1)
        order = sorted(range(n), key=lambda i: (-pts[i, 0], -pts[i, 1], -pts[i, 2], i))
        P = pts[order]
        keep = stair_walk(P, cap)
        want = oracle.nd_keep(P.astype(np.int32))
        assert np.array_equal(oracle.sorted_set(P[keep]), oracle.sorted_set(P[want])), t
        assert keep.sum() == want.sum()


@pytest.mark.parametrize("seg,cap", [(64, 64), (64, 5), (32, 64)])
def test_segmented_walk_gives_the_same_keep_flags(seg, cap):
    rng = np.random.default_rng(seg * 100 + cap)
    for t in range(40):
        n = int(rng.integers(1, 700))
        hi = int(rng.choice([4, 10, 50, 1000, 100000]))
        pts = rng.integers(0, hi, size=(n, 3)).astype(np.int64)
        if t % 4 == 0:
            pts[n // 3:2 * n // 3] = pts[:2 * n // 3 - n // 3]
        if t % 5 == 1:
            x = rng.integers(0, 1000, size=n)
            y = rng.integers(0, 1000, size=n)
            pts = np.stack([x, y, 2000 - x - y + rng.integers(0, 5, size=n)], 1)
        order = sorted(range(n), key=lambda i: (-pts[i, 0], -pts[i, 1], -pts[i, 2], i))
        P = pts[order]
        got = segmented_walk(P, seg, cap)
        assert np.array_equal(got, oracle.nd_keep(P.astype(np.int32))), t
