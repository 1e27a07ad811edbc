"""The method-3 chain rule (chain.cu, count.cu, Engine::step), on CPU.

A method-3 request expands one side per ordinary step: the top-down side when its score
(the candidates of its next layer) is at most the bottom-up side's (1.5 × the candidates
of its next layer), else the bottom-up side, until the sides meet.  A chained step lets
the side it expanded go on while that rule would pick it again -- the device compares the
side's new score with the other side's, which does not move meanwhile -- and stops one
layer short of the other side.  This replays both on random per-layer candidate counts
and checks that they expand the same sides in the same order and meet at the same layer,
whatever the chain lengths.
"""
import numpy as np
import pytest


def side_goes_on(total, other_score, bu):
    """chain_side_goes_on (common.cuh): whether a chained side takes its next layer."""
    return other_score > int(1.5 * float(total)) if bu else total <= other_score


def unchained(td_counts, bu_counts, L):
    """Sides of the ordinary steps: td_counts[l] are the candidates of top-down layer l,
    bu_counts[l] those of bottom-up layer l (the next layer each side would expand)."""
    td, bu = 0, L - 1
    td_score, bu_score = td_counts[1], int(1.5 * float(bu_counts[L - 2]))
    seq = []
    while td != bu:
        if td_score <= bu_score:
            td += 1
            seq.append("td")
            if td != bu:
                td_score = td_counts[td + 1]
        else:
            bu -= 1
            seq.append("bu")
            if td != bu:
                bu_score = int(1.5 * float(bu_counts[bu - 1]))
    return seq, td


def chained(td_counts, bu_counts, L, lengths):
    """The same with a chain after every step that left the sides apart: `lengths` gives
    each chain's most layers (the engine's chain_len), cut to the distance to the other
    side minus one."""
    td, bu = 0, L - 1
    td_score, bu_score = td_counts[1], int(1.5 * float(bu_counts[L - 2]))
    seq = []
    k = 0
    while td != bu:
        side_td = td_score <= bu_score
        if side_td:
            td += 1
            seq.append("td")
        else:
            bu -= 1
            seq.append("bu")
        if td == bu:
            break
        # the step's own count of the expanded side
        if side_td:
            td_score = td_counts[td + 1]
        else:
            bu_score = int(1.5 * float(bu_counts[bu - 1]))
        last = min(lengths[k % len(lengths)], (bu - td) - 1)
        k += 1
        for _ in range(max(last, 0)):
            if side_td:
                if not side_goes_on(td_counts[td + 1], bu_score, False):
                    break
                td += 1
                seq.append("td")
                td_score = td_counts[td + 1]
            else:
                if not side_goes_on(bu_counts[bu - 1], td_score, True):
                    break
                bu -= 1
                seq.append("bu")
                bu_score = int(1.5 * float(bu_counts[bu - 1]))
    return seq, td


@pytest.mark.parametrize("seed", range(40))
def test_chained_sides_equal_unchained(seed):
    rng = np.random.default_rng(seed)
    L = int(rng.integers(3, 120))
    shape = rng.choice(["flat", "peak", "noisy"])
    x = np.arange(L)
    if shape == "flat":
        base = np.full(L, 1000.0)
    elif shape == "peak":
        base = 10.0 + 5000.0 * np.exp(-((x - L / 2) ** 2) / (2 * (L / 5 + 1) ** 2))
    else:
        base = rng.uniform(1, 5000, size=L)
    td_counts = [int(v) for v in base * rng.uniform(0.5, 1.5, size=L)]
    bu_counts = [int(v) for v in base * rng.uniform(0.5, 1.5, size=L)]
    want = unchained(td_counts, bu_counts, L)
    for lengths in ([1], [2], [8], [64], [2, 4, 8, 16], [1, 64, 3]):
        assert chained(td_counts, bu_counts, L, lengths) == want, (seed, lengths)
