// The two-dimensional staircase a warp keeps while it walks one destination's
// candidates in descending lexicographic order (three objectives).
//
// Every point before q in that order has objective 0 >= q's, so q is dominated (or is a
// later copy of an equal point) iff some earlier point has objectives 1 and 2 both >=
// q's.  The staircase holds the two-dimensional maxima of (objective 1, objective 2) over
// the points walked so far, sorted by objective 1 descending (objective 2 then
// ascending), so one binary search answers the question for q.  The warp walks 32
// candidates at a time: each lane looks its candidate up in the staircase, the chunk's
// survivors are checked against each other (an earlier one dominates; a later one that
// is at least as large in both objectives and differs removes an entry from the next
// staircase), and the next staircase is the surviving entries merged with the chunk's
// new maxima.  Used by the tile kernel (tile_lex.cu) and the oversized-destination path
// (big_lex.cu).
#pragma once

#include <cstdint>

namespace pmdd {
namespace dev {

template <typename T, int CAP>
struct StairBuf {
    static_assert(CAP % 32 == 0, "whole warps of entries");
    T v1[2][CAP];   // objective 1, descending, current and next buffer
    T v2[2][CAP];   // objective 2, ascending
};

// Warp state of one staircase walk (warp-uniform values).
struct StairState {
    int cur = 0;            // buffer in use
    int m = 0;              // entries
    bool overflow = false;  // the maxima outgrew CAP: the caller falls back to pairwise checks
};

// One chunk of up to 32 candidates (lane's candidate (q1, q2) when `valid`), all lanes of
// the warp calling.  Returns whether the lane's candidate is dominated (true for invalid
// lanes).  With `update` the staircase is rebuilt for the next chunk, or st.overflow is
// set when it would exceed CAP (the candidates of this chunk are decided either way).
template <typename T, int CAP>
__device__ __forceinline__ bool stair_chunk(StairBuf<T, CAP> &sb, StairState &st, bool valid, T q1, T q2,
                                            bool update) {
    constexpr unsigned kAll = 0xffffffffu;
    constexpr int G = CAP / 32;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int cur = st.cur, m = st.m;
    bool dom = !valid;
    // entries with objective 1 >= q1: the last of them has the largest objective 2
    int cnt = 0;
    if (valid && m > 0) {
        int a = 0, b = m;
        while (a < b) {
            const int mid = (a + b) >> 1;
            if (sb.v1[cur][mid] >= q1) a = mid + 1;
            else b = mid;
        }
        cnt = a;
        dom = cnt > 0 && sb.v2[cur][cnt - 1] >= q2;
    }
    // the chunk's survivors against each other
    const unsigned alive = __ballot_sync(kAll, !dom);
    bool rem = false;
    unsigned mm = alive;
    while (mm) {
        const int j = __ffs(mm) - 1;
        mm &= mm - 1;
        const T a1 = __shfl_sync(kAll, q1, j), a2 = __shfl_sync(kAll, q2, j);
        const bool ge = (a1 >= q1) & (a2 >= q2);
        dom |= ge & (j < lane);
        rem |= ge & (j > lane) & ((a1 != q1) | (a2 != q2));
    }
    if (!update) return dom;
    // next staircase: surviving entries and the chunk's new maxima, objective 1 descending.
    // No two of them share objective 1 (one would dominate the other), so positions are
    // (entries before) + (new maxima with larger objective 1).
    const bool fresh = !dom && !rem;
    const unsigned nmask = __ballot_sync(kAll, fresh);
    const int groups = (m + 31) >> 5;
    T e1[G], e2[G];
    bool kill[G];
    int gt[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
        kill[g] = false;
        gt[g] = 0;
        e1[g] = 0;
        e2[g] = 0;
        if (g < groups && lane + 32 * g < m) {
            e1[g] = sb.v1[cur][lane + 32 * g];
            e2[g] = sb.v2[cur][lane + 32 * g];
        }
    }
    int gtq = 0;
    unsigned nn = nmask;
    while (nn) {
        const int j = __ffs(nn) - 1;
        nn &= nn - 1;
        const T n1 = __shfl_sync(kAll, q1, j), n2 = __shfl_sync(kAll, q2, j);
#pragma unroll
        for (int g = 0; g < G; ++g) {
            if (g < groups) {
                kill[g] |= (n1 >= e1[g]) & (n2 >= e2[g]);
                gt[g] += (n1 > e1[g]) ? 1 : 0;
            }
        }
        gtq += (n1 > q1) ? 1 : 0;
    }
    unsigned surv[G];
    int before[G];  // surviving entries in the groups before g
    int kept = 0;
#pragma unroll
    for (int g = 0; g < G; ++g) {
        surv[g] = 0;
        if (g < groups) surv[g] = __ballot_sync(kAll, (lane + 32 * g < m) && !kill[g]);
        before[g] = kept;
        kept += __popc(surv[g]);
    }
    const int m_next = kept + __popc(nmask);
    if (m_next > CAP) {
        st.overflow = true;
        return dom;
    }
    const int nxt = cur ^ 1;
#pragma unroll
    for (int g = 0; g < G; ++g) {
        if (g < groups && ((surv[g] >> lane) & 1u)) {
            const int pos = before[g] + __popc(surv[g] & lt_mask) + gt[g];
            sb.v1[nxt][pos] = e1[g];
            sb.v2[nxt][pos] = e2[g];
        }
    }
    if (fresh) {
        // surviving entries before q are among the first cnt (objective 1 >= q1); an entry
        // with objective 1 == q1 is dominated by q and did not survive
        int pos = gtq;
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const int c = min(max(cnt - 32 * g, 0), 32);
            const unsigned mk = c >= 32 ? kAll : ((1u << c) - 1u);
            pos += __popc(surv[g] & mk);
        }
        sb.v1[nxt][pos] = q1;
        sb.v2[nxt][pos] = q2;
    }
    __syncwarp();
    st.cur = nxt;
    st.m = m_next;
    return dom;
}

}  // namespace dev
}  // namespace pmdd
