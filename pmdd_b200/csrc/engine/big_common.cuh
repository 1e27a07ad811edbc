// Shared device helpers of the oversized-destination paths (big.cu, big_lex.cu): the
// destination behind a work item or a flat candidate index of one scratch pass, and the
// arc run a candidate belongs to.
#pragma once

#include "common.cuh"

namespace pmdd {
namespace dev {
namespace big {

struct BigItem {
    int32_t item;      // job-local destination
    int32_t a0, a1;    // its arcs (global ids)
    int64_t soff;      // scratch offset (candidates) within this pass's window
    int64_t c0;        // job-local candidate start (the slot start)
    int64_t n;         // candidates
};

__device__ __forceinline__ void fill_item(const ExpandJob &J, int64_t k, int64_t lo, BigItem *b) {
    b->item = static_cast<int32_t>(J.big_list[2 * k]);
    b->soff = J.big_list[2 * k + 1] - lo;
    const int32_t v = J.item_base + b->item;
    b->a0 = J.item_arc_off[v];
    b->a1 = J.item_arc_off[v + 1];
    b->c0 = J.arc_cand_off[b->a0 - J.arc_base];
    b->n = J.arc_cand_off[b->a1 - J.arc_base] - b->c0;
}

// Destinations of three objectives whose runs all come from sorted frontiers, at most
// J.lex_max_arcs of them: the lexicographic path (big_lex.cu) filters these.
__device__ __forceinline__ bool lex_eligible(const ExpandJob &J, const BigItem &B) {
    if (J.prev_sorted == nullptr || B.a1 - B.a0 > J.lex_max_arcs) return false;
    for (int32_t a = B.a0; a < B.a1; ++a)
        if (J.prev_sorted[J.arc_nbr[a] - J.prev_base] == 0) return false;
    return true;
}

// The destination of work item W, if pass `pass` takes it (its scratch offset lies in the
// pass's window); its scratch offset is then re-based to the window.
__device__ __forceinline__ bool big_item(const ExpandJob &J, const BigWork &W, int64_t pass, BigItem *b) {
    const int64_t lo = pass * J.big_window;
    const int64_t s = J.big_list[2 * W.big + 1];
    if (s < lo || s >= lo + J.big_window) return false;
    fill_item(J, W.big, lo, b);
    return !(J.lex_big && lex_eligible(J, *b));
}

__device__ __forceinline__ int find_job(const int64_t *bases, int n, int64_t g) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (bases[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Flat candidate g of a group's pass: its job, destination and position in it (false
// if g falls past the pass's destinations or into another pass's).
struct BigCand {
    int job;
    int64_t i;   // position within the destination
    BigItem B;
};

__device__ __forceinline__ bool big_cand(const ExpandJob *jobs, const int64_t *job_bases, int num_jobs, int64_t g,
                                         int64_t pass, BigCand *c) {
    const int j = find_job(job_bases, num_jobs, g);
    const ExpandJob &J = jobs[j];
    const int64_t cl = g - job_bases[j];
    if (J.num_big <= 0 || cl >= J.big_rows) return false;
    const int64_t lo = pass * J.big_window;
    const int64_t s = lo + cl;  // index in the job's whole oversized candidate order
    int a = 0, b = J.num_big - 1;
    while (a < b) {
        const int mid = (a + b + 1) >> 1;
        if (J.big_list[2 * mid + 1] <= s) a = mid;
        else b = mid - 1;
    }
    const int64_t soff = J.big_list[2 * a + 1];
    if (soff > s || soff < lo || soff >= lo + J.big_window) return false;
    fill_item(J, a, lo, &c->B);
    c->i = s - soff;
    if (c->i >= c->B.n) return false;
    c->job = j;
    return true;
}

// Arc run [rs, re) (destination-local) of position i, and its arc.
__device__ __forceinline__ int32_t run_of(const ExpandJob &J, const BigItem &B, int64_t i, int64_t *rs, int64_t *re) {
    int lo = B.a0, hi = B.a1 - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (J.arc_cand_off[mid - J.arc_base] - B.c0 <= i) lo = mid;
        else hi = mid - 1;
    }
    *rs = J.arc_cand_off[lo - J.arc_base] - B.c0;
    *re = J.arc_cand_off[lo + 1 - J.arc_base] - B.c0;
    return lo;
}

}  // namespace big
}  // namespace dev
}  // namespace pmdd
