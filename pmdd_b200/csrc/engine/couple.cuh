// Method-3 coupling and DD-preparation launchers (couple.cu).
#pragma once

#include <algorithm>

#include "common.cuh"

namespace pmdd {
namespace dev {

constexpr int kCoupleThreads = 256;
constexpr int kCoupleFS = 2048;  // running-frontier points staged in shared memory for pruning

// Per-job device counters (int64 each).
enum CoupleCtr {
    kCtrF = 0,          // points of the running frontier at the front of U
    kCtrB = 1,          // survivors appended this round (may exceed room; clamped)
    kCtrResume = 2,     // first cutset node whose survivors did not fit (num_nodes: none)
    kCtrCursor = 3,     // next cutset node to hand out this round
    kCtrEvaluated = 4,  // products compared one by one (statistics)
    kCtrDone = 5,       // 1 once a product round finished every node
    kCtrValidEnd = 6,   // U slots below this index hold written points (set on overflow)
    kCtrProducts = 7,   // sum over cutset nodes of |TD_v| * |BU_v| (statistics)
    kCtrSumMax = 8,     // refilter: largest objective sum among F + this round's survivors
    kCtrWidth = 9,      // refilter: sum range of one bucket
    kCtrBuckets = 10,   // refilter: number of sum buckets
    kCtrFMax = 11,      // the running frontier is in bucket order under these three
    kCtrFWidth = 12,    //   (0: no order known)
    kCtrFBuckets = 13,
    kCtrCount = 14
};

constexpr int64_t kMaxBuckets = 65536;  // sum buckets of one refilter

struct CoupleJob {
    const void *td_pts;
    const int64_t *td_off;
    const int32_t *td_size;
    const void *bu_pts;
    const int64_t *bu_off;
    const int32_t *bu_size;
    int32_t num_nodes;
    int32_t pad0;
    void *U;            // running frontier followed by this round's survivors
    void *U_alt;        // receives the next running frontier (the buffers swap each round)
    int64_t ucap;       // points each of U / U_alt can hold
    void *sc_pts2;      // refilter scratch: ucap points (F + survivors in sum-bucket order)
    void *sc_surv;      // refilter scratch: ucap points (the survivors alone, bucket order)
    int32_t *sc_idx;    // refilter scratch: ucap ints (keep and origin flags, a byte each)
    int32_t *sc_sidx;   // refilter scratch: ucap ints (position of each sorted survivor)
    int32_t *sc_hist;   // refilter scratch: 2 * (kMaxBuckets + 1) ints (bucket counts / ends)
    int64_t *ctr;       // kCtrCount counters
};

// Bytes of device memory a coupling job with capacity ucap needs besides the counters.
inline size_t couple_bytes(int64_t ucap, int d, size_t elem) {
    const size_t pts = (static_cast<size_t>(ucap) * d * elem + 255) / 256 * 256;
    const size_t idx = (static_cast<size_t>(ucap) * 4 + 255) / 256 * 256;
    const size_t hist = (2 * (static_cast<size_t>(kMaxBuckets) + 1) * 4 + 255) / 256 * 256;
    return 4 * pts + 2 * idx + hist;
}

cudaError_t launch_build_out_csr(const int32_t *in_off, const int32_t *arc_src, const int32_t *arc_w,
                                 int32_t num_nodes, int32_t num_arcs, int32_t *out_off, int32_t *cursor,
                                 int32_t *out_head, int32_t *out_w, cudaStream_t stream);

// One coupling round for `num_jobs` jobs of one (d, wide) group.  A seed round appends,
// per cutset node, the sums of the two frontiers' per-objective and sum maximisers and
// filters them into the first running frontier; a product round streams the remaining
// products against the running frontier and re-filters frontier + survivors (survivors
// bucketed by decreasing objective sum, then one GPU-wide mark pass and a compaction).
// Either way the next running frontier lands in U_alt.
cudaError_t launch_couple_round(int d, bool wide, const CoupleJob *jobs, int num_jobs, int blocks_per_job,
                                bool seed, cudaStream_t stream);
// Once per job at the start of coupling: kCtrProducts = sum of |TD_v| * |BU_v|.
cudaError_t launch_couple_products(const CoupleJob *jobs, int num_jobs, cudaStream_t stream);

}  // namespace dev
}  // namespace pmdd
