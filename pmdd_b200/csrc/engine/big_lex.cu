// Oversized destinations of three objectives, in lexicographic order.
//
// A destination too large for a tile (tile_resident()) whose arc runs all come from
// frontiers kept in descending lexicographic order, at most ExpandJob::lex_max_arcs, is
// filtered here instead of by big.cu's sort-filter-skyline or pivot/mark passes:
//
//   big_lex_rank_kernel:   thread per candidate of the scratch pass (the flat space of
//       big_expand_kernel, which it replaces for these jobs): the candidate is its parent
//       point + arc weight; its position in the destination's lexicographic order is its
//       index in its run plus, per other run, a binary search of that run's parent
//       frontier (parent point + that arc's weight, compared with the candidate; equal
//       points: the lower run first); it is written to scratch at that position.
//       Candidates of destinations this path does not take are written in run order, as
//       big_expand_kernel writes them;
//   big_lex_merge_kernel:  destinations of more than kBigDirectArcs runs are written in run
//       order by the rank kernel and sorted by ceil(log2(runs)) rounds that merge
//       neighbouring groups of runs (thread per candidate, a binary search into the
//       sibling group), alternating between the two scratch buffers;
//   big_lex_filter_kernel: one warp per destination walks the sorted candidates 32 at a
//       time with the staircase of stair.cuh and writes the survivors to the slot in
//       order (so the destination's frontier is sorted, out_sorted = 1) -- its work is
//       linear in the candidates instead of quadratic in what the pivots leave.  If the
//       staircase outgrows kStairBig entries the warp checks each remaining candidate
//       against every point before it.
//
// Keep rule as everywhere (src/pmdd/enum/gpu/dominance_utils.cuh:10-23): of equal points
// the first in the merged order stays.
#include "big_common.cuh"
#include "kernels.cuh"
#include "scan.cuh"
#include "stair.cuh"

#include <algorithm>

namespace pmdd {
namespace dev {

namespace {

using namespace big;

constexpr int kRankThreads = 256;
constexpr int kStairBig = 256;
// staircases of one block in 32 KB of static shared memory: 8 warps (int32), 4 (int64)
template <typename T>
struct FilterCfg {
    static constexpr int kWarps = 32768 / static_cast<int>(sizeof(StairBuf<T, kStairBig>));
    static constexpr int kThreads = 32 * kWarps;
};
constexpr unsigned kAll = 0xffffffffu;

template <typename T>
__device__ __forceinline__ bool before(T a0, T a1, T a2, T b0, T b1, T b2, bool tie) {
    if (a0 != b0) return a0 > b0;
    if (a1 != b1) return a1 > b1;
    if (a2 != b2) return a2 > b2;
    return tie;
}

// Work item W's destination if pass `pass` takes it, whichever path filters it.
__device__ __forceinline__ bool big_item_any(const ExpandJob &J, const BigWork &W, int64_t pass, BigItem *b) {
    const int64_t lo = pass * J.big_window;
    const int64_t s = J.big_list[2 * W.big + 1];
    if (s < lo || s >= lo + J.big_window) return false;
    fill_item(J, W.big, lo, b);
    return true;
}

}  // namespace

template <typename T>
__global__ void __launch_bounds__(kRankThreads) big_lex_rank_kernel(const ExpandJob *__restrict__ jobs,
                                                                    const int64_t *__restrict__ job_bases,
                                                                    int num_jobs, int64_t total, int64_t pass) {
    for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < total;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        BigCand c;
        if (!big_cand(jobs, job_bases, num_jobs, g, pass, &c)) continue;
        const ExpandJob &J = jobs[c.job];
        const T *prev = static_cast<const T *>(J.prev_pts);
        int64_t rs, re;
        const int32_t a = run_of(J, c.B, c.i, &rs, &re);
        const int32_t u = J.arc_nbr[a] - J.prev_base;
        const T *src = prev + (J.prev_off[u] + (c.i - rs)) * 3;
        const int32_t *w = J.weights + static_cast<int64_t>(J.arc_wrow[a]) * 3;
        const T q0 = src[0] + static_cast<T>(w[0]), q1 = src[1] + static_cast<T>(w[1]),
                q2 = src[2] + static_cast<T>(w[2]);
        int64_t pos = c.i;
        if (J.lex_big && c.B.a1 - c.B.a0 <= kBigDirectArcs && lex_eligible(J, c.B)) {
            pos = c.i - rs;
            for (int32_t b = c.B.a0; b < c.B.a1; ++b) {
                if (b == a) continue;
                const int64_t bs = J.arc_cand_off[b - J.arc_base] - c.B.c0;
                const int64_t len = J.arc_cand_off[b + 1 - J.arc_base] - c.B.c0 - bs;
                if (len <= 0) continue;
                const T *ps = prev + J.prev_off[J.arc_nbr[b] - J.prev_base] * 3;
                const int32_t *wb = J.weights + static_cast<int64_t>(J.arc_wrow[b]) * 3;
                const bool tie = b < a;
                int64_t lo = 0, hi = len;  // points of run b before q: a prefix
                while (lo < hi) {
                    const int64_t mid = (lo + hi) >> 1;
                    const T *p = ps + mid * 3;
                    if (before<T>(p[0] + static_cast<T>(wb[0]), p[1] + static_cast<T>(wb[1]),
                                  p[2] + static_cast<T>(wb[2]), q0, q1, q2, tie))
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                pos += lo;
            }
        }
        T *dst = static_cast<T *>(J.big_pts) + (c.B.soff + pos) * 3;
        dst[0] = q0;
        dst[1] = q1;
        dst[2] = q2;
    }
}

// Merge round `round` of the lexicographic destinations with more than kBigDirectArcs
// runs: at round r the destination consists of sorted groups of 2^r consecutive runs
// (in big_pts for even r, big_pts2 for odd r); each candidate moves to its place in the
// union with its sibling group (a binary search there; equal points: the left group
// first), in the other buffer.  Thread per candidate of the scratch pass.
template <typename T>
__global__ void __launch_bounds__(kRankThreads) big_lex_merge_kernel(const ExpandJob *__restrict__ jobs,
                                                                     const int64_t *__restrict__ job_bases,
                                                                     int num_jobs, int64_t total, int64_t pass,
                                                                     int round) {
    for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < total;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        BigCand c;
        if (!big_cand(jobs, job_bases, num_jobs, g, pass, &c)) continue;
        const ExpandJob &J = jobs[c.job];
        const int K = c.B.a1 - c.B.a0;
        if (!J.lex_big || round >= lex_merge_rounds(K) || !lex_eligible(J, c.B)) continue;
        const T *src = static_cast<const T *>(round & 1 ? J.big_pts2 : J.big_pts) + c.B.soff * 3;
        T *dst = static_cast<T *>(round & 1 ? J.big_pts : J.big_pts2) + c.B.soff * 3;
        // start of run x of the destination (x <= K), destination-local
        auto st = [&](int x) -> int64_t {
            return x >= K ? c.B.n : J.arc_cand_off[c.B.a0 + x - J.arc_base] - c.B.c0;
        };
        int64_t rs, re;
        const int32_t a = run_of(J, c.B, c.i, &rs, &re);
        const int grp = (a - c.B.a0) >> round;
        const int sib = grp ^ 1;
        const int64_t my0 = st(grp << round);
        const T q0 = src[c.i * 3], q1 = src[c.i * 3 + 1], q2 = src[c.i * 3 + 2];
        int64_t cnt = 0;
        const int64_t merged0 = st((grp >> 1) << (round + 1));
        if ((sib << round) < K) {
            const int64_t lo0 = st(sib << round), hi0 = st(min((sib + 1) << round, K));
            const bool tie = sib < grp;  // the left group's equal points come first
            int64_t lo = lo0, hi = hi0;
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                const T *p = src + mid * 3;
                if (before<T>(p[0], p[1], p[2], q0, q1, q2, tie)) lo = mid + 1;
                else hi = mid;
            }
            cnt = lo - lo0;
        }
        T *o = dst + (merged0 + (c.i - my0) + cnt) * 3;
        o[0] = q0;
        o[1] = q1;
        o[2] = q2;
    }
}

template <typename T>
__global__ void __launch_bounds__(FilterCfg<T>::kThreads) big_lex_filter_kernel(const ExpandJob *__restrict__ jobs,
                                                                                const BigWork *__restrict__ work,
                                                                                int num_work, int64_t pass) {
    constexpr int kFilterWarps = FilterCfg<T>::kWarps;
    __shared__ StairBuf<T, kStairBig> bufs[kFilterWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (int wi = blockIdx.x * kFilterWarps + warp; wi < num_work; wi += gridDim.x * kFilterWarps) {
        const BigWork W = work[wi];
        const ExpandJob &J = jobs[W.job];
        BigItem B;
        if (!J.lex_big || !big_item_any(J, W, pass, &B) || !lex_eligible(J, B)) continue;
        // sorted candidates: big_pts after an even number of merge rounds, else big_pts2
        const T *cand = static_cast<const T *>(lex_merge_rounds(B.a1 - B.a0) & 1 ? J.big_pts2 : J.big_pts) + B.soff * 3;
        T *out = static_cast<T *>(J.out_pts) + B.c0 * 3;
        StairState st;
        int64_t kept = 0;
        for (int64_t c0 = 0; c0 < B.n; c0 += 32) {
            const int64_t p = c0 + lane;
            const bool valid = p < B.n;
            T q0 = 0, q1 = 0, q2 = 0;
            if (valid) {
                q0 = cand[p * 3];
                q1 = cand[p * 3 + 1];
                q2 = cand[p * 3 + 2];
            }
            bool dom = !valid;
            if (st.overflow) {
                // staircase given up: every candidate before p, chunk-mates included
                const int64_t hi = min(B.n, c0 + 32) - 1;
                for (int64_t j = 0; j < hi; ++j) {
                    if (j < p) dom |= (cand[j * 3 + 1] >= q1) & (cand[j * 3 + 2] >= q2);
                    if ((j & 31) == 31 && __all_sync(kAll, dom)) break;
                }
            } else {
                dom = stair_chunk<T, kStairBig>(bufs[warp], st, valid, q1, q2, c0 + 32 < B.n);
            }
            const unsigned keep = __ballot_sync(kAll, !dom);
            if (!dom) {
                T *o = out + (kept + __popc(keep & lt_mask)) * 3;
                o[0] = q0;
                o[1] = q1;
                o[2] = q2;
            }
            kept += __popc(keep);
        }
        if (lane == 0) {
            J.out_size[B.item] = static_cast<int32_t>(kept);
            if (J.out_sorted) J.out_sorted[B.item] = 1;
            if (J.tile_surv) atomicAdd(J.tile_surv + 1, static_cast<unsigned long long>(B.n));
        }
    }
}

cudaError_t launch_big_lex_rank(bool wide, const BigLaunch &L, cudaStream_t stream) {
    const int64_t want = (L.total + kRankThreads - 1) / kRankThreads;
    const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(L.sms) * 32)));
    if (wide) big_lex_rank_kernel<int64_t><<<grid, kRankThreads, 0, stream>>>(L.jobs, L.job_bases, L.num_jobs, L.total, L.pass);
    else big_lex_rank_kernel<int32_t><<<grid, kRankThreads, 0, stream>>>(L.jobs, L.job_bases, L.num_jobs, L.total, L.pass);
    return cudaGetLastError();
}

template <typename T>
static cudaError_t launch_filter_t(const BigLaunch &L, cudaStream_t stream) {
    using Cfg = FilterCfg<T>;
    const unsigned grid = static_cast<unsigned>(
        std::max<int64_t>(1, std::min<int64_t>((L.num_work + Cfg::kWarps - 1) / Cfg::kWarps, int64_t(L.sms) * 16)));
    big_lex_filter_kernel<T><<<grid, Cfg::kThreads, 0, stream>>>(L.jobs, L.work, L.num_work, L.pass);
    return cudaGetLastError();
}

cudaError_t launch_big_lex_merge(bool wide, const BigLaunch &L, int round, cudaStream_t stream) {
    const int64_t want = (L.total + kRankThreads - 1) / kRankThreads;
    const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(L.sms) * 32)));
    if (wide)
        big_lex_merge_kernel<int64_t><<<grid, kRankThreads, 0, stream>>>(L.jobs, L.job_bases, L.num_jobs, L.total,
                                                                         L.pass, round);
    else
        big_lex_merge_kernel<int32_t><<<grid, kRankThreads, 0, stream>>>(L.jobs, L.job_bases, L.num_jobs, L.total,
                                                                         L.pass, round);
    return cudaGetLastError();
}

cudaError_t launch_big_lex_filter(bool wide, const BigLaunch &L, cudaStream_t stream) {
    return wide ? launch_filter_t<int64_t>(L, stream) : launch_filter_t<int32_t>(L, stream);
}

}  // namespace dev
}  // namespace pmdd
