// Oversized destinations of three objectives, in lexicographic order.
//
// A destination too large for a tile (tile_resident()) whose arc runs all come from
// frontiers kept in descending lexicographic order, at most kBigLexMaxArcs of them, is
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
//   big_lex_seg_*_kernel:  the sorted candidates are walked with the staircase of
//       stair.cuh in segments of kSeg, one warp each, the segments joined by prefix
//       staircases, and the survivors written to the slot in order (so the destination's
//       frontier is sorted, out_sorted = 1) -- work linear in the candidates instead of
//       quadratic in what the pivots leave, spread over a warp per segment.
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

// ---------------------------------------------------------------- segmented filter
// A destination's sorted candidates are cut into segments of kSeg.  A candidate is
// dominated iff it is dominated within its segment or by the staircase of all earlier
// segments, so:
//   seg_local:  warp per segment walks it with a staircase from empty (local keep flags
//               in big_idx) and stores the segment's final staircase SK_s;
//   seg_prefix: warp per destination merges SK_0, SK_1, ... in order into the prefix
//               staircases P_1, P_2, ... (P_s: everything before segment s);
//   seg_final:  warp per segment drops its locally kept candidates that P_s dominates
//               and counts the rest;
//   seg_write:  warp per segment writes its survivors after those of earlier segments,
//               so the destination's frontier comes out in order.
// Scratch of a destination (pass offset soff, n candidates, S segments): keep flags
// big_idx[soff + i]; big_surv_idx[soff + s*kSeg] = survivors of segment s, and for a
// full segment t < S-1 also [+1] = |SK_t|, [+2] = |P_{t+1}|; big_surv_idx[soff + 3] = 1
// when a staircase outgrew kStairBig (then one warp walks the whole destination, checking
// every earlier candidate once the staircase is given up); segment t's 3*kSeg values of
// big_surv hold SK_t and P_{t+1}.
constexpr int kSeg = 1024;

template <typename T>
struct SegView {
    const T *cand;   // sorted candidates, 3 values each
    int32_t *flag;
    int32_t *meta;
    T *reg;          // segment t's region: reg + t * kSeg * 3
    int64_t n;
    int S;
    __device__ T *sk1(int t) const { return reg + static_cast<int64_t>(t) * kSeg * 3; }
    __device__ T *sk2(int t) const { return sk1(t) + kStairBig; }
    __device__ T *p1(int t) const { return sk1(t) + 2 * kStairBig; }
    __device__ T *p2(int t) const { return sk1(t) + 3 * kStairBig; }
    __device__ bool overflow() const { return S > 1 && meta[3] != 0; }
};

template <typename T>
__device__ __forceinline__ bool seg_view(const ExpandJob &J, const BigWork &W, int64_t pass, SegView<T> *v) {
    BigItem B;
    if (!J.lex_big || !big_item_any(J, W, pass, &B) || !lex_eligible(J, B)) return false;
    v->cand = static_cast<const T *>(lex_merge_rounds(B.a1 - B.a0) & 1 ? J.big_pts2 : J.big_pts) + B.soff * 3;
    v->flag = J.big_idx + B.soff;
    v->meta = J.big_surv_idx + B.soff;
    v->reg = static_cast<T *>(J.big_surv) + B.soff * 3;
    v->n = B.n;
    v->S = static_cast<int>((B.n + kSeg - 1) / kSeg);
    return true;
}

// One warp: candidates [b, e) against the points before them in [lo, e) (pairwise).
template <typename T>
__device__ void pairwise_walk(const T *cand, int32_t *flag, int64_t lo, int64_t b, int64_t e, int lane) {
    for (int64_t c0 = b; c0 < e; c0 += 32) {
        const int64_t p = c0 + lane;
        const bool valid = p < e;
        T q1 = 0, q2 = 0;
        if (valid) {
            q1 = cand[p * 3 + 1];
            q2 = cand[p * 3 + 2];
        }
        bool dom = !valid;
        const int64_t hi = min(e, c0 + 32) - 1;
        for (int64_t j = lo; j < hi; ++j) {
            if (j < p) dom |= (cand[j * 3 + 1] >= q1) & (cand[j * 3 + 2] >= q2);
            if (((j - lo) & 31) == 31 && __all_sync(kAll, dom)) break;
        }
        if (valid) flag[p] = dom ? 0 : 1;
    }
}

// One warp: candidates [b, e) with a staircase from empty (keep flags); returns false if
// the staircase outgrew kStairBig (the rest of [b, e) is then checked pairwise against
// [b, e)).  `keep_last` keeps the staircase after the last chunk.
template <typename T>
__device__ bool stair_walk(const T *cand, int32_t *flag, int64_t b, int64_t e, bool keep_last,
                           StairBuf<T, kStairBig> &buf, StairState &st, int lane) {
    for (int64_t c0 = b; c0 < e; c0 += 32) {
        const int64_t p = c0 + lane;
        const bool valid = p < e;
        if (st.overflow) {
            pairwise_walk<T>(cand, flag, b, c0, e, lane);
            return false;
        }
        T q1 = 0, q2 = 0;
        if (valid) {
            q1 = cand[p * 3 + 1];
            q2 = cand[p * 3 + 2];
        }
        const bool dom = stair_chunk<T, kStairBig>(buf, st, valid, q1, q2, keep_last || c0 + 32 < e);
        if (valid) flag[p] = dom ? 0 : 1;
    }
    return !st.overflow;
}

template <typename T>
__global__ void __launch_bounds__(FilterCfg<T>::kThreads) big_lex_seg_local_kernel(const ExpandJob *__restrict__ jobs,
                                                                                   const BigWork *__restrict__ work,
                                                                                   int64_t pass) {
    constexpr int NW = FilterCfg<T>::kWarps;
    __shared__ StairBuf<T, kStairBig> bufs[NW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const BigWork W = work[blockIdx.x];
    SegView<T> v;
    if (!seg_view<T>(jobs[W.job], W, pass, &v)) return;
    const int s = blockIdx.y * NW + warp;
    if (s >= v.S) return;
    const int64_t b = static_cast<int64_t>(s) * kSeg, e = min(v.n, b + kSeg);
    StairState st;
    const bool ok = stair_walk<T>(v.cand, v.flag, b, e, s < v.S - 1, bufs[warp], st, lane);
    if (s < v.S - 1) {
        if (!ok) {
            if (lane == 0) v.meta[3] = 1;
            return;
        }
        for (int i = lane; i < st.m; i += 32) {
            v.sk1(s)[i] = bufs[warp].v1[st.cur][i];
            v.sk2(s)[i] = bufs[warp].v2[st.cur][i];
        }
        if (lane == 0) v.meta[static_cast<int64_t>(s) * kSeg + 1] = st.m;
    }
}

template <typename T>
__global__ void __launch_bounds__(FilterCfg<T>::kThreads) big_lex_seg_prefix_kernel(const ExpandJob *__restrict__ jobs,
                                                                                    const BigWork *__restrict__ work,
                                                                                    int num_work, int64_t pass) {
    constexpr int NW = FilterCfg<T>::kWarps;
    __shared__ StairBuf<T, kStairBig> bufs[NW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wi = blockIdx.x * NW + warp;
    if (wi >= num_work) return;
    const BigWork W = work[wi];
    SegView<T> v;
    if (!seg_view<T>(jobs[W.job], W, pass, &v) || v.S <= 1 || v.overflow()) return;
    StairState P;  // the staircase of everything before the next segment
    for (int t = 0; t + 1 < v.S; ++t) {
        const int m = v.meta[static_cast<int64_t>(t) * kSeg + 1];
        for (int c0 = 0; c0 < m; c0 += 32) {
            const bool valid = c0 + lane < m;
            T e1 = 0, e2 = 0;
            if (valid) {
                e1 = v.sk1(t)[c0 + lane];
                e2 = v.sk2(t)[c0 + lane];
            }
            (void)stair_chunk<T, kStairBig>(bufs[warp], P, valid, e1, e2, true);
            if (P.overflow) {
                if (lane == 0) v.meta[3] = 1;
                return;
            }
        }
        for (int i = lane; i < P.m; i += 32) {
            v.p1(t)[i] = bufs[warp].v1[P.cur][i];
            v.p2(t)[i] = bufs[warp].v2[P.cur][i];
        }
        if (lane == 0) v.meta[static_cast<int64_t>(t) * kSeg + 2] = P.m;
    }
}

template <typename T>
__global__ void __launch_bounds__(FilterCfg<T>::kThreads) big_lex_seg_final_kernel(const ExpandJob *__restrict__ jobs,
                                                                                   const BigWork *__restrict__ work,
                                                                                   int64_t pass) {
    constexpr int NW = FilterCfg<T>::kWarps;
    __shared__ StairBuf<T, kStairBig> bufs[NW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const BigWork W = work[blockIdx.x];
    SegView<T> v;
    if (!seg_view<T>(jobs[W.job], W, pass, &v)) return;
    const int s = blockIdx.y * NW + warp;
    if (s >= v.S) return;
    if (v.overflow()) {
        // a staircase outgrew its buffer: one warp walks the whole destination again
        if (s != 0) return;
        StairState st;
        (void)stair_walk<T>(v.cand, v.flag, 0, v.n, false, bufs[warp], st, lane);
        for (int t = 0; t < v.S; ++t) {
            const int64_t b = static_cast<int64_t>(t) * kSeg, e = min(v.n, b + kSeg);
            int cnt = 0;
            for (int64_t c0 = b; c0 < e; c0 += 32)
                cnt += __popc(__ballot_sync(kAll, c0 + lane < e && v.flag[c0 + lane] != 0));
            if (lane == 0) v.meta[b] = cnt;
        }
        return;
    }
    const int64_t b = static_cast<int64_t>(s) * kSeg, e = min(v.n, b + kSeg);
    int m = 0;
    if (s > 0) {  // P_s, kept in the region of segment s-1
        m = v.meta[static_cast<int64_t>(s - 1) * kSeg + 2];
        for (int i = lane; i < m; i += 32) {
            bufs[warp].v1[0][i] = v.p1(s - 1)[i];
            bufs[warp].v2[0][i] = v.p2(s - 1)[i];
        }
        __syncwarp();
    }
    int cnt = 0;
    for (int64_t c0 = b; c0 < e; c0 += 32) {
        const int64_t p = c0 + lane;
        bool keep = p < e && v.flag[p] != 0;
        if (keep && m > 0) {
            const T q1 = v.cand[p * 3 + 1], q2 = v.cand[p * 3 + 2];
            int lo = 0, hi = m;  // entries with objective 1 >= q1
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (bufs[warp].v1[0][mid] >= q1) lo = mid + 1;
                else hi = mid;
            }
            if (lo > 0 && bufs[warp].v2[0][lo - 1] >= q2) {
                keep = false;
                v.flag[p] = 0;
            }
        }
        cnt += __popc(__ballot_sync(kAll, keep));
    }
    if (lane == 0) v.meta[b] = cnt;
}

template <typename T>
__global__ void __launch_bounds__(FilterCfg<T>::kThreads) big_lex_seg_write_kernel(const ExpandJob *__restrict__ jobs,
                                                                                   const BigWork *__restrict__ work,
                                                                                   int64_t pass) {
    constexpr int NW = FilterCfg<T>::kWarps;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    const BigWork W = work[blockIdx.x];
    const ExpandJob &J = jobs[W.job];
    SegView<T> v;
    if (!seg_view<T>(J, W, pass, &v)) return;
    const int s = blockIdx.y * NW + warp;
    if (s >= v.S) return;
    int64_t before = 0;  // survivors of the earlier segments
    for (int t = lane; t < s; t += 32) before += v.meta[static_cast<int64_t>(t) * kSeg];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) before += __shfl_xor_sync(kAll, before, o);
    BigItem B;
    fill_item(J, W.big, pass * J.big_window, &B);
    T *out = static_cast<T *>(J.out_pts) + B.c0 * 3;
    const int64_t b = static_cast<int64_t>(s) * kSeg, e = min(v.n, b + kSeg);
    int64_t kept = before;
    for (int64_t c0 = b; c0 < e; c0 += 32) {
        const int64_t p = c0 + lane;
        const bool keep = p < e && v.flag[p] != 0;
        const unsigned k = __ballot_sync(kAll, keep);
        if (keep) {
            T *o = out + (kept + __popc(k & lt_mask)) * 3;
            o[0] = v.cand[p * 3];
            o[1] = v.cand[p * 3 + 1];
            o[2] = v.cand[p * 3 + 2];
        }
        kept += __popc(k);
    }
    if (s == v.S - 1 && lane == 0) {
        J.out_size[B.item] = static_cast<int32_t>(kept);
        if (J.out_sorted) J.out_sorted[B.item] = 1;
        if (J.tile_surv) atomicAdd(J.tile_surv + 1, static_cast<unsigned long long>(v.n));
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
    if (L.num_work <= 0) return cudaSuccess;
    const int64_t max_seg = std::max<int64_t>(1, (L.max_n + kSeg - 1) / kSeg);
    const dim3 grid(static_cast<unsigned>(L.num_work), static_cast<unsigned>((max_seg + Cfg::kWarps - 1) / Cfg::kWarps));
    const unsigned pgrid = static_cast<unsigned>((L.num_work + Cfg::kWarps - 1) / Cfg::kWarps);
    big_lex_seg_local_kernel<T><<<grid, Cfg::kThreads, 0, stream>>>(L.jobs, L.work, L.pass);
    big_lex_seg_prefix_kernel<T><<<pgrid, Cfg::kThreads, 0, stream>>>(L.jobs, L.work, L.num_work, L.pass);
    big_lex_seg_final_kernel<T><<<grid, Cfg::kThreads, 0, stream>>>(L.jobs, L.work, L.pass);
    big_lex_seg_write_kernel<T><<<grid, Cfg::kThreads, 0, stream>>>(L.jobs, L.work, L.pass);
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
