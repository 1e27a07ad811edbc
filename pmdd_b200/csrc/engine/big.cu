// Oversized destinations (those tile_resident() rejects).  Their candidates are
// materialised in scratch, then filtered; everything works on one scratch pass at a time
// (see ExpandJob::big_window).
//
//   big_expand_kernel: thread per candidate over the pass's flat candidate space, so a
//       destination of n candidates gets ~n threads whatever the other sizes are;
//   big_sfs_kernel:    destinations below ExpandJob::big_mark_min candidates: one block
//       each runs the sort-filter-skyline of sfs.cuh, which compares each point only
//       with the maxima found so far; many such destinations keep the GPU busy side by
//       side;
//   big_plan_kernel .. big_write_kernel: destinations of big_mark_min candidates and
//       more, each spread over every SM.  The plan lists their 256-candidate chunks.
//       big_pivot_kernel picks each destination's pivots (the candidates of largest
//       objective sum, from a sorted sample of sums);
//       big_prefilter_kernel drops every candidate a pivot dominates; big_compact_kernel
//       packs the rest, in candidate order; big_rplan_kernel lists their chunks; one
//       big_mark_kernel block per chunk streams the remaining rows through shared memory
//       with warp-uniform broadcast reads and stops once its rows are all dominated (of
//       equal points the first stays); one big_write_kernel block per destination
//       compacts the survivors into the slot.  The pivots leave the pairwise sweep a
//       fraction of the candidates, and it costs the square of what it is given.
//
// With the pivots the GPU-wide pass wins from the smallest oversized destinations up (on
// the batched knapsack / set-packing stream as on single 5-objective TSPs), so by default
// it takes every destination above kSmallMax candidates; SFS blocks keep those that leave
// the tiles for their arc count, and whatever a fixed or tuned crossover assigns them.
#include "big_common.cuh"
#include "kernels.cuh"
#include "sfs.cuh"

#include <algorithm>

namespace pmdd {
namespace dev {

namespace {

using namespace big;

constexpr int kFlatThreads = 256;
constexpr int kMarkThreads = 256;
constexpr int kWriteThreads = 512;
constexpr int kPlanThreads = 1024;
constexpr unsigned kFull = 0xffffffffu;

template <int D, typename T>
struct MarkCfg {
    static constexpr int kTile = 32768 / static_cast<int>(sizeof(PackedPt<D, T>));  // points per shared tile
};

// The destinations that take the mark path in one pass.  Destination h is work item
// work_idx[h]; its candidates form chunks [chunk_base[h], chunk_base[h + 1]) of 256, its
// piv_count[h] pivots sit in big_surv / big_surv_idx, the r_count[h] candidates no pivot
// dominates sit in big_pts2 and form chunks [rchunk_base[h], rchunk_base[h + 1]).
struct MarkPlan {
    int32_t count;
    int32_t pad;
    int64_t total;   // chunks over all candidates
    int64_t rtotal;  // chunks over the candidates left by the pivots
};

struct PlanArrays {
    int32_t *work_idx;     // [cap]
    int64_t *chunk_base;   // [cap + 1]
    int64_t *rchunk_base;  // [cap + 1]
    int64_t *r_count;      // [cap]
    int32_t *piv_count;    // [cap]
};

__host__ __device__ __forceinline__ size_t plan_round(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }

__device__ __forceinline__ PlanArrays plan_arrays(const MarkPlan *plan, int cap) {
    char *p = reinterpret_cast<char *>(const_cast<MarkPlan *>(plan)) + 256;
    const size_t c = static_cast<size_t>(cap);
    PlanArrays A;
    A.work_idx = reinterpret_cast<int32_t *>(p);
    p += plan_round(c * 4);
    A.chunk_base = reinterpret_cast<int64_t *>(p);
    p += plan_round((c + 1) * 8);
    A.rchunk_base = reinterpret_cast<int64_t *>(p);
    p += plan_round((c + 1) * 8);
    A.r_count = reinterpret_cast<int64_t *>(p);
    p += plan_round(c * 8);
    A.piv_count = reinterpret_cast<int32_t *>(p);
    return A;
}

// The destination of mark-path chunk b (chunk bases `base` over plan->count destinations).
__device__ __forceinline__ int chunk_owner(const int64_t *base, int count, int64_t b) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (base[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

}  // namespace

size_t big_plan_bytes(int cap) {
    const size_t c = static_cast<size_t>(cap);
    return 256 + plan_round(c * 4) + 2 * plan_round((c + 1) * 8) + plan_round(c * 8) + plan_round(c * 4);
}

// Materialise the oversized candidates of one pass (AoS, D values each).
template <int D, typename T>
__global__ void __launch_bounds__(kFlatThreads) big_expand_kernel(const ExpandJob *__restrict__ jobs,
                                                                  const int64_t *__restrict__ job_bases, int num_jobs,
                                                                  int64_t total, int64_t pass) {
    for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < total;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        BigCand c;
        if (!big_cand(jobs, job_bases, num_jobs, g, pass, &c)) continue;
        const ExpandJob &J = jobs[c.job];
        int64_t rs, re;
        const int32_t a = run_of(J, c.B, c.i, &rs, &re);
        const int32_t u = J.arc_nbr[a] - J.prev_base;
        const T *src = static_cast<const T *>(J.prev_pts) + (J.prev_off[u] + (c.i - rs)) * D;
        const int32_t *w = J.weights + static_cast<int64_t>(J.arc_wrow[a]) * D;
        T *dst = static_cast<T *>(J.big_pts) + (c.B.soff + c.i) * D;
#pragma unroll
        for (int o = 0; o < D; ++o) dst[o] = src[o] + static_cast<T>(w[o]);
    }
}

// One block: the chunk list of this pass's mark-path destinations (at most `cap`).
__global__ void __launch_bounds__(kPlanThreads) big_plan_kernel(const ExpandJob *__restrict__ jobs,
                                                                const BigWork *__restrict__ work, int num_work,
                                                                int64_t pass, MarkPlan *plan, int cap) {
    __shared__ int64_t warp_buf[32];
    __shared__ int64_t s_total;
    const PlanArrays A = plan_arrays(plan, cap);
    int32_t *work_idx = A.work_idx;
    int64_t *chunk_base = A.chunk_base;
    int64_t chunks = 0, count = 0;
    for (int b0 = 0; b0 < num_work; b0 += kPlanThreads) {
        const int w = b0 + threadIdx.x;
        int64_t nch = 0;
        if (w < num_work) {
            const ExpandJob &J = jobs[work[w].job];
            BigItem B;
            if (big_item(J, work[w], pass, &B) && B.n >= J.big_mark_min) nch = (B.n + kMarkThreads - 1) / kMarkThreads;
        }
        const int64_t sel = nch > 0 ? 1 : 0;
        const int64_t pos = count + block_exclusive_scan<int64_t, kPlanThreads>(sel, warp_buf, &s_total);
        const int64_t nsel = s_total;
        const int64_t cb = chunks + block_exclusive_scan<int64_t, kPlanThreads>(nch, warp_buf, &s_total);
        const int64_t nchunks = s_total;
        if (sel && pos < cap) {
            work_idx[pos] = w;
            chunk_base[pos] = cb;
        }
        count += nsel;
        chunks += nchunks;
    }
    if (threadIdx.x == 0) {
        if (count > cap) {  // cap is an upper bound by construction; never drop work silently
            atomicOr(jobs[0].err, kErrBounds);
            count = cap;
            chunks = cap > 0 ? chunk_base[cap - 1] : 0;
            plan->total = 0;
        } else {
            plan->total = chunks;
        }
        chunk_base[count] = chunks;
        plan->count = static_cast<int32_t>(count);
    }
}

// Sweep of tile points [a, b) that come before every lane's candidate: >= dominates.
template <int D, typename T>
__device__ __forceinline__ bool sweep_before(const PackedPt<D, T> *ys, int a, int b, const T (&p)[D], bool dom) {
    int j = a, it = 0;
    for (; j + 4 <= b; j += 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) dom |= ge_all<D, T>(ys[j + u], p);
        if ((++it & 7) == 0 && __all_sync(kFull, dom)) return true;
    }
    for (; j < b; ++j) dom |= ge_all<D, T>(ys[j], p);
    return dom;
}

// Sweep of tile points [a, b) that come after every lane's candidate: >= and different.
template <int D, typename T>
__device__ __forceinline__ bool sweep_after(const PackedPt<D, T> *ys, int a, int b, const T (&p)[D], bool dom) {
    int j = a, it = 0;
    for (; j + 4 <= b; j += 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const PackedPt<D, T> c = ys[j + u];
            dom |= ge_all<D, T>(c, p) && !eq_all<D, T>(c, p);
        }
        if ((++it & 7) == 0 && __all_sync(kFull, dom)) return true;
    }
    for (; j < b; ++j) {
        const PackedPt<D, T> c = ys[j];
        dom |= ge_all<D, T>(c, p) && !eq_all<D, T>(c, p);
    }
    return dom;
}

// Pivots: the candidates of largest objective sum, about pivot_target(n, rule) of a destination's
// n.  A candidate that a pivot dominates is dropped at once.  Whatever dominates a remaining
// candidate is itself remaining (a pivot dominating the dominator would dominate the
// candidate as well, equal points included), so the exact pairwise sweep then runs over the
// remaining candidates only: on 5-objective TSP destinations about a quarter of them.
constexpr int kPivotThreads = 1024;
constexpr int kPivotSample = 4096;
constexpr int kPivotMax = 8192;
constexpr int kCompactThreads = 1024;

__device__ __forceinline__ int64_t pivot_target(int64_t n, int rule) {
    const int64_t t = rule == 1 ? static_cast<int64_t>(4.0 * sqrt(static_cast<double>(n))) : n / 64;
    const int64_t lo = rule == 1 ? 32 : 512;
    return t < lo ? lo : (t > 4096 ? 4096 : t);
}

// Objective sum as the pivot ranking key; it wraps for int64 objectives, which changes only
// the choice of pivots, never the result.
template <int D, typename T>
__device__ __forceinline__ long long pivot_key(const T *p) {
    unsigned long long s = 0;
#pragma unroll
    for (int o = 0; o < D; ++o) s += static_cast<unsigned long long>(static_cast<long long>(p[o]));
    return static_cast<long long>(s);
}

// One block per mark-path destination: the sums of an even sample of up to 4096 candidates,
// sorted, give the threshold of the pivot_target(n, rule) largest; the candidates at or above it
// (the first kPivotMax in candidate order) are copied with their positions to the
// destination's big_surv / big_surv_idx rows.
template <int D, typename T>
__global__ void __launch_bounds__(kPivotThreads) big_pivot_kernel(const ExpandJob *__restrict__ jobs,
                                                                  const BigWork *__restrict__ work, int64_t pass,
                                                                  const MarkPlan *__restrict__ plan, int cap) {
    __shared__ long long key[kPivotSample];
    __shared__ int32_t warp_buf[32];
    __shared__ int32_t s_total;
    const int h = blockIdx.x;
    if (h >= plan->count) return;
    const PlanArrays A = plan_arrays(plan, cap);
    const BigWork W = work[A.work_idx[h]];
    const ExpandJob &J = jobs[W.job];
    BigItem B;
    big_item(J, W, pass, &B);
    const int64_t n = B.n;
    if (n >= 0x7fffffffLL) {  // positions are int32: no pivots, every candidate stays
        if (threadIdx.x == 0) A.piv_count[h] = 0;
        return;
    }
    const T *P = static_cast<const T *>(J.big_pts) + B.soff * D;
    T *PV = static_cast<T *>(J.big_surv) + B.soff * D;
    int32_t *PI = J.big_surv_idx + B.soff;
    const int m = n < kPivotSample ? static_cast<int>(n) : kPivotSample;
    int msz = 1;
    while (msz < m) msz <<= 1;
    constexpr long long kLowest = -0x7fffffffffffffffLL - 1;
    for (int k = threadIdx.x; k < msz; k += kPivotThreads)
        key[k] = k < m ? pivot_key<D, T>(P + (static_cast<int64_t>(k) * n / m) * D) : kLowest;
    __syncthreads();
    for (int k = 2; k <= msz; k <<= 1)  // bitonic sort, descending
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < msz; i += kPivotThreads) {
                const int q = i ^ j;
                if (q > i) {
                    const long long a = key[i], b = key[q];
                    if (((i & k) == 0) == (a < b)) {
                        key[i] = b;
                        key[q] = a;
                    }
                }
            }
            __syncthreads();
        }
    int64_t r = (static_cast<int64_t>(m) * pivot_target(n, J.pivot_rule) + n - 1) / n - 1;
    r = r < 0 ? 0 : (r >= m ? m - 1 : r);
    const long long tau = key[r];
    int32_t carry = 0;
    for (int64_t b0 = 0; b0 < n && carry < kPivotMax; b0 += kPivotThreads) {
        const int64_t i = b0 + threadIdx.x;
        const int32_t sel = (i < n && pivot_key<D, T>(P + i * D) >= tau) ? 1 : 0;
        const int32_t ex = block_exclusive_scan<int32_t, kPivotThreads>(sel, warp_buf, &s_total);
        const int32_t pos = carry + ex;
        if (sel && pos < kPivotMax) {
#pragma unroll
            for (int o = 0; o < D; ++o) PV[static_cast<int64_t>(pos) * D + o] = P[i * D + o];
            PI[pos] = static_cast<int32_t>(i);
        }
        carry += s_total;
    }
    if (threadIdx.x == 0) A.piv_count[h] = carry < kPivotMax ? carry : kPivotMax;
}

// One block per 256-candidate chunk (grid: an upper bound; extra blocks leave): flags, in
// the keep bytes, the candidates no pivot dominates (of equal points the earlier one
// dominates).
template <int D, typename T>
__global__ void __launch_bounds__(kMarkThreads) big_prefilter_kernel(const ExpandJob *__restrict__ jobs,
                                                                     const BigWork *__restrict__ work, int64_t pass,
                                                                     const MarkPlan *__restrict__ plan, int cap) {
    constexpr int TY = MarkCfg<D, T>::kTile;
    __shared__ PackedPt<D, T> ys[TY];
    __shared__ int32_t yi[TY];
    const int64_t b = blockIdx.x;
    if (b >= plan->total) return;
    const PlanArrays A = plan_arrays(plan, cap);
    const int h = chunk_owner(A.chunk_base, plan->count, b);
    const BigWork W = work[A.work_idx[h]];
    const ExpandJob &J = jobs[W.job];
    BigItem B;
    big_item(J, W, pass, &B);
    const T *P = static_cast<const T *>(J.big_pts) + B.soff * D;
    const T *PV = static_cast<const T *>(J.big_surv) + B.soff * D;
    const int32_t *PI = J.big_surv_idx + B.soff;
    uint8_t *flag = reinterpret_cast<uint8_t *>(J.big_idx) + B.soff;
    const int npiv = A.piv_count[h];
    const int64_t i = (b - A.chunk_base[h]) * kMarkThreads + threadIdx.x;
    const bool valid = i < B.n;
    T p[D];
#pragma unroll
    for (int o = 0; o < D; ++o) p[o] = valid ? P[i * D + o] : T(0);
    bool dom = !valid;
    for (int t0 = 0; t0 < npiv; t0 += TY) {
        const int cnt = npiv - t0 < TY ? npiv - t0 : TY;
        for (int k = threadIdx.x; k < cnt; k += kMarkThreads) {
            ys[k] = load_global_pt<D, T>(PV, t0 + k);
            yi[k] = PI[t0 + k];
        }
        __syncthreads();
        if (!__all_sync(kFull, dom)) {
            for (int j = 0; j < cnt; ++j) {
                const PackedPt<D, T> c = ys[j];
                dom |= ge_all<D, T>(c, p) && (yi[j] < i || !eq_all<D, T>(c, p));
                if ((j & 31) == 31 && __all_sync(kFull, dom)) break;
            }
        }
        if (__syncthreads_and(dom)) break;  // also: the tile may be overwritten now
    }
    if (valid) flag[i] = dom ? 0 : 1;
}

// One block per mark-path destination: the flagged candidates, in candidate order, into
// the destination's big_pts2 rows.
template <int D, typename T>
__global__ void __launch_bounds__(kCompactThreads) big_compact_kernel(const ExpandJob *__restrict__ jobs,
                                                                      const BigWork *__restrict__ work, int64_t pass,
                                                                      const MarkPlan *__restrict__ plan, int cap) {
    __shared__ int32_t warp_buf[32];
    __shared__ int32_t s_total;
    const int h = blockIdx.x;
    if (h >= plan->count) return;
    const PlanArrays A = plan_arrays(plan, cap);
    const BigWork W = work[A.work_idx[h]];
    const ExpandJob &J = jobs[W.job];
    BigItem B;
    big_item(J, W, pass, &B);
    const T *P = static_cast<const T *>(J.big_pts) + B.soff * D;
    T *R = static_cast<T *>(J.big_pts2) + B.soff * D;
    const uint8_t *flag = reinterpret_cast<const uint8_t *>(J.big_idx) + B.soff;
    int64_t carry = 0;
    for (int64_t b0 = 0; b0 < B.n; b0 += kCompactThreads) {
        const int64_t i = b0 + threadIdx.x;
        const int32_t k = i < B.n ? flag[i] : 0;
        const int32_t ex = block_exclusive_scan<int32_t, kCompactThreads>(k, warp_buf, &s_total);
        if (k) {
#pragma unroll
            for (int o = 0; o < D; ++o) R[(carry + ex) * D + o] = P[i * D + o];
        }
        carry += s_total;
    }
    if (threadIdx.x == 0) A.r_count[h] = carry;
}

// One block: the 256-row chunks of the pivot-filtered rows.
__global__ void __launch_bounds__(kPlanThreads) big_rplan_kernel(MarkPlan *plan, int cap) {
    __shared__ int64_t warp_buf[32];
    __shared__ int64_t s_total;
    const PlanArrays A = plan_arrays(plan, cap);
    const int count = plan->count;
    int64_t chunks = 0;
    for (int b0 = 0; b0 < count; b0 += kPlanThreads) {
        const int h = b0 + threadIdx.x;
        const int64_t nch = h < count ? (A.r_count[h] + kMarkThreads - 1) / kMarkThreads : 0;
        const int64_t cb = chunks + block_exclusive_scan<int64_t, kPlanThreads>(nch, warp_buf, &s_total);
        if (h < count) A.rchunk_base[h] = cb;
        chunks += s_total;
    }
    if (threadIdx.x == 0) {
        A.rchunk_base[count] = chunks;
        plan->rtotal = chunks;
    }
}

// One block per 256 pivot-filtered rows (grid: an upper bound; extra blocks leave): each
// row streams all rows of its destination through shared memory with warp-uniform broadcast
// reads and stops once its block's rows are all dominated.  Rows keep candidate order, so a
// row before the warp's 32 dominates on >= alone, one after them only when it also differs
// (of equal points the first stays).
template <int D, typename T>
__global__ void __launch_bounds__(kMarkThreads) big_mark_kernel(const ExpandJob *__restrict__ jobs,
                                                                const BigWork *__restrict__ work, int64_t pass,
                                                                const MarkPlan *__restrict__ plan, int cap) {
    constexpr int TY = MarkCfg<D, T>::kTile;
    __shared__ PackedPt<D, T> ys[TY];
    const int64_t b = blockIdx.x;
    if (b >= plan->rtotal) return;
    const PlanArrays A = plan_arrays(plan, cap);
    const int h = chunk_owner(A.rchunk_base, plan->count, b);
    const BigWork W = work[A.work_idx[h]];
    const ExpandJob &J = jobs[W.job];
    BigItem B;
    big_item(J, W, pass, &B);  // the plan only lists destinations of this pass
    const int64_t n = A.r_count[h];
    const T *R = static_cast<const T *>(J.big_pts2) + B.soff * D;
    uint8_t *keep = reinterpret_cast<uint8_t *>(J.big_idx) + B.soff;
    const int64_t base = (b - A.rchunk_base[h]) * kMarkThreads;
    const int64_t i = base + threadIdx.x;
    const int64_t w0 = base + (threadIdx.x & ~31);
    const bool valid = i < n;
    T p[D];
#pragma unroll
    for (int o = 0; o < D; ++o) p[o] = valid ? R[i * D + o] : T(0);
    bool dom = !valid;
    for (int64_t t0 = 0; t0 < n; t0 += TY) {
        const int cnt = static_cast<int>(n - t0 < TY ? n - t0 : TY);
        for (int k = threadIdx.x; k < cnt; k += kMarkThreads) ys[k] = load_global_pt<D, T>(R, t0 + k);
        __syncthreads();
        if (!__all_sync(kFull, dom)) {
            const int64_t bb = w0 - t0, aa = w0 + 32 - t0;
            const int b_end = static_cast<int>(bb < 0 ? 0 : (bb > cnt ? cnt : bb));
            const int a_beg = static_cast<int>(aa < 0 ? 0 : (aa > cnt ? cnt : aa));
            dom = sweep_before<D, T>(ys, 0, b_end, p, dom);
            if (!__all_sync(kFull, dom)) {
                for (int j = b_end; j < a_beg; ++j) {  // the warp's own rows
                    const PackedPt<D, T> c = ys[j];
                    dom |= ge_all<D, T>(c, p) && (t0 + j < i || !eq_all<D, T>(c, p));
                }
                dom = sweep_after<D, T>(ys, a_beg, cnt, p, dom);
            }
        }
        if (__syncthreads_and(dom)) break;  // also: the tile may be overwritten now
    }
    if (valid) keep[i] = dom ? 0 : 1;
}

// One block per planned destination (grid: `cap`; extra blocks leave): the kept rows, in
// candidate order, into the destination's slot.
template <int D, typename T>
__global__ void __launch_bounds__(kWriteThreads) big_write_kernel(const ExpandJob *__restrict__ jobs,
                                                                  const BigWork *__restrict__ work, int64_t pass,
                                                                  const MarkPlan *__restrict__ plan, int cap) {
    __shared__ int32_t warp_buf[32];
    __shared__ int32_t s_total;
    if (static_cast<int>(blockIdx.x) >= plan->count) return;
    const PlanArrays A = plan_arrays(plan, cap);
    const BigWork W = work[A.work_idx[blockIdx.x]];
    const ExpandJob &J = jobs[W.job];
    BigItem B;
    big_item(J, W, pass, &B);
    const int64_t n = A.r_count[blockIdx.x];
    const T *R = static_cast<const T *>(J.big_pts2) + B.soff * D;
    const uint8_t *keep = reinterpret_cast<const uint8_t *>(J.big_idx) + B.soff;
    T *out = static_cast<T *>(J.out_pts) + B.c0 * D;
    int64_t carry = 0;
    for (int64_t b0 = 0; b0 < n; b0 += kWriteThreads) {
        const int64_t i = b0 + threadIdx.x;
        const int32_t k = i < n ? keep[i] : 0;
        const int32_t ex = block_exclusive_scan<int32_t, kWriteThreads>(k, warp_buf, &s_total);
        if (k) {
#pragma unroll
            for (int o = 0; o < D; ++o) out[(carry + ex) * D + o] = R[i * D + o];
        }
        carry += s_total;
    }
    if (threadIdx.x == 0) J.out_size[B.item] = static_cast<int32_t>(carry);
}

// Destinations below big_mark_min candidates: one block each.
template <int D, typename T>
__global__ void __launch_bounds__(SfsSmallCfg<D, T>::kThreads) big_sfs_kernel(const ExpandJob *__restrict__ jobs,
                                                                         const BigWork *__restrict__ work,
                                                                         const int32_t *__restrict__ order,
                                                                         int64_t pass) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const BigWork W = work[order ? order[blockIdx.x] : blockIdx.x];
    const ExpandJob &J = jobs[W.job];
    BigItem B;
    if (!big_item(J, W, pass, &B) || B.n >= J.big_mark_min) return;
    SfsScratch<T> s;
    s.P2 = static_cast<T *>(J.big_pts2) + B.soff * D;
    s.I2 = J.big_idx + B.soff;
    s.SV = static_cast<T *>(J.big_surv) + B.soff * D;
    s.SVI = J.big_surv_idx + B.soff;
    const int32_t kept = sfs_block<D, T, SfsSmallCfg<D, T>>(smem_raw, static_cast<const T *>(J.big_pts) + B.soff * D,
                                                            B.n, s, static_cast<T *>(J.out_pts) + B.c0 * D);
    if (threadIdx.x == 0) J.out_size[B.item] = kept;
}

// SFS blocks largest destination first: one block sorts the pass's work list by
// candidate count, descending (ties in list order; destinations outside the pass or for
// the mark path count as empty), so that the longest blocks start first and the tail of
// the launch is short.  num_work <= kBigOrderMax.
__global__ void __launch_bounds__(1024) big_order_kernel(const ExpandJob *__restrict__ jobs,
                                                         const BigWork *__restrict__ work, int num_work, int64_t pass,
                                                         int32_t *__restrict__ order) {
    __shared__ unsigned long long key[kBigOrderMax];
    int m = 1;
    while (m < num_work) m <<= 1;
    constexpr unsigned long long kMaxN = (1ULL << 40) - 1;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        unsigned long long k = ~0ULL;
        if (i < num_work) {
            const BigWork W = work[i];
            const ExpandJob &J = jobs[W.job];
            BigItem B;
            unsigned long long n = 0;
            if (big_item(J, W, pass, &B) && B.n < J.big_mark_min)
                n = B.n > static_cast<int64_t>(kMaxN) ? kMaxN : static_cast<unsigned long long>(B.n);
            k = ((kMaxN - n) << 12) | static_cast<unsigned long long>(i);
        }
        key[i] = k;
    }
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                const int p = i ^ j;
                if (p > i) {
                    const unsigned long long a = key[i], b = key[p];
                    if (((i & k) == 0) == (a > b)) {
                        key[i] = b;
                        key[p] = a;
                    }
                }
            }
            __syncthreads();
        }
    for (int i = threadIdx.x; i < num_work; i += blockDim.x) order[i] = static_cast<int32_t>(key[i] & 4095ULL);
}

template <int D, typename T>
static cudaError_t launch_big_t(const BigLaunch &L, cudaStream_t stream) {
    if (L.num_work <= 0 || L.total <= 0) return cudaSuccess;
    using Cfg = SfsSmallCfg<D, T>;
    {
        const cudaError_t e = ensure_smem_limit(reinterpret_cast<const void *>(big_sfs_kernel<D, T>), Cfg::kSmem);
        if (e != cudaSuccess) return e;
    }
    const bool lex = D == 3 && L.lex_big;
    if (lex) {
        cudaError_t e = launch_big_lex_rank(sizeof(T) == 8, L, stream);
        for (int r = 0; e == cudaSuccess && r < L.lex_rounds; ++r) e = launch_big_lex_merge(sizeof(T) == 8, L, r, stream);
        if (e != cudaSuccess) return e;
    } else {
        const int64_t want = (L.total + kFlatThreads - 1) / kFlatThreads;
        const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(L.sms) * 32)));
        big_expand_kernel<D, T><<<grid, kFlatThreads, 0, stream>>>(L.jobs, L.job_bases, L.num_jobs, L.total, L.pass);
    }
    if (L.with_sfs) {
        const int32_t *order = nullptr;
        if (L.order && L.num_work <= kBigOrderMax) {
            big_order_kernel<<<1, 1024, 0, stream>>>(L.jobs, L.work, L.num_work, L.pass, L.order);
            order = L.order;
        }
        big_sfs_kernel<D, T><<<L.num_work, Cfg::kThreads, Cfg::kSmem, stream>>>(L.jobs, L.work, order, L.pass);
    }
    if (L.mark_cap > 0) {
        MarkPlan *plan = static_cast<MarkPlan *>(L.plan);
        big_plan_kernel<<<1, kPlanThreads, 0, stream>>>(L.jobs, L.work, L.num_work, L.pass, plan, L.mark_cap);
        // chunks: at most one per 256 candidates of the pass plus one per listed destination
        const unsigned chunks = static_cast<unsigned>((L.total + kMarkThreads - 1) / kMarkThreads + L.mark_cap);
        big_pivot_kernel<D, T><<<L.mark_cap, kPivotThreads, 0, stream>>>(L.jobs, L.work, L.pass, plan, L.mark_cap);
        big_prefilter_kernel<D, T><<<chunks, kMarkThreads, 0, stream>>>(L.jobs, L.work, L.pass, plan, L.mark_cap);
        big_compact_kernel<D, T><<<L.mark_cap, kCompactThreads, 0, stream>>>(L.jobs, L.work, L.pass, plan, L.mark_cap);
        big_rplan_kernel<<<1, kPlanThreads, 0, stream>>>(plan, L.mark_cap);
        big_mark_kernel<D, T><<<chunks, kMarkThreads, 0, stream>>>(L.jobs, L.work, L.pass, plan, L.mark_cap);
        big_write_kernel<D, T><<<L.mark_cap, kWriteThreads, 0, stream>>>(L.jobs, L.work, L.pass, plan, L.mark_cap);
    }
    if (lex) return launch_big_lex_filter(sizeof(T) == 8, L, stream);
    return cudaGetLastError();
}

cudaError_t launch_big(int d, bool wide, const BigLaunch &L, cudaStream_t stream) {
    if (wide) { PMDD_DISPATCH_D(d, (launch_big_t<DD, int64_t>(L, stream))); }
    PMDD_DISPATCH_D(d, (launch_big_t<DD, int32_t>(L, stream)));
}

}  // namespace dev
}  // namespace pmdd
