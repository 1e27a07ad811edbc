// sm_100a kernels of the enumeration hot path: next-layer counting, the fused
// expand+dominance-filter tile kernel, and the global-memory path for destinations
// too large for one tile.
//
// Dominance rule (same as the reference GPU filter, src/pmdd/enum/gpu/dominance_utils.cuh:10-23,
// and the weak-dominance insert of src/pmdd/enum/pareto_frontier.hpp:237-303): a candidate
// q of a destination is dropped iff another candidate p of the same destination has
// p >= q on every objective and (p != q or p comes first).  Candidates from the same arc
// are shifts of one non-dominated, duplicate-free parent frontier, so they never drop each
// other and are not compared.
#include "kernels.cuh"

#include <algorithm>
#include <climits>

namespace pmdd {
namespace dev {

// ------------------------------------------------------------------ block scans
template <typename V, int THREADS>
__device__ __forceinline__ V block_exclusive_scan(V x, V *warp_buf, V *total) {
    static_assert(THREADS % 32 == 0 && THREADS <= 1024, "block size");
    constexpr int NW = THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    V inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        V y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_buf[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        V w = lane < NW ? warp_buf[lane] : V(0);
        V winc = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            V y = __shfl_up_sync(0xffffffffu, winc, o);
            if (lane >= o) winc += y;
        }
        if (lane < NW) warp_buf[lane] = winc - w;
        if (lane == NW - 1) *total = winc;
    }
    __syncthreads();
    const V r = inc - x + warp_buf[warp];
    __syncthreads();  // warp_buf / total may be reused right after
    return r;
}

// Candidate start of destination `i` (local) of a job whose arc offsets are known.
__device__ __forceinline__ int64_t item_start(const int32_t *item_arc_off, const int64_t *arc_cand_off,
                                              int32_t item_base, int32_t arc_base, int32_t i) {
    return arc_cand_off[item_arc_off[item_base + i] - arc_base];
}

// -------------------------------------------------------------- counting pass
// One block per job: exclusive scan of per-arc candidate counts (the neighbour's
// frontier size), destination sizes, and the list of oversized destinations with
// their scratch offsets.
__global__ void __launch_bounds__(kCountThreads) count_scan_kernel(const CountJob *jobs) {
    const CountJob J = jobs[blockIdx.x];
    __shared__ int64_t warp_buf[32];
    __shared__ int64_t s_total;
    __shared__ int64_t s_carry;
    __shared__ unsigned long long s_max;
    __shared__ int s_nbig;
    const int tid = threadIdx.x;
    if (tid == 0) {
        s_carry = 0;
        s_max = 0;
        s_nbig = 0;
    }
    __syncthreads();
    for (int base = 0; base < J.num_arcs; base += kCountThreads) {
        const int a = base + tid;
        int64_t c = 0;
        if (a < J.num_arcs) c = J.cur_size[J.arc_nbr[J.arc_base + a] - J.cur_base];
        const int64_t ex = block_exclusive_scan<int64_t, kCountThreads>(c, warp_buf, &s_total);
        if (a < J.num_arcs) J.arc_cand_off[a] = s_carry + ex;
        __syncthreads();
        if (tid == 0) s_carry += s_total;
        __syncthreads();
    }
    if (tid == 0) J.arc_cand_off[J.num_arcs] = s_carry;
    __syncthreads();
    for (int i = tid; i < J.num_items; i += kCountThreads) {
        const int32_t v = J.item_base + i;
        const int64_t b = J.arc_cand_off[J.item_arc_off[v] - J.arc_base];
        const int64_t e = J.arc_cand_off[J.item_arc_off[v + 1] - J.arc_base];
        const int64_t c = e - b;
        atomicMax(&s_max, static_cast<unsigned long long>(c));
        if (c > kSmallMax) {
            const int k = atomicAdd(&s_nbig, 1);
            J.big_list[2 * k] = i;
            J.big_list[2 * k + 1] = c;
        }
    }
    __syncthreads();
    // scratch offsets of the oversized destinations (exclusive scan of their sizes)
    const int nbig = s_nbig;
    if (tid == 0) s_carry = 0;
    __syncthreads();
    for (int base = 0; base < nbig; base += kCountThreads) {
        const int k = base + tid;
        const int64_t c = k < nbig ? J.big_list[2 * k + 1] : 0;
        const int64_t ex = block_exclusive_scan<int64_t, kCountThreads>(c, warp_buf, &s_total);
        if (k < nbig) J.big_list[2 * k + 1] = s_carry + ex;
        __syncthreads();
        if (tid == 0) s_carry += s_total;
        __syncthreads();
    }
    // survivors of the current layer
    int64_t cur = 0;
    for (int i = tid; i < J.cur_nodes; i += kCountThreads) cur += J.cur_size[i];
    for (int s = 16; s > 0; s >>= 1) cur += __shfl_xor_sync(0xffffffffu, cur, s);
    if ((tid & 31) == 0) warp_buf[tid >> 5] = cur;
    __syncthreads();
    if (tid == 0) {
        int64_t cur_total = 0;
        for (int w = 0; w < kCountThreads / 32; ++w) cur_total += warp_buf[w];
        J.result->total = J.arc_cand_off[J.num_arcs];
        J.result->max_item = static_cast<int64_t>(s_max);
        J.result->big_total = s_carry;
        J.result->cur_total = cur_total;
        J.result->num_big = nbig;
    }
}

// ----------------------------------------------------------- fused tile kernel
template <int D, typename T>
struct TileSmem {
    T comp[D][kTileCap];            // candidates, one plane per objective
    int32_t tag[kTileCap];          // arc of each candidate
    int16_t item_of[kTileCap];      // staged destination of each candidate
    int32_t keep_ex[kTileCap + 1];  // exclusive scan of keep flags
    int32_t item_s[kTileItemCap + 1];   // staged destination -> first candidate slot
    int64_t item_c0[kTileItemCap];      // staged destination -> job-local candidate start
    int32_t warp_i[32];
    int32_t tot_i;
    int32_t i0, i1;
    int32_t job;
};

// Job owning global tile `tile` (jobs sorted by tile_base).
__device__ __forceinline__ int find_job(const ExpandJob *jobs, int num_jobs, int64_t tile) {
    int lo = 0, hi = num_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].tile_base <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// First destination whose candidate start is >= x.
__device__ __forceinline__ int32_t lower_bound_item(const ExpandJob &J, int64_t x) {
    int32_t lo = 0, hi = J.num_items;
    while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (item_start(J.item_arc_off, J.arc_cand_off, J.item_base, J.arc_base, mid) < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

template <int D, typename T>
__global__ void __launch_bounds__(kTileThreads) expand_tile_kernel(const ExpandJob *__restrict__ jobs, int num_jobs,
                                                                   int64_t total_tiles) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TileSmem<D, T> &S = *reinterpret_cast<TileSmem<D, T> *>(smem_raw);
    const int tid = threadIdx.x;
    for (int64_t tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
        if (tid == 0) {
            const int j = find_job(jobs, num_jobs, tile);
            const ExpandJob &J = jobs[j];
            const int64_t t = tile - J.tile_base;
            const int64_t w0 = t * kTileWindow;
            S.job = j;
            S.i0 = lower_bound_item(J, w0);
            S.i1 = (t == J.num_tiles - 1) ? J.num_items : lower_bound_item(J, w0 + kTileWindow);
        }
        __syncthreads();
        const ExpandJob &J = jobs[S.job];
        const int32_t i0 = S.i0, i1 = S.i1;
        const T *__restrict__ prev = static_cast<const T *>(J.prev_pts);
        T *__restrict__ outp = static_cast<T *>(J.out_pts);
        for (int32_t ic = i0; ic < i1; ic += kTileItemCap) {
            const int n_it = min(kTileItemCap, i1 - ic);
            // --- stage destinations: start, size, slot offsets (4 per thread)
            constexpr int PER = kTileItemCap / kTileThreads;
            int32_t cnt[PER];
            int32_t local = 0;
#pragma unroll
            for (int r = 0; r < PER; ++r) {
                const int k = tid * PER + r;
                cnt[r] = 0;
                if (k < n_it) {
                    const int32_t i = ic + k;
                    const int32_t v = J.item_base + i;
                    const int64_t s = J.arc_cand_off[J.item_arc_off[v] - J.arc_base];
                    const int64_t e = J.arc_cand_off[J.item_arc_off[v + 1] - J.arc_base];
                    const int64_t c = e - s;
                    J.out_off[i] = s;
                    if (c == 0) J.out_size[i] = 0;
                    S.item_c0[k] = s;
                    cnt[r] = c <= kSmallMax ? static_cast<int32_t>(c) : 0;
                }
                local += cnt[r];
            }
            const int32_t ex = block_exclusive_scan<int32_t, kTileThreads>(local, S.warp_i, &S.tot_i);
            {
                int32_t run = ex;
#pragma unroll
                for (int r = 0; r < PER; ++r) {
                    const int k = tid * PER + r;
                    if (k < n_it) S.item_s[k] = run;
                    run += cnt[r];
                }
            }
            const int32_t total = S.tot_i;
            if (tid == 0) S.item_s[n_it] = total;
            __syncthreads();
            if (total > kTileCap) {  // cannot happen for well-formed offsets; skip defensively
                if (tid == 0) atomicOr(J.err, kErrBounds);
                __syncthreads();
                continue;
            }
            // --- expand: candidate q = parent point + arc weight
            for (int q = tid; q < total; q += kTileThreads) {
                int lo = 0, hi = n_it - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (S.item_s[mid] <= q) lo = mid;
                    else hi = mid - 1;
                }
                const int k = lo;
                const int64_t cidx = S.item_c0[k] + (q - S.item_s[k]);
                const int32_t v = J.item_base + ic + k;
                int32_t alo = J.item_arc_off[v], ahi = J.item_arc_off[v + 1] - 1;
                while (alo < ahi) {
                    const int32_t mid = (alo + ahi + 1) >> 1;
                    if (J.arc_cand_off[mid - J.arc_base] <= cidx) alo = mid;
                    else ahi = mid - 1;
                }
                const int32_t a = alo;
                const int64_t idx = cidx - J.arc_cand_off[a - J.arc_base];
                const int32_t u = J.arc_nbr[a] - J.prev_base;
                const T *src = prev + (J.prev_off[u] + idx) * D;
                const int32_t *w = J.weights + static_cast<int64_t>(J.arc_wrow[a]) * D;
#pragma unroll
                for (int o = 0; o < D; ++o) S.comp[o][q] = src[o] + static_cast<T>(w[o]);
                S.tag[q] = a;
                S.item_of[q] = static_cast<int16_t>(k);
            }
            __syncthreads();
            // --- filter within each destination, other arcs only
            constexpr int QPER = kTileCap / kTileThreads;
            int32_t kept[QPER];
            int32_t kept_local = 0;
#pragma unroll
            for (int r = 0; r < QPER; ++r) {
                const int q = tid * QPER + r;
                kept[r] = 0;
                if (q < total) {
                    const int k = S.item_of[q];
                    const int js = S.item_s[k], je = S.item_s[k + 1];
                    T p[D];
#pragma unroll
                    for (int o = 0; o < D; ++o) p[o] = S.comp[o][q];
                    const int32_t my_tag = S.tag[q];
                    bool dom = false;
                    for (int j = js; j < je; ++j) {
                        if (S.tag[j] == my_tag) continue;
                        bool ge = true, eq = true;
#pragma unroll
                        for (int o = 0; o < D; ++o) {
                            const T x = S.comp[o][j];
                            ge &= (x >= p[o]);
                            eq &= (x == p[o]);
                        }
                        if (ge && (!eq || j < q)) {
                            dom = true;
                            break;
                        }
                    }
                    kept[r] = dom ? 0 : 1;
                }
                kept_local += kept[r];
            }
            const int32_t kex = block_exclusive_scan<int32_t, kTileThreads>(kept_local, S.warp_i, &S.tot_i);
            {
                int32_t run = kex;
#pragma unroll
                for (int r = 0; r < QPER; ++r) {
                    const int q = tid * QPER + r;
                    if (q < total) S.keep_ex[q] = run;
                    run += kept[r];
                }
                if (tid == kTileThreads - 1) S.keep_ex[total] = run;
            }
            __syncthreads();
            // --- write survivors into each destination's slot
#pragma unroll
            for (int r = 0; r < QPER; ++r) {
                const int q = tid * QPER + r;
                if (q < total && kept[r]) {
                    const int k = S.item_of[q];
                    const int64_t dst = S.item_c0[k] + (S.keep_ex[q] - S.keep_ex[S.item_s[k]]);
                    T *o_ = outp + dst * D;
#pragma unroll
                    for (int o = 0; o < D; ++o) o_[o] = S.comp[o][q];
                }
            }
            for (int k = tid; k < n_it; k += kTileThreads) {
                const int js = S.item_s[k], je = S.item_s[k + 1];
                if (je > js) J.out_size[ic + k] = S.keep_ex[je] - S.keep_ex[js];
            }
            __syncthreads();
        }
        __syncthreads();  // tile bookkeeping in shared memory is rewritten next iteration
    }
}

// ------------------------------------------------------- oversized destinations
// Destinations with more than kSmallMax candidates.  Their candidates are materialised
// in scratch, then filtered by a bucketed sort-filter-skyline sweep (the presorting
// idea of Chomicki, Godfrey, Gryz and Liang, "Skyline with presorting", ICDE 2003):
// points are grouped into buckets of decreasing objective sum; a dominator of p has a
// sum >= p's, so it lies in p's bucket or an earlier one.  Each bucket's points are
// checked against the kept set K of earlier buckets (all of which are maximal), the
// bucket's survivors against each other, and the bucket's maxima are appended to K --
// which is the destination's slot in the output.

template <int D, typename T>
__device__ __forceinline__ int64_t point_sum(const T *p) {
    int64_t s = 0;
#pragma unroll
    for (int o = 0; o < D; ++o) s += static_cast<int64_t>(p[o]);
    return s;
}

// Materialise the candidates of one oversized destination (AoS).
template <int D, typename T>
__global__ void __launch_bounds__(kBigThreads) big_expand_kernel(const ExpandJob *__restrict__ jobs,
                                                                 const BigWork *__restrict__ work) {
    const BigWork W = work[blockIdx.y];
    const ExpandJob &J = jobs[W.job];
    const int32_t item = static_cast<int32_t>(J.big_list[2 * W.big]);
    const int64_t soff = J.big_list[2 * W.big + 1];
    T *spts = static_cast<T *>(J.big_pts);
    const int32_t v = J.item_base + item;
    const int32_t a0 = J.item_arc_off[v], a1 = J.item_arc_off[v + 1];
    const int64_t c0 = J.arc_cand_off[a0 - J.arc_base];
    const T *prev = static_cast<const T *>(J.prev_pts);
    for (int32_t a = a0; a < a1; ++a) {
        const int64_t b = J.arc_cand_off[a - J.arc_base];
        const int64_t n = J.arc_cand_off[a + 1 - J.arc_base] - b;
        if (n == 0) continue;
        const int32_t u = J.arc_nbr[a] - J.prev_base;
        const T *src = prev + J.prev_off[u] * D;
        const int32_t *w = J.weights + static_cast<int64_t>(J.arc_wrow[a]) * D;
        T wv[D];
#pragma unroll
        for (int o = 0; o < D; ++o) wv[o] = static_cast<T>(w[o]);
        for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n;
             idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
            const int64_t dst = soff + (b - c0) + idx;
#pragma unroll
            for (int o = 0; o < D; ++o) spts[dst * D + o] = src[idx * D + o] + wv[o];
        }
    }
}

template <int D, typename T>
struct SfsCfg {
    static constexpr int kThreads = 512;
    static constexpr int kMaxBuckets = 8192;
    static constexpr int kKeepCache = 65536 / (D * static_cast<int>(sizeof(T)));             // K points in smem
    static constexpr int kSurvCache = 49152 / (D * static_cast<int>(sizeof(T)) + 8);         // survivors in smem
    static constexpr size_t kSmem = sizeof(int32_t) * kMaxBuckets + sizeof(T) * D * kKeepCache +
                                    (sizeof(T) * D + 2 * sizeof(int32_t)) * kSurvCache + 512;
};

template <int D, typename T>
__global__ void __launch_bounds__(SfsCfg<D, T>::kThreads) big_sfs_kernel(const ExpandJob *__restrict__ jobs,
                                                                         const BigWork *__restrict__ work) {
    using Cfg = SfsCfg<D, T>;
    constexpr int NT = Cfg::kThreads, KS = Cfg::kKeepCache, SC = Cfg::kSurvCache;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int32_t *hist = reinterpret_cast<int32_t *>(smem_raw);
    T *kc = reinterpret_cast<T *>(hist + Cfg::kMaxBuckets);             // [D][KS]
    T *sc = kc + static_cast<size_t>(D) * KS;                            // [D][SC]
    int32_t *sidx = reinterpret_cast<int32_t *>(sc + static_cast<size_t>(D) * SC);  // [SC]
    int32_t *sflag = sidx + SC;                                          // [SC]
    __shared__ int64_t red_min[NT / 32], red_max[NT / 32];
    __shared__ int32_t warp_i[32];
    __shared__ int32_t tot_i;
    __shared__ int64_t s_min, s_max;
    __shared__ int32_t s_kn, s_m;

    const BigWork W = work[blockIdx.x];
    const ExpandJob &J = jobs[W.job];
    const int32_t item = static_cast<int32_t>(J.big_list[2 * W.big]);
    const int64_t soff = J.big_list[2 * W.big + 1];
    const int32_t v = J.item_base + item;
    const int64_t s0 = J.arc_cand_off[J.item_arc_off[v] - J.arc_base];
    const int64_t n = J.arc_cand_off[J.item_arc_off[v + 1] - J.arc_base] - s0;
    const T *P = static_cast<const T *>(J.big_pts) + soff * D;
    T *P2 = static_cast<T *>(J.big_pts2) + soff * D;
    int32_t *I2 = J.big_idx + soff;
    T *SV = static_cast<T *>(J.big_surv) + soff * D;
    int32_t *SVI = J.big_surv_idx + soff;
    T *out = static_cast<T *>(J.out_pts) + s0 * D;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // 1. range of point sums
    int64_t mn = INT64_MAX, mx = INT64_MIN;
    for (int64_t i = tid; i < n; i += NT) {
        const int64_t sm = point_sum<D, T>(P + i * D);
        mn = min(mn, sm);
        mx = max(mx, sm);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (lane == 0) {
        red_min[warp] = mn;
        red_max[warp] = mx;
    }
    __syncthreads();
    if (tid == 0) {
        int64_t a = red_min[0], b = red_max[0];
        for (int w = 1; w < NT / 32; ++w) {
            a = min(a, red_min[w]);
            b = max(b, red_max[w]);
        }
        s_min = a;
        s_max = b;
        s_kn = 0;
    }
    __syncthreads();
    // 2. counting sort into buckets of decreasing sum (bucket 0 = largest sums)
    const int64_t nb64 = n / 32 < 1 ? 1 : n / 32;
    const int nb = static_cast<int>(nb64 < Cfg::kMaxBuckets ? nb64 : static_cast<int64_t>(Cfg::kMaxBuckets));
    const int64_t width = (s_max - s_min) / nb + 1;
    for (int b = tid; b < nb; b += NT) hist[b] = 0;
    __syncthreads();
    for (int64_t i = tid; i < n; i += NT) {
        const int b = static_cast<int>((s_max - point_sum<D, T>(P + i * D)) / width);
        atomicAdd(&hist[b], 1);
    }
    __syncthreads();
    {
        constexpr int PER = Cfg::kMaxBuckets / NT;
        int32_t loc[PER];
        int32_t run = 0;
#pragma unroll
        for (int r = 0; r < PER; ++r) {
            const int b = tid * PER + r;
            loc[r] = b < nb ? hist[b] : 0;
            run += loc[r];
        }
        int32_t ex = block_exclusive_scan<int32_t, NT>(run, warp_i, &tot_i);
#pragma unroll
        for (int r = 0; r < PER; ++r) {
            const int b = tid * PER + r;
            if (b < nb) hist[b] = ex;
            ex += loc[r];
        }
    }
    __syncthreads();
    for (int64_t i = tid; i < n; i += NT) {
        const T *p = P + i * D;
        const int b = static_cast<int>((s_max - point_sum<D, T>(p)) / width);
        const int pos = atomicAdd(&hist[b], 1);
#pragma unroll
        for (int o = 0; o < D; ++o) P2[static_cast<int64_t>(pos) * D + o] = p[o];
        I2[pos] = static_cast<int32_t>(i);
    }
    __syncthreads();  // hist[b] is now the end of bucket b

    // 3. sweep the buckets
    for (int b = 0; b < nb; ++b) {
        const int32_t lo = b == 0 ? 0 : hist[b - 1], hi = hist[b];
        if (lo == hi) continue;
        if (tid == 0) s_m = 0;
        __syncthreads();
        const int32_t kn = s_kn;
        // 3a. against the maxima of earlier buckets
        for (int32_t c0 = lo; c0 < hi; c0 += NT) {
            const int32_t i = c0 + tid;
            const bool valid = i < hi;
            T p[D];
            int32_t pidx = 0;
            bool dom = !valid;
            if (valid) {
#pragma unroll
                for (int o = 0; o < D; ++o) p[o] = P2[static_cast<int64_t>(i) * D + o];
                pidx = I2[i];
                for (int32_t j = 0; j < kn; ++j) {
                    bool ge = true;
                    if (j < KS) {
#pragma unroll
                        for (int o = 0; o < D; ++o) ge &= (kc[o * KS + j] >= p[o]);
                    } else {
#pragma unroll
                        for (int o = 0; o < D; ++o) ge &= (out[static_cast<int64_t>(j) * D + o] >= p[o]);
                    }
                    if (ge) {
                        dom = true;
                        break;
                    }
                }
            }
            const int32_t ex = block_exclusive_scan<int32_t, NT>(dom ? 0 : 1, warp_i, &tot_i);
            const int32_t m0 = s_m;
            if (!dom) {
                const int32_t k = m0 + ex;
                if (k < SC) {
#pragma unroll
                    for (int o = 0; o < D; ++o) sc[o * SC + k] = p[o];
                    sidx[k] = pidx;
                } else {
#pragma unroll
                    for (int o = 0; o < D; ++o) SV[static_cast<int64_t>(k) * D + o] = p[o];
                    SVI[k] = pidx;
                }
            }
            __syncthreads();
            if (tid == 0) s_m = m0 + tot_i;
            __syncthreads();
        }
        const int32_t m = s_m;
        // 3b. survivors of this bucket against each other (first duplicate kept)
        for (int32_t k = tid; k < m; k += NT) {
            T p[D];
            int32_t pidx;
            if (k < SC) {
#pragma unroll
                for (int o = 0; o < D; ++o) p[o] = sc[o * SC + k];
                pidx = sidx[k];
            } else {
#pragma unroll
                for (int o = 0; o < D; ++o) p[o] = SV[static_cast<int64_t>(k) * D + o];
                pidx = SVI[k];
            }
            bool dom = false;
            for (int32_t j = 0; j < m && !dom; ++j) {
                if (j == k) continue;
                bool ge = true, eq = true;
                int32_t qidx;
                if (j < SC) {
#pragma unroll
                    for (int o = 0; o < D; ++o) {
                        const T x = sc[o * SC + j];
                        ge &= (x >= p[o]);
                        eq &= (x == p[o]);
                    }
                    qidx = sidx[j];
                } else {
#pragma unroll
                    for (int o = 0; o < D; ++o) {
                        const T x = SV[static_cast<int64_t>(j) * D + o];
                        ge &= (x >= p[o]);
                        eq &= (x == p[o]);
                    }
                    qidx = SVI[j];
                }
                dom = ge && (!eq || qidx < pidx);
            }
            if (k < SC) sflag[k] = dom ? 0 : 1;
            else I2[lo + k] = dom ? 0 : 1;  // bucket entries [lo, hi) were consumed above
        }
        __syncthreads();
        // 3c. append the bucket's maxima to K (the output slot) and the K cache
        for (int32_t c0 = 0; c0 < m; c0 += NT) {
            const int32_t k = c0 + tid;
            int32_t keep = 0;
            if (k < m) keep = k < SC ? sflag[k] : I2[lo + k];
            const int32_t ex = block_exclusive_scan<int32_t, NT>(keep, warp_i, &tot_i);
            const int32_t base = s_kn;
            if (keep) {
                const int32_t dst = base + ex;
#pragma unroll
                for (int o = 0; o < D; ++o) {
                    const T x = k < SC ? sc[o * SC + k] : SV[static_cast<int64_t>(k) * D + o];
                    out[static_cast<int64_t>(dst) * D + o] = x;
                    if (dst < KS) kc[o * KS + dst] = x;
                }
            }
            __syncthreads();
            if (tid == 0) s_kn = base + tot_i;
            __syncthreads();
        }
    }
    if (tid == 0) J.out_size[item] = s_kn;
}

// ----------------------------------------------------------------- launchers
template <int D, typename T>
static cudaError_t launch_expand_tiles_t(const ExpandJob *jobs, int num_jobs, int64_t total_tiles, int grid,
                                         cudaStream_t stream) {
    const size_t smem = sizeof(TileSmem<D, T>);
    static bool attr_set = false;  // per instantiation; setting it twice is harmless
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(expand_tile_kernel<D, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    if (total_tiles <= 0) return cudaSuccess;
    const int64_t g = std::min<int64_t>(total_tiles, grid);
    expand_tile_kernel<D, T><<<static_cast<unsigned>(g), kTileThreads, smem, stream>>>(jobs, num_jobs, total_tiles);
    return cudaGetLastError();
}

template <int D, typename T>
static cudaError_t launch_big_t(const ExpandJob *jobs, const BigWork *work, int num_work, int64_t max_item, int sms,
                                cudaStream_t stream) {
    if (num_work <= 0) return cudaSuccess;
    using Cfg = SfsCfg<D, T>;
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(big_sfs_kernel<D, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(Cfg::kSmem));
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    const int64_t chunks = (max_item + kBigThreads - 1) / kBigThreads;
    const unsigned gx_expand = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(chunks, 64)));
    constexpr int kMaxY = 65535;  // grid.y limit
    for (int w0 = 0; w0 < num_work; w0 += kMaxY) {
        const int nw = std::min(kMaxY, num_work - w0);
        big_expand_kernel<D, T><<<dim3(gx_expand, nw), kBigThreads, 0, stream>>>(jobs, work + w0);
    }
    big_sfs_kernel<D, T><<<num_work, Cfg::kThreads, Cfg::kSmem, stream>>>(jobs, work);
    (void)sms;
    return cudaGetLastError();
}

#define PMDD_DISPATCH_D(D_, CALL)                                   \
    switch (D_) {                                                   \
    case 1: { constexpr int DD = 1; return CALL; }                  \
    case 2: { constexpr int DD = 2; return CALL; }                  \
    case 3: { constexpr int DD = 3; return CALL; }                  \
    case 4: { constexpr int DD = 4; return CALL; }                  \
    case 5: { constexpr int DD = 5; return CALL; }                  \
    case 6: { constexpr int DD = 6; return CALL; }                  \
    case 7: { constexpr int DD = 7; return CALL; }                  \
    case 8: { constexpr int DD = 8; return CALL; }                  \
    default: return cudaErrorInvalidValue;                          \
    }

cudaError_t launch_count_scan(const CountJob *jobs, int num_jobs, cudaStream_t stream) {
    if (num_jobs <= 0) return cudaSuccess;
    count_scan_kernel<<<num_jobs, kCountThreads, 0, stream>>>(jobs);
    return cudaGetLastError();
}

cudaError_t launch_expand_tiles(int d, bool wide, const ExpandJob *jobs, int num_jobs, int64_t total_tiles, int grid,
                                cudaStream_t stream) {
    if (wide) { PMDD_DISPATCH_D(d, (launch_expand_tiles_t<DD, int64_t>(jobs, num_jobs, total_tiles, grid, stream))); }
    PMDD_DISPATCH_D(d, (launch_expand_tiles_t<DD, int32_t>(jobs, num_jobs, total_tiles, grid, stream)));
}

cudaError_t launch_big(int d, bool wide, const ExpandJob *jobs, const BigWork *work, int num_work, int64_t max_item,
                       int sms, cudaStream_t stream) {
    if (wide) { PMDD_DISPATCH_D(d, (launch_big_t<DD, int64_t>(jobs, work, num_work, max_item, sms, stream))); }
    PMDD_DISPATCH_D(d, (launch_big_t<DD, int32_t>(jobs, work, num_work, max_item, sms, stream)));
}

}  // namespace dev
}  // namespace pmdd
