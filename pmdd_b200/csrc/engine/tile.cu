// Fused expand + dominance filter over candidate tiles (the per-layer hot kernel).
//
// A tile owns every destination whose candidate range starts inside its window of
// kTileWindow candidates; destinations with at most kSmallMax candidates are handled
// here entirely in shared memory, larger ones only get their slot offset (the
// oversized path in big.cu filters them).  A tile therefore holds < kTileCap points.
//
//   expand:  candidate = parent frontier point + arc weight vector, read straight from
//            the parent's slot (consecutive candidates of an arc are consecutive parent
//            points, so the loads coalesce);
//   filter:  each warp takes 32 candidates and sweeps the candidates of their
//            destinations with warp-uniform shared-memory broadcast reads, skipping the
//            candidates' own arc (shifts of one non-dominated, duplicate-free parent
//            frontier never dominate each other) and leaving as soon as all 32 are
//            decided;
//   write:   survivors go to the destination's slot in the next layer's frontier.
//
// Dominance rule (the reference GPU filter's dominates_or_tie_before,
// src/pmdd/enum/gpu/dominance_utils.cuh:10-23, and the weak-dominance insert of
// src/pmdd/enum/pareto_frontier.hpp:237-303): candidate q is dropped iff another
// candidate p of the same destination has p >= q on every objective and (p != q or p
// comes first).
#include "kernels.cuh"
#include "scan.cuh"

#include <algorithm>

namespace pmdd {
namespace dev {

template <int D, typename T>
struct TileSmem {
    PackedPt<D, T> pts[kTileCap];
    int32_t tag[kTileCap];              // arc of each candidate
    uint16_t seg_lo[kTileCap];          // tile positions of the candidate's own arc run
    uint16_t seg_hi[kTileCap];
    uint16_t item_of[kTileCap];         // staged destination of each candidate
    uint8_t keep[kTileCap];
    int32_t keep_ex[kTileCap + 1];      // exclusive scan of keep flags
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

// Warp sweep over [a, b) for 32 candidates: lane's candidate (p, position q, arc tag)
// is dominated by some j in [max(a, js), min(b, je)) with a different arc.
template <int D, typename T>
__device__ __forceinline__ bool sweep_range(const TileSmem<D, T> &S, int a, int b, const T (&p)[D], int q, int32_t tag,
                                            int js, int je, bool dom) {
    for (int j = a; j < b; ++j) {
        const PackedPt<D, T> c = S.pts[j];
        const int32_t tj = S.tag[j];
        if (!dom && ge_all<D, T>(c, p) && j >= js && j < je && tj != tag) {
            if (!eq_all<D, T>(c, p) || j < q) dom = true;
        }
        if ((j & 31) == 31 && __all_sync(0xffffffffu, dom)) return true;
    }
    return dom;
}

template <int D, typename T>
__global__ void __launch_bounds__(kTileThreads) expand_tile_kernel(const ExpandJob *__restrict__ jobs, int num_jobs,
                                                                   int64_t total_tiles) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TileSmem<D, T> &S = *reinterpret_cast<TileSmem<D, T> *>(smem_raw);
    constexpr int NW = kTileThreads / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
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
            // --- stage destinations: start, size, slot offsets
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
            if (total > kTileCap) {  // impossible for well-formed offsets; skip defensively
                if (tid == 0) atomicOr(J.err, kErrBounds);
                __syncthreads();
                continue;
            }
            // --- expand: candidate = parent point + arc weight
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
                const int64_t a0 = J.arc_cand_off[a - J.arc_base];
                const int64_t na = J.arc_cand_off[a + 1 - J.arc_base] - a0;
                const int64_t idx = cidx - a0;
                const int32_t u = J.arc_nbr[a] - J.prev_base;
                const T *src = prev + (J.prev_off[u] + idx) * D;
                const int32_t *w = J.weights + static_cast<int64_t>(J.arc_wrow[a]) * D;
                PackedPt<D, T> pt;
#pragma unroll
                for (int o = 0; o < PackedPt<D, T>::kPad; ++o) pt.v[o] = o < D ? src[o] + static_cast<T>(w[o]) : T(0);
                S.pts[q] = pt;
                S.tag[q] = a;
                S.seg_lo[q] = static_cast<uint16_t>(q - idx);
                S.seg_hi[q] = static_cast<uint16_t>(q - idx + na);
                S.item_of[q] = static_cast<uint16_t>(k);
            }
            __syncthreads();
            // --- filter: warp per 32 candidates, uniform sweep over their destinations
            for (int c0 = warp * 32; c0 < total; c0 += NW * 32) {
                const int q = c0 + lane;
                const bool valid = q < total;
                T p[D];
                int32_t my_tag = -1;
                int js = INT_MAX, je = INT_MIN, slo = 0, shi = 0;
                if (valid) {
                    const PackedPt<D, T> me = S.pts[q];
#pragma unroll
                    for (int o = 0; o < D; ++o) p[o] = me.v[o];
                    my_tag = S.tag[q];
                    const int k = S.item_of[q];
                    js = S.item_s[k];
                    je = S.item_s[k + 1];
                    slo = S.seg_lo[q];
                    shi = S.seg_hi[q];
                } else {
#pragma unroll
                    for (int o = 0; o < D; ++o) p[o] = T(0);
                }
                const int J0 = warp_min_i(js), J1 = warp_max_i(je);
                // all lanes in one arc run: skip that run entirely
                const bool one_run = __all_sync(0xffffffffu, valid) && warp_min_i(slo) == warp_max_i(slo) &&
                                     warp_min_i(shi) == warp_max_i(shi);
                bool dom = !valid;
                if (one_run) {
                    dom = sweep_range<D, T>(S, J0, slo, p, q, my_tag, js, je, dom);
                    if (!__all_sync(0xffffffffu, dom)) dom = sweep_range<D, T>(S, shi, J1, p, q, my_tag, js, je, dom);
                } else {
                    dom = sweep_range<D, T>(S, J0, J1, p, q, my_tag, js, je, dom);
                }
                if (valid) S.keep[q] = dom ? 0 : 1;
            }
            __syncthreads();
            // --- exclusive scan of keep flags
            constexpr int QPER = kTileCap / kTileThreads;
            int32_t kept_local = 0;
#pragma unroll
            for (int r = 0; r < QPER; ++r) {
                const int q = tid * QPER + r;
                if (q < total) kept_local += S.keep[q];
            }
            const int32_t kex = block_exclusive_scan<int32_t, kTileThreads>(kept_local, S.warp_i, &S.tot_i);
            {
                int32_t run = kex;
#pragma unroll
                for (int r = 0; r < QPER; ++r) {
                    const int q = tid * QPER + r;
                    if (q < total) {
                        S.keep_ex[q] = run;
                        run += S.keep[q];
                    }
                }
                if (tid == kTileThreads - 1) S.keep_ex[total] = run;
            }
            __syncthreads();
            // --- write survivors into each destination's slot
            for (int q = tid; q < total; q += kTileThreads) {
                if (!S.keep[q]) continue;
                const int k = S.item_of[q];
                const int64_t dst = S.item_c0[k] + (S.keep_ex[q] - S.keep_ex[S.item_s[k]]);
                T *o_ = outp + dst * D;
                const PackedPt<D, T> me = S.pts[q];
#pragma unroll
                for (int o = 0; o < D; ++o) o_[o] = me.v[o];
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

cudaError_t launch_expand_tiles(int d, bool wide, const ExpandJob *jobs, int num_jobs, int64_t total_tiles, int grid,
                                cudaStream_t stream) {
    if (wide) { PMDD_DISPATCH_D(d, (launch_expand_tiles_t<DD, int64_t>(jobs, num_jobs, total_tiles, grid, stream))); }
    PMDD_DISPATCH_D(d, (launch_expand_tiles_t<DD, int32_t>(jobs, num_jobs, total_tiles, grid, stream)));
}

}  // namespace dev
}  // namespace pmdd
