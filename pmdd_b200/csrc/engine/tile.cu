// Fused expand + dominance filter over candidate tiles (the per-layer hot kernel).
//
// A tile owns every destination assigned to it by tile_plan_kernel (those whose
// candidate range starts inside the tile's window of J.tile_window <= kTileWindow
// candidates);
// destinations with at most kSmallMax candidates are handled here entirely in shared
// memory, larger ones only get their slot offset (the oversized path in big.cu filters
// them).  A tile therefore holds < kTileCap points.
//
//   stage:   the tile's destinations and their arcs (candidate offsets, parent slot
//            starts, weight rows) are read once into shared memory;
//   expand:  candidate = parent frontier point + arc weight vector; consecutive
//            candidates of an arc are consecutive parent points, so loads coalesce and
//            each candidate costs one independent global load;
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

constexpr int kTT = kTileThreads;

template <int D, typename T>
struct TileSmem {
    PackedPt<D, T> pts[kTileCap];
    int16_t tag[kTileCap];              // staged arc of each candidate
    uint16_t item_of[kTileCap];         // staged destination of each candidate
    uint8_t keep[kTileCap];
    int16_t keep_ex[kTileCap + 1];      // exclusive scan of keep flags
    int16_t item_s[kTileItemCap + 1];   // staged destination -> first candidate position
    int16_t item_arc0[kTileItemCap + 1];  // staged destination -> first staged arc
    int32_t item_a0g[kTileItemCap];     // staged destination -> first arc (global id)
    int64_t item_c0[kTileItemCap];      // staged destination -> job-local candidate start
    int16_t arc_pos[kTileArcCap + 1];   // staged arc -> first candidate position
    int32_t arc_w[kTileArcCap];         // staged arc -> weight row
    int64_t arc_src[kTileArcCap];       // staged arc -> parent slot start (points)
    int32_t warp_i[32];
    int32_t tot_i;
    int32_t tot_a;
    int32_t i0, i1;
    int32_t job;
    int32_t chunk;                      // next 32-candidate chunk to filter
    int64_t tile;                       // tile taken from the launch's queue
};

// ------------------------------------------------------------------ tile plan
__global__ void tile_plan_kernel(const ExpandJob *__restrict__ jobs, const int64_t *__restrict__ item_bases,
                                 int num_jobs, int64_t total_items) {
    for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < total_items;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int j = find_base(item_bases, num_jobs, g);
        const ExpandJob &J = jobs[j];
        const int32_t i = static_cast<int32_t>(g - item_bases[j]);
        const int64_t T = J.num_tiles;
        if (T == 0) continue;  // a chained expansion that stopped (chain.cu)
        auto tile_of = [&](int32_t k) -> int64_t {
            const int64_t s = item_start(J.item_arc_off, J.arc_cand_off, J.item_base, J.arc_base, k);
            const int64_t t = s / J.tile_window;
            return t < T - 1 ? t : T - 1;
        };
        const int64_t ti = tile_of(i);
        const int64_t tp = i == 0 ? -1 : tile_of(i - 1);
        for (int64_t t = tp + 1; t <= ti; ++t) J.tile_first[t] = i;
        if (i == J.num_items - 1)
            for (int64_t t = ti + 1; t <= T; ++t) J.tile_first[t] = J.num_items;
    }
}

cudaError_t launch_tile_plan(const ExpandJob *jobs, const int64_t *item_bases, int num_jobs, int64_t total_items,
                             cudaStream_t stream) {
    if (num_jobs <= 0 || total_items <= 0) return cudaSuccess;
    const int64_t g = std::min<int64_t>((total_items + 255) / 256, 148 * 16);
    tile_plan_kernel<<<static_cast<unsigned>(g), 256, 0, stream>>>(jobs, item_bases, num_jobs, total_items);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ the tile
// Warp sweep over [a, b) for 32 candidates: lane's candidate (p, position q, arc tag)
// is dominated by some j in [max(a, js), min(b, je)) with a different arc.
template <int D, typename T>
__device__ __forceinline__ bool sweep_range(const TileSmem<D, T> &S, int a, int b, const T (&p)[D], int q, int tag,
                                            int js, int je, bool dom) {
    for (int j = a; j < b; ++j) {
        const PackedPt<D, T> c = S.pts[j];
        const int tj = S.tag[j];
        if (!dom && ge_all<D, T>(c, p) && j >= js && j < je && tj != tag) {
            if (!eq_all<D, T>(c, p) || j < q) dom = true;
        }
        if ((j & 31) == 31 && __all_sync(0xffffffffu, dom)) return true;
    }
    return dom;
}

// The common case: every lane's candidate lies in the same arc run of the same
// destination, and [a, b) holds none of that run, so [a, b) lies wholly before or
// wholly after every lane's candidate.  No per-lane range or arc checks.  Points before
// the lanes dominate on >= alone (of equal points the first stays); points after them
// only when they also differ.
template <int D, typename T, bool kBefore>
__device__ __forceinline__ bool sweep_other_arcs(const TileSmem<D, T> &S, int a, int b, const T (&p)[D], bool dom) {
    int j = a;
    int it = 0;
    for (; j + 4 <= b; j += 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const PackedPt<D, T> c = S.pts[j + u];
            if (kBefore) dom |= ge_all<D, T>(c, p);
            else dom |= ge_all<D, T>(c, p) && !eq_all<D, T>(c, p);
        }
        if ((++it & 7) == 0 && __all_sync(0xffffffffu, dom)) return true;
    }
    for (; j < b; ++j) {
        const PackedPt<D, T> c = S.pts[j];
        if (kBefore) dom |= ge_all<D, T>(c, p);
        else dom |= ge_all<D, T>(c, p) && !eq_all<D, T>(c, p);
    }
    return dom;
}

template <int D, typename T>
__global__ void __launch_bounds__(kTT) expand_tile_kernel(const ExpandJob *__restrict__ jobs,
                                                          const int64_t *__restrict__ tile_bases, int num_jobs,
                                                          int64_t total_tiles, unsigned long long *queue,
                                                          const int64_t *tiles_dev) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TileSmem<D, T> &S = *reinterpret_cast<TileSmem<D, T> *>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31;
    // tiles are handed out by an atomic counter over all the launch's jobs, so a block
    // that drew cheap tiles takes more
    auto next_tile = [&]() -> int64_t {
        if (tid == 0) S.tile = static_cast<int64_t>(atomicAdd(queue, 1ull));
        __syncthreads();
        return S.tile;
    };
    // jobs sized on the device (chain.cu) publish their tiles' total there
    if (tiles_dev != nullptr) total_tiles = min(total_tiles, *tiles_dev);
    for (int64_t tile = next_tile(); tile < total_tiles; tile = next_tile()) {
        if (tid == 0) {
            const int j = find_base(tile_bases, num_jobs, tile);
            const ExpandJob &J = jobs[j];
            const int64_t t = tile - tile_bases[j];
            S.job = j;
            // a job sized on the device may have fewer tiles than the launch allows for
            S.i0 = t < J.num_tiles ? J.tile_first[t] : 0;
            S.i1 = t < J.num_tiles ? J.tile_first[t + 1] : 0;
        }
        __syncthreads();
        const ExpandJob &J = jobs[S.job];
        const int32_t i0 = S.i0, i1 = S.i1;
        const T *__restrict__ prev = static_cast<const T *>(J.prev_pts);
        T *__restrict__ outp = static_cast<T *>(J.out_pts);
        int32_t ic = i0;
        while (ic < i1) {
            const int n_stage = min(kTileItemCap, i1 - ic);
            // --- stage destinations: candidate starts and sizes, arc ranges
            constexpr int PER = kTileItemCap / kTT;
            int32_t cnt[PER], narc[PER];
            int32_t local = 0, local_a = 0;
#pragma unroll
            for (int r = 0; r < PER; ++r) {
                const int k = tid * PER + r;
                cnt[r] = 0;
                narc[r] = 0;
                if (k < n_stage) {
                    const int32_t i = ic + k;
                    const int32_t v = J.item_base + i;
                    const int32_t a0 = J.item_arc_off[v], a1 = J.item_arc_off[v + 1];
                    const int64_t s = J.arc_cand_off[a0 - J.arc_base];
                    const int64_t c = J.arc_cand_off[a1 - J.arc_base] - s;
                    J.out_off[i] = s;
                    if (c == 0) J.out_size[i] = 0;
                    if (J.out_sorted) J.out_sorted[i] = c == 0 ? 1 : 0;  // written in arc order
                    S.item_c0[k] = s;
                    S.item_a0g[k] = a0;
                    if (c > 0 && tile_resident(c, a1 - a0)) {
                        cnt[r] = static_cast<int32_t>(c);
                        narc[r] = a1 - a0;
                    }
                }
                local += cnt[r];
                local_a += narc[r];
            }
            const int32_t ex = block_exclusive_scan<int32_t, kTT>(local, S.warp_i, &S.tot_i);
            const int32_t exa = block_exclusive_scan<int32_t, kTT>(local_a, S.warp_i, &S.tot_a);
            // this pass takes the longest prefix of staged destinations whose arcs fit
            int32_t fit = 0;
            {
                int32_t run = ex, runa = exa;
#pragma unroll
                for (int r = 0; r < PER; ++r) {
                    const int k = tid * PER + r;
                    if (k < n_stage) {
                        S.item_s[k] = static_cast<int16_t>(run);
                        S.item_arc0[k] = static_cast<int16_t>(runa);
                        if (runa + narc[r] <= kTileArcCap) ++fit;
                    }
                    run += cnt[r];
                    runa += narc[r];
                }
            }
            const int32_t fit_ex = block_exclusive_scan<int32_t, kTT>(fit, S.warp_i, &S.tot_i);
            (void)fit_ex;
            const int n_it = S.tot_i;  // >= 1: one destination has at most kTileArcCap / 2 arcs
            if (n_it == 0) {           // impossible for well-formed plans; skip defensively
                if (tid == 0) atomicOr(J.err, kErrBounds);
                break;
            }
            __syncthreads();
            if (tid == 0) {
                // end markers of this pass
                int32_t e = S.item_s[n_it - 1], ea = S.item_arc0[n_it - 1];
                const int32_t v = J.item_base + ic + n_it - 1;
                const int32_t a0 = J.item_arc_off[v], a1 = J.item_arc_off[v + 1];
                const int64_t c = J.arc_cand_off[a1 - J.arc_base] - J.arc_cand_off[a0 - J.arc_base];
                if (c > 0 && tile_resident(c, a1 - a0)) {
                    e += static_cast<int32_t>(c);
                    ea += a1 - a0;
                }
                S.item_s[n_it] = static_cast<int16_t>(e);
                S.item_arc0[n_it] = static_cast<int16_t>(ea);
                S.tot_i = e;
                S.tot_a = ea;
                S.chunk = 0;
            }
            __syncthreads();
            const int32_t total = S.tot_i, total_a = S.tot_a;
            if (total > kTileCap || total_a > kTileArcCap) {  // impossible for well-formed offsets
                if (tid == 0) atomicOr(J.err, kErrBounds);
                break;
            }
            // --- stage the arcs of the small destinations
            for (int x = tid; x < total_a; x += kTT) {
                int lo = 0, hi = n_it - 1;  // destination owning staged arc x
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (S.item_arc0[mid] <= x) lo = mid;
                    else hi = mid - 1;
                }
                const int k = lo;
                const int32_t a = S.item_a0g[k] + (x - S.item_arc0[k]);
                const int64_t c0 = J.arc_cand_off[a - J.arc_base];
                S.arc_pos[x] = static_cast<int16_t>(S.item_s[k] + (c0 - S.item_c0[k]));
                S.arc_src[x] = J.prev_off[J.arc_nbr[a] - J.prev_base];
                S.arc_w[x] = J.arc_wrow[a];
            }
            if (tid == 0) S.arc_pos[total_a] = static_cast<int16_t>(total);
            __syncthreads();
            // --- expand: candidate = parent point + arc weight
            for (int q = tid; q < total; q += kTT) {
                int lo = 0, hi = n_it - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (S.item_s[mid] <= q) lo = mid;
                    else hi = mid - 1;
                }
                const int k = lo;
                int alo = S.item_arc0[k], ahi = S.item_arc0[k + 1] - 1;
                while (alo < ahi) {
                    const int mid = (alo + ahi + 1) >> 1;
                    if (S.arc_pos[mid] <= q) alo = mid;
                    else ahi = mid - 1;
                }
                const int x = alo;
                const int64_t idx = q - S.arc_pos[x];
                const T *src = prev + (S.arc_src[x] + idx) * D;
                const int32_t *w = J.weights + static_cast<int64_t>(S.arc_w[x]) * D;
                PackedPt<D, T> pt;
#pragma unroll
                for (int o = 0; o < PackedPt<D, T>::kPad; ++o) pt.v[o] = o < D ? src[o] + static_cast<T>(w[o]) : T(0);
                S.pts[q] = pt;
                S.tag[q] = static_cast<int16_t>(x);
                S.item_of[q] = static_cast<uint16_t>(k);
            }
            __syncthreads();
            // --- filter: warp per 32 candidates, uniform sweep over their destinations
            while (true) {
                int c0 = 0;
                if (lane == 0) c0 = atomicAdd(&S.chunk, 1) * 32;
                c0 = __shfl_sync(0xffffffffu, c0, 0);
                if (c0 >= total) break;
                const int q = c0 + lane;
                const bool valid = q < total;
                T p[D];
                int my_tag = -1;
                int js = INT_MAX, je = INT_MIN, slo = 0, shi = 0;
                if (valid) {
                    const PackedPt<D, T> me = S.pts[q];
#pragma unroll
                    for (int o = 0; o < D; ++o) p[o] = me.v[o];
                    my_tag = S.tag[q];
                    const int k = S.item_of[q];
                    js = S.item_s[k];
                    je = S.item_s[k + 1];
                    slo = S.arc_pos[my_tag];
                    shi = my_tag + 1 < S.item_arc0[k + 1] ? S.arc_pos[my_tag + 1] : je;
                } else {
#pragma unroll
                    for (int o = 0; o < D; ++o) p[o] = T(0);
                }
                const int J0 = warp_min_i(js), J1 = warp_max_i(je);
                // all lanes in one arc run: skip that run entirely
                const bool one_run = __all_sync(0xffffffffu, valid) && warp_min_i(my_tag) == warp_max_i(my_tag);
                bool dom = !valid;
                if (one_run) {
                    dom = sweep_other_arcs<D, T, true>(S, J0, slo, p, dom);
                    if (!__all_sync(0xffffffffu, dom)) dom = sweep_other_arcs<D, T, false>(S, shi, J1, p, dom);
                } else {
                    dom = sweep_range<D, T>(S, J0, J1, p, q, my_tag, js, je, dom);
                }
                if (valid) S.keep[q] = dom ? 0 : 1;
            }
            __syncthreads();
            // --- exclusive scan of keep flags
            constexpr int QPER = kTileCap / kTT;
            int32_t kept_local = 0;
#pragma unroll
            for (int r = 0; r < QPER; ++r) {
                const int q = tid * QPER + r;
                if (q < total) kept_local += S.keep[q];
            }
            const int32_t kex = block_exclusive_scan<int32_t, kTT>(kept_local, S.warp_i, &S.tot_i);
            {
                int32_t run = kex;
#pragma unroll
                for (int r = 0; r < QPER; ++r) {
                    const int q = tid * QPER + r;
                    if (q < total) {
                        S.keep_ex[q] = static_cast<int16_t>(run);
                        run += S.keep[q];
                    }
                }
                if (tid == kTT - 1) S.keep_ex[total] = static_cast<int16_t>(run);
            }
            __syncthreads();
            if (tid == 0 && J.tile_surv != nullptr && S.keep_ex[total] > 0)
                atomicAdd(J.tile_surv, static_cast<unsigned long long>(S.keep_ex[total]));
            // --- write survivors into each destination's slot
            for (int q = tid; q < total; q += kTT) {
                if (!S.keep[q]) continue;
                const int k = S.item_of[q];
                const int64_t dst = S.item_c0[k] + (S.keep_ex[q] - S.keep_ex[S.item_s[k]]);
                T *o_ = outp + dst * D;
                const PackedPt<D, T> me = S.pts[q];
#pragma unroll
                for (int o = 0; o < D; ++o) o_[o] = me.v[o];
            }
            for (int k = tid; k < n_it; k += kTT) {
                const int js = S.item_s[k], je = S.item_s[k + 1];
                if (je > js) J.out_size[ic + k] = S.keep_ex[je] - S.keep_ex[js];
            }
            __syncthreads();
            ic += n_it;
        }
        __syncthreads();  // tile bookkeeping in shared memory is rewritten next iteration
    }
}

template <int D, typename T>
static cudaError_t launch_expand_tiles_t(const ExpandJob *jobs, const int64_t *tile_bases, int num_jobs,
                                         int64_t total_tiles, int grid, unsigned long long *queue,
                                         const int64_t *tiles_dev, cudaStream_t stream) {
    const size_t smem = sizeof(TileSmem<D, T>);
    {
        const cudaError_t e = ensure_smem_limit(reinterpret_cast<const void *>(expand_tile_kernel<D, T>), smem);
        if (e != cudaSuccess) return e;
    }
    if (total_tiles <= 0) return cudaSuccess;
    const int64_t g = std::min<int64_t>(total_tiles, grid);
    expand_tile_kernel<D, T><<<static_cast<unsigned>(g), kTT, smem, stream>>>(jobs, tile_bases, num_jobs, total_tiles,
                                                                                queue, tiles_dev);
    return cudaGetLastError();
}

cudaError_t launch_expand_tiles(int d, bool wide, const ExpandJob *jobs, const int64_t *tile_bases, int num_jobs,
                                int64_t total_tiles, int grid, unsigned long long *queue, const int64_t *tiles_dev,
                                cudaStream_t stream) {
    if (wide) {
        PMDD_DISPATCH_D(d, (launch_expand_tiles_t<DD, int64_t>(jobs, tile_bases, num_jobs, total_tiles, grid, queue,
                                                               tiles_dev, stream)));
    }
    PMDD_DISPATCH_D(d, (launch_expand_tiles_t<DD, int32_t>(jobs, tile_bases, num_jobs, total_tiles, grid, queue,
                                                           tiles_dev, stream)));
}

}  // namespace dev
}  // namespace pmdd
