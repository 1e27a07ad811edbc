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
// Scratch of a job's oversized destination `big`: its points start at big_list[2*big+1].
// Materialise the candidates of one oversized destination (AoS) with their arcs.
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
            J.big_tag[dst] = a;
        }
    }
}

// Pairwise filter of one oversized destination: block x handles candidates
// [x*256, ...) striding by gridDim.x*256 and sweeps shared-memory tiles of the whole
// destination, leaving the sweep as soon as every candidate of the block is decided.
template <int D, typename T>
__global__ void __launch_bounds__(kBigThreads) big_filter_kernel(const ExpandJob *__restrict__ jobs,
                                                                 const BigWork *__restrict__ work) {
    constexpr int JT = (kBigJTile * D * static_cast<int>(sizeof(T)) > 32768)
                           ? 32768 / (D * static_cast<int>(sizeof(T)))
                           : kBigJTile;
    __shared__ T sj[D][JT];
    __shared__ int32_t st[JT];
    const BigWork W = work[blockIdx.y];
    const ExpandJob &J = jobs[W.job];
    const int32_t item = static_cast<int32_t>(J.big_list[2 * W.big]);
    const int64_t soff = J.big_list[2 * W.big + 1];
    const T *spts = static_cast<const T *>(J.big_pts);
    const int32_t *stag = J.big_tag;
    const int32_t v = J.item_base + item;
    const int64_t n = J.arc_cand_off[J.item_arc_off[v + 1] - J.arc_base] - J.arc_cand_off[J.item_arc_off[v] - J.arc_base];
    for (int64_t i0 = static_cast<int64_t>(blockIdx.x) * kBigThreads; i0 < n;
         i0 += static_cast<int64_t>(gridDim.x) * kBigThreads) {
        const int64_t i = i0 + threadIdx.x;
        const bool valid = i < n;
        T p[D];
        int32_t my_tag = -1;
        if (valid) {
#pragma unroll
            for (int o = 0; o < D; ++o) p[o] = spts[(soff + i) * D + o];
            my_tag = stag[soff + i];
        }
        bool dom = !valid;
        for (int64_t j0 = 0; j0 < n; j0 += JT) {
            if (__syncthreads_and(dom)) break;
            const int m = static_cast<int>(n - j0 < JT ? n - j0 : static_cast<int64_t>(JT));
            for (int k = threadIdx.x; k < m; k += kBigThreads) {
#pragma unroll
                for (int o = 0; o < D; ++o) sj[o][k] = spts[(soff + j0 + k) * D + o];
                st[k] = stag[soff + j0 + k];
            }
            __syncthreads();
            if (!dom) {
                for (int k = 0; k < m; ++k) {
                    if (st[k] == my_tag) continue;
                    bool ge = true, eq = true;
#pragma unroll
                    for (int o = 0; o < D; ++o) {
                        const T x = sj[o][k];
                        ge &= (x >= p[o]);
                        eq &= (x == p[o]);
                    }
                    if (ge && (!eq || j0 + k < i)) {
                        dom = true;
                        break;
                    }
                }
            }
        }
        if (valid) J.big_keep[soff + i] = dom ? 0 : 1;
        __syncthreads();
    }
}

// Compaction of one oversized destination into its slot, and its survivor count.
template <int D, typename T>
__global__ void __launch_bounds__(kCountThreads) big_compact_kernel(const ExpandJob *__restrict__ jobs,
                                                                    const BigWork *__restrict__ work) {
    __shared__ int32_t warp_buf[32];
    __shared__ int32_t s_total;
    __shared__ int64_t s_carry;
    const BigWork W = work[blockIdx.x];
    const ExpandJob &J = jobs[W.job];
    const int32_t item = static_cast<int32_t>(J.big_list[2 * W.big]);
    const int64_t soff = J.big_list[2 * W.big + 1];
    const T *spts = static_cast<const T *>(J.big_pts);
    const int32_t v = J.item_base + item;
    const int64_t s = J.arc_cand_off[J.item_arc_off[v] - J.arc_base];
    const int64_t n = J.arc_cand_off[J.item_arc_off[v + 1] - J.arc_base] - s;
    T *outp = static_cast<T *>(J.out_pts);
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < n; base += kCountThreads) {
        const int64_t i = base + threadIdx.x;
        const int32_t k = (i < n && J.big_keep[soff + i]) ? 1 : 0;
        const int32_t ex = block_exclusive_scan<int32_t, kCountThreads>(k, warp_buf, &s_total);
        if (k) {
            const int64_t dst = s + s_carry + ex;
#pragma unroll
            for (int o = 0; o < D; ++o) outp[dst * D + o] = spts[(soff + i) * D + o];
        }
        __syncthreads();  // every thread has read s_carry
        if (threadIdx.x == 0) s_carry += s_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) J.out_size[item] = static_cast<int32_t>(s_carry);
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
    const int64_t chunks = (max_item + kBigThreads - 1) / kBigThreads;
    const unsigned gx_expand = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(chunks, 64)));
    // enough blocks per destination to fill the SMs when few destinations are big
    int64_t per = std::max<int64_t>(1, (static_cast<int64_t>(sms) * 8) / num_work);
    per = std::max<int64_t>(1, std::min<int64_t>(per, chunks));
    constexpr int kMaxY = 65535;  // grid.y limit
    for (int w0 = 0; w0 < num_work; w0 += kMaxY) {
        const int nw = std::min(kMaxY, num_work - w0);
        big_expand_kernel<D, T><<<dim3(gx_expand, nw), kBigThreads, 0, stream>>>(jobs, work + w0);
    }
    for (int w0 = 0; w0 < num_work; w0 += kMaxY) {
        const int nw = std::min(kMaxY, num_work - w0);
        big_filter_kernel<D, T><<<dim3(static_cast<unsigned>(per), nw), kBigThreads, 0, stream>>>(jobs, work + w0);
    }
    big_compact_kernel<D, T><<<num_work, kCountThreads, 0, stream>>>(jobs, work);
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
