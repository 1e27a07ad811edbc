// Oversized destinations (those tile_resident() rejects).  Their candidates are
// materialised in scratch (big_expand_kernel), then filtered one of two ways.
//
// Below ExpandJob::big_mark_min candidates: one block per destination runs the
// sort-filter-skyline of sfs.cuh (big_sfs_kernel), which compares each point only with
// the maxima found so far; many such destinations keep the GPU busy side by side.
//
// From big_mark_min candidates up, one block would take far longer than the rest of the
// step, so the destination is filtered across the whole GPU:
//
//   big_mark_kernel:  one block per 256 candidates of a destination, so a destination
//       of n candidates is spread over ceil(n / 256) blocks.  The block streams the
//       destination's candidates through shared memory in tiles; each warp sweeps a tile
//       for its 32 candidates with warp-uniform broadcast reads, skipping the
//       candidates' own arc run (shifts of one non-dominated, duplicate-free parent
//       frontier never dominate each other).  A point before the run dominates on >=
//       alone, a point after it only when it also differs (equal points: the first
//       stays).  The block stops once all of its candidates are dominated.
//   big_write_kernel: one block per destination compacts the survivors, in candidate
//       order, into the destination's slot and writes its size.
//
// The GPU-wide pass compares a survivor with every candidate of the other arc runs
// (quadratic work); the SFS block does less work but runs on one SM.
#include "kernels.cuh"
#include "sfs.cuh"

#include <algorithm>

namespace pmdd {
namespace dev {

namespace {

constexpr int kMarkThreads = 256;
constexpr int kWriteThreads = 512;
constexpr unsigned kFull = 0xffffffffu;

template <int D, typename T>
struct MarkCfg {
    static constexpr int kTile = 32768 / static_cast<int>(sizeof(PackedPt<D, T>));  // points per shared tile
};

struct BigItem {
    int32_t item;      // job-local destination
    int32_t a0, a1;    // its arcs (global ids)
    int64_t soff;      // scratch offset (candidates) within this pass's window
    int64_t c0;        // job-local candidate start (the slot start)
    int64_t n;         // candidates
};

// The destination of work item W, if pass `pass` takes it (its scratch offset lies in the
// pass's window); its scratch offset is then re-based to the window.
__device__ __forceinline__ bool big_item(const ExpandJob &J, const BigWork &W, int64_t pass, BigItem *b) {
    const int64_t lo = pass * J.big_window;
    b->soff = J.big_list[2 * W.big + 1];
    if (b->soff < lo || b->soff >= lo + J.big_window) return false;
    b->soff -= lo;
    b->item = static_cast<int32_t>(J.big_list[2 * W.big]);
    const int32_t v = J.item_base + b->item;
    b->a0 = J.item_arc_off[v];
    b->a1 = J.item_arc_off[v + 1];
    b->c0 = J.arc_cand_off[b->a0 - J.arc_base];
    b->n = J.arc_cand_off[b->a1 - J.arc_base] - b->c0;
    return true;
}

}  // namespace

// Materialise the candidates of one oversized destination (AoS, D values each).
template <int D, typename T>
__global__ void __launch_bounds__(kBigThreads) big_expand_kernel(const ExpandJob *__restrict__ jobs,
                                                                 const BigWork *__restrict__ work, int64_t pass) {
    const BigWork W = work[blockIdx.y];
    const ExpandJob &J = jobs[W.job];
    BigItem B;
    if (!big_item(J, W, pass, &B)) return;
    T *spts = static_cast<T *>(J.big_pts);
    const T *prev = static_cast<const T *>(J.prev_pts);
    for (int32_t a = B.a0; a < B.a1; ++a) {
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
            const int64_t dst = B.soff + (b - B.c0) + idx;
#pragma unroll
            for (int o = 0; o < D; ++o) spts[dst * D + o] = src[idx * D + o] + wv[o];
        }
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

template <int D, typename T>
__global__ void __launch_bounds__(kMarkThreads) big_mark_kernel(const ExpandJob *__restrict__ jobs,
                                                                const BigWork *__restrict__ work, int64_t pass) {
    constexpr int TY = MarkCfg<D, T>::kTile;
    __shared__ PackedPt<D, T> ys[TY];
    const BigWork W = work[blockIdx.y];
    const ExpandJob &J = jobs[W.job];
    BigItem B;
    if (!big_item(J, W, pass, &B) || B.n < J.big_mark_min) return;
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kMarkThreads;
    if (base >= B.n) return;  // the whole block leaves together
    const T *P = static_cast<const T *>(J.big_pts) + B.soff * D;
    uint8_t *keep = reinterpret_cast<uint8_t *>(J.big_idx) + B.soff;
    const int tid = threadIdx.x;
    const int64_t i = base + tid;
    const bool valid = i < B.n;
    // this candidate's arc run [rs, re) (destination-local positions)
    int64_t rs = 0, re = 0;
    T p[D];
    if (valid) {
        int lo = B.a0, hi = B.a1 - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (J.arc_cand_off[mid - J.arc_base] - B.c0 <= i) lo = mid;
            else hi = mid - 1;
        }
        rs = J.arc_cand_off[lo - J.arc_base] - B.c0;
        re = J.arc_cand_off[lo + 1 - J.arc_base] - B.c0;
#pragma unroll
        for (int o = 0; o < D; ++o) p[o] = P[i * D + o];
    } else {
#pragma unroll
        for (int o = 0; o < D; ++o) p[o] = T(0);
    }
    const int64_t rs0 = __shfl_sync(kFull, rs, 0), re0 = __shfl_sync(kFull, re, 0);
    const bool uni = __all_sync(kFull, valid && rs == rs0 && re == re0);
    bool dom = !valid;
    for (int64_t t0 = 0; t0 < B.n; t0 += TY) {
        const int cnt = static_cast<int>(B.n - t0 < TY ? B.n - t0 : TY);
        for (int k = tid; k < cnt; k += kMarkThreads) ys[k] = load_global_pt<D, T>(P, t0 + k);
        __syncthreads();
        if (!__all_sync(kFull, dom)) {
            if (uni) {
                // tile positions before the run, then after it
                const int64_t bb = rs0 - t0, aa = re0 - t0;
                const int b_end = static_cast<int>(bb < 0 ? 0 : (bb > cnt ? cnt : bb));
                const int a_beg = static_cast<int>(aa < 0 ? 0 : (aa > cnt ? cnt : aa));
                dom = sweep_before<D, T>(ys, 0, b_end, p, dom);
                if (!__all_sync(kFull, dom)) dom = sweep_after<D, T>(ys, a_beg, cnt, p, dom);
            } else {
                for (int j = 0; j < cnt; ++j) {
                    const int64_t jg = t0 + j;
                    const PackedPt<D, T> c = ys[j];
                    if (!dom && (jg < rs || jg >= re) && ge_all<D, T>(c, p) && (jg < i || !eq_all<D, T>(c, p)))
                        dom = true;
                    if ((j & 31) == 31 && __all_sync(kFull, dom)) break;
                }
            }
        }
        if (__syncthreads_and(dom)) break;  // also: the tile may be overwritten now
    }
    if (valid) keep[i] = dom ? 0 : 1;
}

template <int D, typename T>
__global__ void __launch_bounds__(kWriteThreads) big_write_kernel(const ExpandJob *__restrict__ jobs,
                                                                  const BigWork *__restrict__ work, int64_t pass) {
    __shared__ int32_t warp_buf[32];
    __shared__ int32_t s_total;
    const BigWork W = work[blockIdx.x];
    const ExpandJob &J = jobs[W.job];
    BigItem B;
    if (!big_item(J, W, pass, &B) || B.n < J.big_mark_min) return;
    const T *P = static_cast<const T *>(J.big_pts) + B.soff * D;
    const uint8_t *keep = reinterpret_cast<const uint8_t *>(J.big_idx) + B.soff;
    T *out = static_cast<T *>(J.out_pts) + B.c0 * D;
    int64_t carry = 0;
    for (int64_t b0 = 0; b0 < B.n; b0 += kWriteThreads) {
        const int64_t i = b0 + threadIdx.x;
        const int32_t k = i < B.n ? keep[i] : 0;
        const int32_t ex = block_exclusive_scan<int32_t, kWriteThreads>(k, warp_buf, &s_total);
        if (k) {
#pragma unroll
            for (int o = 0; o < D; ++o) out[(carry + ex) * D + o] = P[i * D + o];
        }
        carry += s_total;
    }
    if (threadIdx.x == 0) J.out_size[B.item] = static_cast<int32_t>(carry);
}

// Destinations below big_mark_min candidates: one block each.
template <int D, typename T>
__global__ void __launch_bounds__(SfsCfg<D, T>::kThreads) big_sfs_kernel(const ExpandJob *__restrict__ jobs,
                                                                         const BigWork *__restrict__ work,
                                                                         int64_t pass) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const BigWork W = work[blockIdx.x];
    const ExpandJob &J = jobs[W.job];
    BigItem B;
    if (!big_item(J, W, pass, &B) || B.n >= J.big_mark_min) return;
    SfsScratch<T> s;
    s.P2 = static_cast<T *>(J.big_pts2) + B.soff * D;
    s.I2 = J.big_idx + B.soff;
    s.SV = static_cast<T *>(J.big_surv) + B.soff * D;
    s.SVI = J.big_surv_idx + B.soff;
    const int32_t kept = sfs_block<D, T>(smem_raw, static_cast<const T *>(J.big_pts) + B.soff * D, B.n, s,
                                         static_cast<T *>(J.out_pts) + B.c0 * D);
    if (threadIdx.x == 0) J.out_size[B.item] = kept;
}

template <int D, typename T>
static cudaError_t launch_big_t(const ExpandJob *jobs, const BigWork *work, int num_work, int64_t max_item,
                                bool with_mark, int64_t pass, cudaStream_t stream) {
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
    const unsigned gx_mark = static_cast<unsigned>(std::max<int64_t>(1, (max_item + kMarkThreads - 1) / kMarkThreads));
    constexpr int kMaxY = 65535;  // grid.y limit
    for (int w0 = 0; w0 < num_work; w0 += kMaxY) {
        const int nw = std::min(kMaxY, num_work - w0);
        big_expand_kernel<D, T><<<dim3(gx_expand, nw), kBigThreads, 0, stream>>>(jobs, work + w0, pass);
    }
    big_sfs_kernel<D, T><<<num_work, Cfg::kThreads, Cfg::kSmem, stream>>>(jobs, work, pass);
    if (with_mark) {
        for (int w0 = 0; w0 < num_work; w0 += kMaxY) {
            const int nw = std::min(kMaxY, num_work - w0);
            big_mark_kernel<D, T><<<dim3(gx_mark, nw), kMarkThreads, 0, stream>>>(jobs, work + w0, pass);
        }
        big_write_kernel<D, T><<<num_work, kWriteThreads, 0, stream>>>(jobs, work, pass);
    }
    return cudaGetLastError();
}

cudaError_t launch_big(int d, bool wide, const ExpandJob *jobs, const BigWork *work, int num_work, int64_t max_item,
                       bool with_mark, int64_t pass, cudaStream_t stream) {
    if (wide) {
        PMDD_DISPATCH_D(d, (launch_big_t<DD, int64_t>(jobs, work, num_work, max_item, with_mark, pass, stream)));
    }
    PMDD_DISPATCH_D(d, (launch_big_t<DD, int32_t>(jobs, work, num_work, max_item, with_mark, pass, stream)));
}

}  // namespace dev
}  // namespace pmdd
