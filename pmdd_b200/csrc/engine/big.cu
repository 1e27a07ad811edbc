// Oversized destinations (those tile_resident() rejects): candidates are materialised
// in scratch, then filtered by the block-wide sort-filter-skyline sweep of sfs.cuh,
// whose output is the destination's slot in the next layer's frontier.
#include "kernels.cuh"
#include "sfs.cuh"

#include <algorithm>

namespace pmdd {
namespace dev {

// Materialise the candidates of one oversized destination (AoS, D values each).
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

// One block per oversized destination.
template <int D, typename T>
__global__ void __launch_bounds__(SfsCfg<D, T>::kThreads) big_sfs_kernel(const ExpandJob *__restrict__ jobs,
                                                                         const BigWork *__restrict__ work) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const BigWork W = work[blockIdx.x];
    const ExpandJob &J = jobs[W.job];
    const int32_t item = static_cast<int32_t>(J.big_list[2 * W.big]);
    const int64_t soff = J.big_list[2 * W.big + 1];
    const int32_t v = J.item_base + item;
    const int64_t s0 = J.arc_cand_off[J.item_arc_off[v] - J.arc_base];
    const int64_t n = J.arc_cand_off[J.item_arc_off[v + 1] - J.arc_base] - s0;
    SfsScratch<T> s;
    s.P2 = static_cast<T *>(J.big_pts2) + soff * D;
    s.I2 = J.big_idx + soff;
    s.SV = static_cast<T *>(J.big_surv) + soff * D;
    s.SVI = J.big_surv_idx + soff;
    const int32_t kept = sfs_block<D, T>(smem_raw, static_cast<const T *>(J.big_pts) + soff * D, n, s,
                                         static_cast<T *>(J.out_pts) + s0 * D);
    if (threadIdx.x == 0) J.out_size[item] = kept;
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

cudaError_t launch_big(int d, bool wide, const ExpandJob *jobs, const BigWork *work, int num_work, int64_t max_item,
                       int sms, cudaStream_t stream) {
    if (wide) { PMDD_DISPATCH_D(d, (launch_big_t<DD, int64_t>(jobs, work, num_work, max_item, sms, stream))); }
    PMDD_DISPATCH_D(d, (launch_big_t<DD, int32_t>(jobs, work, num_work, max_item, sms, stream)));
}

}  // namespace dev
}  // namespace pmdd
