// Next-layer counting: per-arc candidate offsets (exclusive scan of the neighbour's
// frontier size), destination sizes, the list of oversized destinations with their
// scratch offsets, and the current layer's survivor total.  One block per job.
#include "kernels.cuh"
#include "scan.cuh"

namespace pmdd {
namespace dev {

__global__ void __launch_bounds__(kCountThreads) count_scan_kernel(const CountJob *jobs) {
    const CountJob J = jobs[blockIdx.x];
    __shared__ int64_t warp_buf[32];
    __shared__ int64_t s_total;
    __shared__ int64_t s_carry;
    __shared__ unsigned long long s_max;
    __shared__ int s_nbig;
    __shared__ int s_maxarcs;
    const int tid = threadIdx.x;
    if (tid == 0) {
        s_carry = 0;
        s_max = 0;
        s_nbig = 0;
        s_maxarcs = 0;
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
        if (c > 0 && !tile_resident(c, J.item_arc_off[v + 1] - J.item_arc_off[v])) {
            atomicMax(&s_maxarcs, J.item_arc_off[v + 1] - J.item_arc_off[v]);
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
        J.result->max_big_arcs = s_maxarcs;
    }
}

cudaError_t launch_count_scan(const CountJob *jobs, int num_jobs, cudaStream_t stream) {
    if (num_jobs <= 0) return cudaSuccess;
    count_scan_kernel<<<num_jobs, kCountThreads, 0, stream>>>(jobs);
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace pmdd
