// Next-layer counting: per-arc candidate offsets (exclusive scan of the neighbour's
// frontier size), destination sizes, the list of oversized destinations with their
// scratch offsets, and the current layer's survivor total.  One block per job.
//
// In a chained layer (chain.cu) the block also sizes its request's next chained
// expansion from these counts -- candidates and tiles, or a stop at an oversized
// destination, a full buffer or the request's last chained layer -- and writes that
// expansion's tile plan (each tile's first destination, as tile_plan_kernel does); the
// last block of the launch to finish then writes the first tile of every request, so
// the next layer's tile kernel follows with no other launch in between.
#include "kernels.cuh"
#include "scan.cuh"

namespace pmdd {
namespace dev {

namespace {

// Next chained expansion of the block's request (every thread of the block calls it).
__device__ void chain_next(const CountJob &J, bool skip, int64_t *warp_buf, int64_t *s_total) {
    __shared__ int64_t s_tiles;
    __shared__ int s_last;
    ExpandJob &N = *J.next;
    const int tid = threadIdx.x;
    if (tid == 0) {
        int64_t tiles = 0;
        bool stop = skip || J.next_layer > J.last;
        if (!stop) {
            const CountResult r = *J.result;  // written by this block's thread 0
            stop = r.num_big > 0 || r.total > J.cap || !chain_side_goes_on(r.total, J.other_score, J.bu != 0);
            if (!stop) {
                tiles = r.total > 0 ? (r.total + N.tile_window - 1) / N.tile_window : 1;
                N.total_cand = r.total;
                N.num_tiles = tiles;
            }
        }
        if (stop) {
            N.total_cand = 0;
            N.num_tiles = 0;
            if (*J.stop == 0) {
                *J.stop = 1;
                *J.stopped_at = J.next_layer;
            }
        }
        s_tiles = tiles;
    }
    __syncthreads();
    const int64_t T = s_tiles;
    if (T > 0) {  // tile plan: destination i belongs to tile min(start_i / window, T - 1)
        auto tile_of = [&](int32_t k) -> int64_t {
            const int64_t t = item_start(N.item_arc_off, J.arc_cand_off, N.item_base, N.arc_base, k) / N.tile_window;
            return t < T - 1 ? t : T - 1;
        };
        for (int32_t i = tid; i < N.num_items; i += kCountThreads) {
            const int64_t ti = tile_of(i);
            const int64_t tp = i == 0 ? -1 : tile_of(i - 1);
            for (int64_t t = tp + 1; t <= ti; ++t) N.tile_first[t] = i;
            if (i == N.num_items - 1)
                for (int64_t t = ti + 1; t <= T; ++t) N.tile_first[t] = N.num_items;
        }
    }
    // the last block to finish writes every request's first tile
    if (tid == 0) {
        J.next_tiles[J.slot] = T;
        __threadfence();
        s_last = atomicAdd(J.done, 1u) == static_cast<unsigned>(J.chain_n - 1) ? 1 : 0;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int base = 0; base < J.chain_n; base += kCountThreads) {  // chain_n <= kChainThreads
        const int k = base + tid;
        const int64_t x = k < J.chain_n ? __ldcg(J.next_tiles + k) : 0;
        const int64_t ex = block_exclusive_scan<int64_t, kCountThreads>(x, warp_buf, s_total);
        if (k < J.chain_n) J.next_bases[k] = ex;
    }
    if (tid == 0) *J.next_total = *s_total;
}

// The counts of one job (every thread of the block calls it).
__device__ void count_body(const CountJob &J, int64_t *warp_buf) {
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

}  // namespace

__global__ void __launch_bounds__(kCountThreads) count_scan_kernel(const CountJob *jobs) {
    const CountJob J = jobs[blockIdx.x];
    // a chained request whose expansion before did not run has nothing to count
    const bool skip = J.stop != nullptr && *J.stop != 0;
    __shared__ int64_t warp_buf[32];
    __shared__ int64_t s_sum;
    if (!skip) count_body(J, warp_buf);
    if (J.next != nullptr) {
        __syncthreads();
        chain_next(J, skip, warp_buf, &s_sum);
    }
}

cudaError_t launch_count_scan(const CountJob *jobs, int num_jobs, cudaStream_t stream) {
    if (num_jobs <= 0) return cudaSuccess;
    count_scan_kernel<<<num_jobs, kCountThreads, 0, stream>>>(jobs);
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace pmdd
