// State dominance (knapsack and set packing): one warp per node of every job's layer, in
// two launches (mark against the labels as they were, then compact each node's slot in
// place).
#include <algorithm>

#include "scan.cuh"
#include "statedom.cuh"

namespace pmdd {
namespace dev {

namespace {

constexpr int kSdThreads = 256;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int find_job(const int64_t *node_bases, int num_jobs, int64_t w) {
    int lo = 0, hi = num_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (node_bases[mid] <= w) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Arc index of a node's only incoming arc, or -1.
__device__ __forceinline__ int32_t single_in_arc(const StateDomJob &J, int32_t local) {
    const int32_t v = J.node_base + local;
    const int32_t a = J.in_off[v];
    return J.in_off[v + 1] - a == 1 ? a : -1;
}

// Lowest vertex of a set-packing state, or -1 for the empty state.
__device__ __forceinline__ int first_vertex(const uint64_t *s, int W) {
    for (int w = 0; w < W; ++w)
        if (s[w] != 0) return w * 64 + __ffsll(static_cast<long long>(s[w])) - 1;
    return -1;
}

template <int D, typename T>
__global__ void __launch_bounds__(kSdThreads) sd_mark_kernel(const StateDomJob *jobs, const int64_t *node_bases,
                                                             int num_jobs, int64_t total) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (kSdThreads / 32);
    for (int64_t w = static_cast<int64_t>(blockIdx.x) * (kSdThreads / 32) + (threadIdx.x >> 5); w < total;
         w += warps) {
        const int j = find_job(node_bases, num_jobs, w);
        const StateDomJob &J = jobs[j];
        const int32_t pos = static_cast<int32_t>(w - node_bases[j]);
        const int32_t n1 = J.order[pos];
        const int32_t s1 = J.size[n1];
        if (s1 == 0) continue;
        // siblings under one single parent (through different arc types) are not compared
        const int32_t a1 = single_in_arc(J, n1);
        auto skipped = [&](int32_t n2) -> bool {
            if (n2 < 0 || a1 < 0) return false;
            const int32_t a2 = single_in_arc(J, n2);
            return a2 >= 0 && J.arc_src[a1] == J.arc_src[a2] && ((J.arc_w[a1] != 0) != (J.arc_w[a2] != 0));
        };
        int32_t part0 = -1, part1 = -1;
        if (J.kind == 2) {
            // first node of the partner bucket with the same lowest vertex, not a
            // single-parent sibling, whose state contains n1's
            const int32_t qb = J.next[2 * pos], qe = J.next[2 * pos + 1];
            const int W = J.state_words;
            const uint64_t *st1 = J.state + static_cast<int64_t>(J.node_base + n1) * W;
            const int ff1 = first_vertex(st1, W);
            for (int32_t p = qb; p < qe && part0 < 0; p += 32) {
                const int32_t q = p + lane;
                bool ok = false;
                if (q < qe) {
                    const int32_t n2 = J.order[q];
                    const uint64_t *st2 = J.state + static_cast<int64_t>(J.node_base + n2) * W;
                    ok = first_vertex(st2, W) == ff1 && !skipped(n2);
                    for (int w = 0; w < W && ok; ++w) ok = (st1[w] & ~st2[w]) == 0;
                }
                const unsigned m = __ballot_sync(kFull, ok);
                if (m != 0) part0 = J.order[p + __ffs(m) - 1];
            }
        } else {
            // the next two positions of the order whose node holds labels
            int found = 0;
            for (int32_t p = pos + 1; p < J.num_nodes && found < 2; p += 32) {
                const int32_t q = p + lane;
                const bool act = q < J.num_nodes && J.size[J.order[q]] > 0;
                unsigned m = __ballot_sync(kFull, act);
                while (m != 0 && found < 2) {
                    const int b = __ffs(m) - 1;
                    m &= m - 1;
                    const int32_t node = J.order[p + b];
                    if (found == 0) part0 = node;
                    else part1 = node;
                    ++found;
                }
            }
            if (skipped(part0)) part0 = -1;
            if (skipped(part1)) part1 = -1;
        }
        const T *P = static_cast<const T *>(J.pts);
        const int64_t o1 = J.off[n1];
        for (int32_t kb = 0; kb < s1; kb += 32) {
            const int32_t k = kb + lane;
            const bool valid = k < s1;
            T x[D];
#pragma unroll
            for (int o = 0; o < D; ++o) x[o] = valid ? P[(o1 + k) * D + o] : T(0);
            bool dom = !valid;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int32_t n2 = c == 0 ? part0 : part1;
                if (n2 < 0) continue;
                const int64_t o2 = J.off[n2];
                const int32_t s2 = J.size[n2];
                for (int32_t t = 0; t < s2; ++t) {
                    if (__all_sync(kFull, dom)) break;
                    bool ge = true;
#pragma unroll
                    for (int o = 0; o < D; ++o) ge &= (P[(o2 + t) * D + o] >= x[o]);
                    dom |= ge;
                }
            }
            if (valid) J.keep[o1 + k] = dom ? 0 : 1;
        }
    }
}

template <int D, typename T>
__global__ void __launch_bounds__(kSdThreads) sd_compact_kernel(const StateDomJob *jobs, const int64_t *node_bases,
                                                                int num_jobs, int64_t total) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (kSdThreads / 32);
    for (int64_t w = static_cast<int64_t>(blockIdx.x) * (kSdThreads / 32) + (threadIdx.x >> 5); w < total;
         w += warps) {
        const int j = find_job(node_bases, num_jobs, w);
        const StateDomJob &J = jobs[j];
        const int32_t n = static_cast<int32_t>(w - node_bases[j]);
        const int32_t s = J.size[n];
        if (s == 0) continue;
        T *P = static_cast<T *>(J.pts);
        const int64_t o = J.off[n];
        int32_t kept = 0;
        for (int32_t kb = 0; kb < s; kb += 32) {
            const int32_t k = kb + lane;
            const bool keep = k < s && J.keep[o + k] != 0;
            T x[D];
#pragma unroll
            for (int q = 0; q < D; ++q) x[q] = keep ? P[(o + k) * D + q] : T(0);
            const unsigned m = __ballot_sync(kFull, keep);  // every lane has loaded before any stores
            const int32_t dst = kept + __popc(m & ((1u << lane) - 1u));
            if (keep && dst != k) {
#pragma unroll
                for (int q = 0; q < D; ++q) P[(o + dst) * D + q] = x[q];
            }
            kept += __popc(m);
            __syncwarp();
        }
        if (lane == 0 && kept != s) {
            J.size[n] = kept;
            atomicAdd(reinterpret_cast<unsigned long long *>(J.removed), static_cast<unsigned long long>(s - kept));
        }
    }
}

template <int D, typename T>
cudaError_t launch_sd_t(const StateDomJob *jobs, const int64_t *node_bases, int num_jobs, int64_t total, int sms,
                        cudaStream_t stream) {
    if (num_jobs <= 0 || total <= 0) return cudaSuccess;
    const int64_t want = (total + kSdThreads / 32 - 1) / (kSdThreads / 32);
    const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(want, static_cast<int64_t>(sms) * 16)));
    sd_mark_kernel<D, T><<<grid, kSdThreads, 0, stream>>>(jobs, node_bases, num_jobs, total);
    sd_compact_kernel<D, T><<<grid, kSdThreads, 0, stream>>>(jobs, node_bases, num_jobs, total);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_state_dominance(int d, bool wide, const StateDomJob *jobs, const int64_t *node_bases, int num_jobs,
                                   int64_t total_nodes, int sms, cudaStream_t stream) {
    if (wide) { PMDD_DISPATCH_D(d, (launch_sd_t<DD, int64_t>(jobs, node_bases, num_jobs, total_nodes, sms, stream))); }
    PMDD_DISPATCH_D(d, (launch_sd_t<DD, int32_t>(jobs, node_bases, num_jobs, total_nodes, sms, stream)));
}

}  // namespace dev
}  // namespace pmdd
