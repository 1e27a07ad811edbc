// Block- and warp-level building blocks shared by the engine's kernels.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace pmdd {
namespace dev {

// Exclusive scan across a block of THREADS threads; *total receives the block sum.
// Contains __syncthreads(): every thread of the block must call it.
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

__device__ __forceinline__ int warp_min_i(int x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = min(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

__device__ __forceinline__ int warp_max_i(int x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = max(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

__device__ __forceinline__ int64_t warp_min_i64(int64_t x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = min(x, static_cast<int64_t>(__shfl_xor_sync(0xffffffffu, x, o)));
    return x;
}

// A point padded to a 16-byte multiple so that a warp reads one candidate from shared
// memory with vector loads that broadcast to all lanes.
template <int D, typename T>
struct alignas(16) PackedPt {
    static constexpr int kPad = (static_cast<int>(sizeof(T)) * D + 15) / 16 * 16 / static_cast<int>(sizeof(T));
    T v[kPad];
};

// q >= p on every objective
template <int D, typename T>
__device__ __forceinline__ bool ge_all(const PackedPt<D, T> &q, const T (&p)[D]) {
    bool ge = true;
#pragma unroll
    for (int o = 0; o < D; ++o) ge &= (q.v[o] >= p[o]);
    return ge;
}

template <int D, typename T>
__device__ __forceinline__ bool eq_all(const PackedPt<D, T> &q, const T (&p)[D]) {
    bool eq = true;
#pragma unroll
    for (int o = 0; o < D; ++o) eq &= (q.v[o] == p[o]);
    return eq;
}

template <int D, typename T>
__device__ __forceinline__ int64_t point_sum(const T *p) {
    int64_t s = 0;
#pragma unroll
    for (int o = 0; o < D; ++o) s += static_cast<int64_t>(p[o]);
    return s;
}

// Candidate start of destination `i` (local) of a job whose arc offsets are known.
__device__ __forceinline__ int64_t item_start(const int32_t *item_arc_off, const int64_t *arc_cand_off,
                                              int32_t item_base, int32_t arc_base, int32_t i) {
    return arc_cand_off[item_arc_off[item_base + i] - arc_base];
}

// First index in bases[0..n) with bases[idx] <= x < bases[idx+1] (bases ascending).
__device__ __forceinline__ int find_base(const int64_t *__restrict__ bases, int n, int64_t x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(bases + mid) <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

#define PMDD_DISPATCH_D(D_, CALL)                  \
    switch (D_) {                                  \
    case 1: { constexpr int DD = 1; return CALL; } \
    case 2: { constexpr int DD = 2; return CALL; } \
    case 3: { constexpr int DD = 3; return CALL; } \
    case 4: { constexpr int DD = 4; return CALL; } \
    case 5: { constexpr int DD = 5; return CALL; } \
    case 6: { constexpr int DD = 6; return CALL; } \
    case 7: { constexpr int DD = 7; return CALL; } \
    case 8: { constexpr int DD = 8; return CALL; } \
    default: return cudaErrorInvalidValue;         \
    }

}  // namespace dev
}  // namespace pmdd
