// sm_100a kernels for method 3 (dynamic layer cutset) and DD preparation:
//  - out-arc CSR (transpose of the in-arc CSR) for the bottom-up direction;
//  - the cutset join  F = ND( U_v { t + b : t in TD_v, b in BU_v } )  of
//    src/pmdd/enum/gpu/couple.cu:340-498 / src/pmdd/enum/cpu/enum.cpp:333-398, done in
//    rounds without ever materialising all products: a round streams products of the
//    remaining cutset nodes against the running frontier F held in shared memory (with
//    per-node and per-row ideal-point bounds that discard whole groups of products),
//    appends survivors behind F, and re-filters F + survivors.
#include "couple.cuh"

namespace pmdd {
namespace dev {

// ------------------------------------------------------------ out-arc CSR
__global__ void out_degree_kernel(const int32_t *__restrict__ arc_src, int32_t num_arcs, int32_t *__restrict__ out_off) {
    for (int32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < num_arcs; a += gridDim.x * blockDim.x)
        atomicAdd(&out_off[arc_src[a] + 1], 1);
}

// Inclusive scan of out_off[1..n] in place (one block; n is a node count).
__global__ void __launch_bounds__(1024) csr_scan_kernel(int32_t *__restrict__ off, int32_t n, int32_t *__restrict__ cursor) {
    __shared__ int32_t warp_buf[32];
    __shared__ int32_t s_carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int32_t base = 0; base < n; base += 1024) {
        const int32_t i = base + threadIdx.x;
        int32_t x = i < n ? off[i + 1] : 0;
        int32_t inc = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) warp_buf[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            const int32_t w = warp_buf[lane];
            int32_t winc = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t y = __shfl_up_sync(0xffffffffu, winc, o);
                if (lane >= o) winc += y;
            }
            warp_buf[lane] = winc - w;
        }
        __syncthreads();
        const int32_t val = s_carry + warp_buf[warp] + inc;
        if (i < n) {
            off[i + 1] = val;
            cursor[i] = val - x;  // start of node i's out-arcs
        }
        __syncthreads();
        if (threadIdx.x == 1023) s_carry = val;
        __syncthreads();
    }
}

__global__ void out_scatter_kernel(const int32_t *__restrict__ in_off, const int32_t *__restrict__ arc_src,
                                   const int32_t *__restrict__ arc_w, int32_t num_nodes, int32_t *__restrict__ cursor,
                                   int32_t *__restrict__ out_head, int32_t *__restrict__ out_w) {
    for (int32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < num_nodes; v += gridDim.x * blockDim.x) {
        for (int32_t a = in_off[v]; a < in_off[v + 1]; ++a) {
            const int32_t pos = atomicAdd(&cursor[arc_src[a]], 1);
            out_head[pos] = v;
            out_w[pos] = arc_w[a];
        }
    }
}

cudaError_t launch_build_out_csr(const int32_t *in_off, const int32_t *arc_src, const int32_t *arc_w,
                                 int32_t num_nodes, int32_t num_arcs, int32_t *out_off, int32_t *cursor,
                                 int32_t *out_head, int32_t *out_w, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(out_off, 0, sizeof(int32_t) * (static_cast<size_t>(num_nodes) + 1), stream);
    if (e != cudaSuccess) return e;
    if (num_arcs > 0) {
        const int g = std::min(1184, (num_arcs + 255) / 256);
        out_degree_kernel<<<g, 256, 0, stream>>>(arc_src, num_arcs, out_off);
    }
    csr_scan_kernel<<<1, 1024, 0, stream>>>(out_off, num_nodes, cursor);
    if (num_nodes > 0) {
        const int g = std::min(1184, (num_nodes + 255) / 256);
        out_scatter_kernel<<<g, 256, 0, stream>>>(in_off, arc_src, arc_w, num_nodes, cursor, out_head, out_w);
    }
    return cudaGetLastError();
}

// ------------------------------------------------------------------ coupling
template <int D, typename T>
__device__ __forceinline__ bool weakly_dominated_by_smem(const T (&p)[D], const T *fs, int nf, int stride) {
    for (int j = 0; j < nf; ++j) {
        bool ge = true;
#pragma unroll
        for (int o = 0; o < D; ++o) ge &= (fs[o * stride + j] >= p[o]);
        if (ge) return true;
    }
    return false;
}

// Warp-cooperative test: is `p` weakly dominated by any staged frontier point?
template <int D, typename T>
__device__ __forceinline__ bool warp_dominated(const T (&p)[D], const T *fs, int nf, int stride, int lane) {
    bool hit = false;
    for (int j = lane; j < nf && !hit; j += 32) {
        bool ge = true;
#pragma unroll
        for (int o = 0; o < D; ++o) ge &= (fs[o * stride + j] >= p[o]);
        hit = ge;
    }
    return __any_sync(0xffffffffu, hit);
}

template <int D, typename T>
__global__ void __launch_bounds__(kCoupleThreads) couple_prune_kernel(const CoupleJob *__restrict__ jobs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *fs = reinterpret_cast<T *>(smem_raw);  // [D][kCoupleFS]
    const CoupleJob &J = jobs[blockIdx.y];
    T *U = static_cast<T *>(J.U);
    const T *td = static_cast<const T *>(J.td_pts);
    const T *bu = static_cast<const T *>(J.bu_pts);
    const int64_t fn = J.ctr[kCtrF];
    const int nf = static_cast<int>(fn < kCoupleFS ? fn : kCoupleFS);
    for (int k = threadIdx.x; k < nf; k += blockDim.x)
#pragma unroll
        for (int o = 0; o < D; ++o) fs[o * kCoupleFS + k] = U[static_cast<int64_t>(k) * D + o];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    unsigned long long evaluated = 0;
    volatile const int64_t *resume_flag = J.ctr + kCtrResume;
    while (true) {
        int32_t v = 0;
        if (lane == 0) {
            // once some node overflowed U, the rest of the round is redone next round
            if (*resume_flag < J.num_nodes) v = J.num_nodes;
            else v = static_cast<int32_t>(atomicAdd(reinterpret_cast<unsigned long long *>(&J.ctr[kCtrCursor]), 1ULL));
        }
        v = __shfl_sync(0xffffffffu, v, 0);
        if (v >= J.num_nodes) break;
        const int32_t nt = J.td_size[v], nb = J.bu_size[v];
        if (nt == 0 || nb == 0) continue;
        const T *tdv = td + J.td_off[v] * D;
        const T *buv = bu + J.bu_off[v] * D;
        // ideal points of both sides
        T mt[D], mb[D];
#pragma unroll
        for (int o = 0; o < D; ++o) {
            mt[o] = tdv[o];
            mb[o] = buv[o];
        }
        for (int i = lane; i < nt; i += 32)
#pragma unroll
            for (int o = 0; o < D; ++o) mt[o] = max(mt[o], tdv[static_cast<int64_t>(i) * D + o]);
        for (int i = lane; i < nb; i += 32)
#pragma unroll
            for (int o = 0; o < D; ++o) mb[o] = max(mb[o], buv[static_cast<int64_t>(i) * D + o]);
#pragma unroll
        for (int o = 0; o < D; ++o)
            for (int s = 16; s > 0; s >>= 1) {
                mt[o] = max(mt[o], __shfl_xor_sync(0xffffffffu, mt[o], s));
                mb[o] = max(mb[o], __shfl_xor_sync(0xffffffffu, mb[o], s));
            }
        T ub[D];
#pragma unroll
        for (int o = 0; o < D; ++o) ub[o] = mt[o] + mb[o];
        if (warp_dominated<D, T>(ub, fs, nf, kCoupleFS, lane)) continue;
        bool overflowed = false;
        for (int t = 0; t < nt && !overflowed; ++t) {
            T tp[D], rub[D];
#pragma unroll
            for (int o = 0; o < D; ++o) {
                tp[o] = tdv[static_cast<int64_t>(t) * D + o];
                rub[o] = tp[o] + mb[o];
            }
            if (warp_dominated<D, T>(rub, fs, nf, kCoupleFS, lane)) continue;
            for (int b0 = 0; b0 < nb; b0 += 32) {
                const int b = b0 + lane;
                bool keep = false;
                T p[D];
                if (b < nb) {
#pragma unroll
                    for (int o = 0; o < D; ++o) p[o] = tp[o] + buv[static_cast<int64_t>(b) * D + o];
                    keep = !weakly_dominated_by_smem<D, T>(p, fs, nf, kCoupleFS);
                    ++evaluated;
                }
                const unsigned m = __ballot_sync(0xffffffffu, keep);
                if (m == 0) continue;
                unsigned long long base = 0;
                if (lane == 0)
                    base = atomicAdd(reinterpret_cast<unsigned long long *>(&J.ctr[kCtrB]),
                                     static_cast<unsigned long long>(__popc(m)));
                base = __shfl_sync(0xffffffffu, base, 0);
                const int64_t pos0 = fn + static_cast<int64_t>(base);
                if (pos0 + __popc(m) > J.ucap) {
                    // every later append lands further out, so [F, pos0) is complete
                    if (lane == 0) {
                        atomicMin(reinterpret_cast<unsigned long long *>(&J.ctr[kCtrResume]),
                                  static_cast<unsigned long long>(v));
                        atomicMin(reinterpret_cast<unsigned long long *>(&J.ctr[kCtrValidEnd]),
                                  static_cast<unsigned long long>(pos0));
                    }
                    overflowed = true;
                    break;
                }
                if (keep) {
                    const int64_t pos = pos0 + __popc(m & ((1u << lane) - 1u));
#pragma unroll
                    for (int o = 0; o < D; ++o) U[pos * D + o] = p[o];
                }
            }
        }
    }
    for (int s = 16; s > 0; s >>= 1) evaluated += __shfl_xor_sync(0xffffffffu, evaluated, s);
    if (lane == 0 && evaluated) atomicAdd(reinterpret_cast<unsigned long long *>(&J.ctr[kCtrEvaluated]), evaluated);
}

// Keep flags of F + survivors: a point is dropped iff another point is >= on every
// objective and (differs, or comes first).  Points of the old frontier (index < F)
// are mutually non-dominated, so they are only compared with the new points.
template <int D, typename T>
__global__ void __launch_bounds__(kBigThreads) couple_filter_kernel(const CoupleJob *__restrict__ jobs) {
    constexpr int JT = (kBigJTile * D * static_cast<int>(sizeof(T)) > 32768) ? 32768 / (D * static_cast<int>(sizeof(T)))
                                                                            : kBigJTile;
    __shared__ T sj[D][JT];
    const CoupleJob &J = jobs[blockIdx.y];
    const T *U = static_cast<const T *>(J.U);
    const int64_t fn = J.ctr[kCtrF];
    int64_t n = fn + J.ctr[kCtrB];
    if (n > J.ctr[kCtrValidEnd]) n = J.ctr[kCtrValidEnd];
    if (n > J.ucap) n = J.ucap;
    for (int64_t i0 = static_cast<int64_t>(blockIdx.x) * kBigThreads; i0 < n;
         i0 += static_cast<int64_t>(gridDim.x) * kBigThreads) {
        const int64_t i = i0 + threadIdx.x;
        const bool valid = i < n;
        T p[D];
        if (valid)
#pragma unroll
            for (int o = 0; o < D; ++o) p[o] = U[i * D + o];
        bool dom = !valid;
        const int64_t jstart = (i0 + kBigThreads <= fn) ? fn : 0;  // whole block in old F: compare new points only
        for (int64_t j0 = jstart; j0 < n; j0 += JT) {
            if (__syncthreads_and(dom)) break;
            const int m = static_cast<int>(n - j0 < JT ? n - j0 : static_cast<int64_t>(JT));
            for (int k = threadIdx.x; k < m; k += kBigThreads)
#pragma unroll
                for (int o = 0; o < D; ++o) sj[o][k] = U[(j0 + k) * D + o];
            __syncthreads();
            if (!dom) {
                for (int k = 0; k < m; ++k) {
                    const int64_t j = j0 + k;
                    if (j == i) continue;
                    bool ge = true, eq = true;
#pragma unroll
                    for (int o = 0; o < D; ++o) {
                        const T x = sj[o][k];
                        ge &= (x >= p[o]);
                        eq &= (x == p[o]);
                    }
                    if (ge && (!eq || j < i)) {
                        dom = true;
                        break;
                    }
                }
            }
        }
        if (valid) J.keep[i] = dom ? 0 : 1;
        __syncthreads();
    }
}

// In-place compaction of F + survivors (one block per job) and round bookkeeping.
template <int D, typename T>
__global__ void __launch_bounds__(1024) couple_compact_kernel(const CoupleJob *__restrict__ jobs) {
    __shared__ int32_t warp_buf[32];
    __shared__ int64_t s_carry;
    const CoupleJob &J = jobs[blockIdx.x];
    T *U = static_cast<T *>(J.U);
    const int64_t fn = J.ctr[kCtrF];
    int64_t n = fn + J.ctr[kCtrB];
    if (n > J.ctr[kCtrValidEnd]) n = J.ctr[kCtrValidEnd];
    if (n > J.ucap) n = J.ucap;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < n; base += 1024) {
        const int64_t i = base + threadIdx.x;
        const int32_t k = (i < n && J.keep[i]) ? 1 : 0;
        T p[D];
        if (k)
#pragma unroll
            for (int o = 0; o < D; ++o) p[o] = U[i * D + o];
        int32_t inc = k;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) warp_buf[warp] = inc;
        __syncthreads();  // also: every read of this chunk happens before any write below
        if (warp == 0) {
            const int32_t w = warp_buf[lane];
            int32_t winc = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t y = __shfl_up_sync(0xffffffffu, winc, o);
                if (lane >= o) winc += y;
            }
            warp_buf[lane] = winc - w;
        }
        __syncthreads();
        if (k) {
            const int64_t dst = s_carry + warp_buf[warp] + inc - 1;
#pragma unroll
            for (int o = 0; o < D; ++o) U[dst * D + o] = p[o];
        }
        __syncthreads();
        if (threadIdx.x == 1023) s_carry += warp_buf[31] + inc;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const int64_t resume = J.ctr[kCtrResume];
        J.ctr[kCtrF] = s_carry;
        J.ctr[kCtrB] = 0;
        J.ctr[kCtrCursor] = resume < J.num_nodes ? resume : J.num_nodes;
        J.ctr[kCtrDone] = resume >= J.num_nodes ? 1 : 0;
        J.ctr[kCtrResume] = J.num_nodes;
        J.ctr[kCtrValidEnd] = J.ucap;
    }
}

template <int D, typename T>
static cudaError_t launch_couple_round_t(const CoupleJob *jobs, int num_jobs, int blocks_per_job, cudaStream_t stream) {
    const size_t smem = static_cast<size_t>(kCoupleFS) * D * sizeof(T);
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(couple_prune_kernel<D, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    couple_prune_kernel<D, T><<<dim3(blocks_per_job, num_jobs), kCoupleThreads, smem, stream>>>(jobs);
    couple_filter_kernel<D, T><<<dim3(blocks_per_job * 2, num_jobs), kBigThreads, 0, stream>>>(jobs);
    couple_compact_kernel<D, T><<<num_jobs, 1024, 0, stream>>>(jobs);
    return cudaGetLastError();
}

__global__ void couple_products_kernel(const CoupleJob *__restrict__ jobs) {
    const CoupleJob &J = jobs[blockIdx.x];
    unsigned long long acc = 0;
    for (int32_t v = threadIdx.x; v < J.num_nodes; v += blockDim.x)
        acc += static_cast<unsigned long long>(J.td_size[v]) * static_cast<unsigned long long>(J.bu_size[v]);
    for (int s = 16; s > 0; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(reinterpret_cast<unsigned long long *>(&J.ctr[kCtrProducts]), acc);
}

cudaError_t launch_couple_products(const CoupleJob *jobs, int num_jobs, cudaStream_t stream) {
    if (num_jobs <= 0) return cudaSuccess;
    couple_products_kernel<<<num_jobs, 256, 0, stream>>>(jobs);
    return cudaGetLastError();
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

cudaError_t launch_couple_round(int d, bool wide, const CoupleJob *jobs, int num_jobs, int blocks_per_job,
                                cudaStream_t stream) {
    if (num_jobs <= 0) return cudaSuccess;
    if (wide) { PMDD_DISPATCH_D(d, (launch_couple_round_t<DD, int64_t>(jobs, num_jobs, blocks_per_job, stream))); }
    PMDD_DISPATCH_D(d, (launch_couple_round_t<DD, int32_t>(jobs, num_jobs, blocks_per_job, stream)));
}

}  // namespace dev
}  // namespace pmdd
