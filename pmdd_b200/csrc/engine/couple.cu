// sm_100a kernels for method 3 (dynamic layer cutset) and DD preparation:
//  - out-arc CSR (transpose of the in-arc CSR) for the bottom-up direction;
//  - the cutset join  F = ND( U_v { t + b : t in TD_v, b in BU_v } )  of
//    src/pmdd/enum/gpu/couple.cu:340-498 / src/pmdd/enum/cpu/enum.cpp:333-398, done in
//    rounds without ever materialising all products.  A seed round builds a first
//    running frontier from a few extreme products per cutset node; each product round
//    streams the remaining products against the running frontier F held in shared
//    memory (per-node and per-row ideal-point bounds discard whole groups of products
//    first), appends survivors behind F, and re-filters F + survivors with the
//    sort-filter-skyline block routine of sfs.cuh.
#include "couple.cuh"
#include "sfs.cuh"

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

// Appends points behind F; warp-aggregated.  Returns false (and records where the
// round must resume) when U is full.
template <int D, typename T>
__device__ __forceinline__ bool append_points(const CoupleJob &J, T *U, int64_t fn, bool keep, const T (&p)[D],
                                              int32_t v, int lane) {
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (m == 0) return true;
    unsigned long long base = 0;
    if (lane == 0)
        base = atomicAdd(reinterpret_cast<unsigned long long *>(&J.ctr[kCtrB]), static_cast<unsigned long long>(__popc(m)));
    base = __shfl_sync(0xffffffffu, base, 0);
    const int64_t pos0 = fn + static_cast<int64_t>(base);
    if (pos0 + __popc(m) > J.ucap) {
        // every later append lands further out, so [F, pos0) is complete
        if (lane == 0) {
            atomicMin(reinterpret_cast<unsigned long long *>(&J.ctr[kCtrResume]), static_cast<unsigned long long>(v));
            atomicMin(reinterpret_cast<unsigned long long *>(&J.ctr[kCtrValidEnd]),
                      static_cast<unsigned long long>(pos0));
        }
        return false;
    }
    if (keep) {
        const int64_t pos = pos0 + __popc(m & ((1u << lane) - 1u));
#pragma unroll
        for (int o = 0; o < D; ++o) U[pos * D + o] = p[o];
    }
    return true;
}

// Seed round: per cutset node, the products of the two frontiers' maximisers of each
// objective and of the objective sum (warp per node).
template <int D, typename T>
__global__ void __launch_bounds__(kCoupleThreads) couple_seed_kernel(const CoupleJob *__restrict__ jobs) {
    const CoupleJob &J = jobs[blockIdx.y];
    T *U = static_cast<T *>(J.U);
    const T *td = static_cast<const T *>(J.td_pts);
    const T *bu = static_cast<const T *>(J.bu_pts);
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (kCoupleThreads / 32);
    for (int32_t v = blockIdx.x * (kCoupleThreads / 32) + (threadIdx.x >> 5); v < J.num_nodes; v += warps) {
        const int32_t nt = J.td_size[v], nb = J.bu_size[v];
        if (nt == 0 || nb == 0) continue;
        const T *tdv = td + J.td_off[v] * D;
        const T *buv = bu + J.bu_off[v] * D;
        // argmax per objective (0..D-1) and of the sum (D), per side
        int64_t bt[D + 1], bb[D + 1];
        int32_t it[D + 1], ib[D + 1];
#pragma unroll
        for (int k = 0; k <= D; ++k) {
            bt[k] = bb[k] = INT64_MIN;
            it[k] = ib[k] = 0;
        }
        for (int32_t i = lane; i < nt; i += 32) {
            int64_t s = 0;
#pragma unroll
            for (int o = 0; o < D; ++o) {
                const int64_t x = tdv[static_cast<int64_t>(i) * D + o];
                s += x;
                if (x > bt[o]) { bt[o] = x; it[o] = i; }
            }
            if (s > bt[D]) { bt[D] = s; it[D] = i; }
        }
        for (int32_t i = lane; i < nb; i += 32) {
            int64_t s = 0;
#pragma unroll
            for (int o = 0; o < D; ++o) {
                const int64_t x = buv[static_cast<int64_t>(i) * D + o];
                s += x;
                if (x > bb[o]) { bb[o] = x; ib[o] = i; }
            }
            if (s > bb[D]) { bb[D] = s; ib[D] = i; }
        }
#pragma unroll
        for (int k = 0; k <= D; ++k) {
            for (int sft = 16; sft > 0; sft >>= 1) {
                const int64_t ot = __shfl_xor_sync(0xffffffffu, bt[k], sft);
                const int32_t oi = __shfl_xor_sync(0xffffffffu, it[k], sft);
                if (ot > bt[k] || (ot == bt[k] && oi < it[k])) { bt[k] = ot; it[k] = oi; }
                const int64_t ob = __shfl_xor_sync(0xffffffffu, bb[k], sft);
                const int32_t oj = __shfl_xor_sync(0xffffffffu, ib[k], sft);
                if (ob > bb[k] || (ob == bb[k] && oj < ib[k])) { bb[k] = ob; ib[k] = oj; }
            }
        }
        // lane k < D+1 emits product k
        T p[D];
        bool keep = false;
#pragma unroll
        for (int k = 0; k <= D; ++k) {
            if (lane == k) {
#pragma unroll
                for (int o = 0; o < D; ++o)
                    p[o] = tdv[static_cast<int64_t>(it[k]) * D + o] + buv[static_cast<int64_t>(ib[k]) * D + o];
                keep = true;
            }
        }
        if (!keep) {
#pragma unroll
            for (int o = 0; o < D; ++o) p[o] = T(0);
        }
        if (!append_points<D, T>(J, U, 0, keep, p, v, lane)) break;
    }
}

// Is a single point weakly dominated by any staged frontier point?  (lanes split F)
template <int D, typename T>
__device__ __forceinline__ bool warp_point_dominated(const PackedPt<D, T> *fs, int nf, const T (&p)[D], int lane) {
    bool hit = false;
    for (int j = lane; j < nf && !hit; j += 32) hit = ge_all<D, T>(fs[j], p);
    return __any_sync(0xffffffffu, hit);
}

template <int D, typename T>
__global__ void __launch_bounds__(kCoupleThreads) couple_prune_kernel(const CoupleJob *__restrict__ jobs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PackedPt<D, T> *fs = reinterpret_cast<PackedPt<D, T> *>(smem_raw);  // [kCoupleFS]
    const CoupleJob &J = jobs[blockIdx.y];
    T *U = static_cast<T *>(J.U);
    const T *td = static_cast<const T *>(J.td_pts);
    const T *bu = static_cast<const T *>(J.bu_pts);
    const int64_t fn = J.ctr[kCtrF];
    const int nf = static_cast<int>(fn < kCoupleFS ? fn : kCoupleFS);
    for (int k = threadIdx.x; k < nf; k += blockDim.x) {
        PackedPt<D, T> q;
#pragma unroll
        for (int o = 0; o < PackedPt<D, T>::kPad; ++o) q.v[o] = o < D ? U[static_cast<int64_t>(k) * D + o] : T(0);
        fs[k] = q;
    }
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
        if (warp_point_dominated<D, T>(fs, nf, ub, lane)) continue;
        bool overflowed = false;
        for (int t = 0; t < nt && !overflowed; ++t) {
            T tp[D], rub[D];
#pragma unroll
            for (int o = 0; o < D; ++o) {
                tp[o] = tdv[static_cast<int64_t>(t) * D + o];
                rub[o] = tp[o] + mb[o];
            }
            if (warp_point_dominated<D, T>(fs, nf, rub, lane)) continue;
            for (int b0 = 0; b0 < nb; b0 += 32) {
                const int b = b0 + lane;
                const bool valid = b < nb;
                T p[D];
#pragma unroll
                for (int o = 0; o < D; ++o) p[o] = valid ? tp[o] + buv[static_cast<int64_t>(b) * D + o] : T(0);
                bool dom = !valid;
                // warp-uniform sweep of the staged frontier
                int j = 0, it = 0;
                for (; j + 4 <= nf; j += 4) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) dom |= ge_all<D, T>(fs[j + u], p);
                    if ((++it & 7) == 0 && __all_sync(0xffffffffu, dom)) break;
                }
                if (!__all_sync(0xffffffffu, dom))
                    for (; j < nf; ++j) dom |= ge_all<D, T>(fs[j], p);
                if (valid) ++evaluated;
                if (!append_points<D, T>(J, U, fn, !dom, p, v, lane)) {
                    overflowed = true;
                    break;
                }
            }
        }
    }
    for (int s = 16; s > 0; s >>= 1) evaluated += __shfl_xor_sync(0xffffffffu, evaluated, s);
    if (lane == 0 && evaluated) atomicAdd(reinterpret_cast<unsigned long long *>(&J.ctr[kCtrEvaluated]), evaluated);
}

// F + survivors -> next running frontier in U_alt (one block per job), and the round's
// bookkeeping.
template <int D, typename T>
__global__ void __launch_bounds__(SfsCfg<D, T>::kThreads) couple_sfs_kernel(const CoupleJob *__restrict__ jobs,
                                                                            int seed) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const CoupleJob &J = jobs[blockIdx.x];
    const int64_t fn = J.ctr[kCtrF];
    int64_t n = fn + J.ctr[kCtrB];
    if (n > J.ctr[kCtrValidEnd]) n = J.ctr[kCtrValidEnd];
    if (n > J.ucap) n = J.ucap;
    SfsScratch<T> s;
    s.P2 = static_cast<T *>(J.sc_pts2);
    s.I2 = J.sc_idx;
    s.SV = static_cast<T *>(J.sc_surv);
    s.SVI = J.sc_sidx;
    const int32_t kept = sfs_block<D, T>(smem_raw, static_cast<const T *>(J.U), n, s, static_cast<T *>(J.U_alt));
    if (threadIdx.x == 0) {
        const int64_t resume = J.ctr[kCtrResume];
        J.ctr[kCtrF] = kept;
        J.ctr[kCtrB] = 0;
        if (seed) {
            J.ctr[kCtrCursor] = 0;
            J.ctr[kCtrDone] = 0;
        } else {
            J.ctr[kCtrCursor] = resume < J.num_nodes ? resume : J.num_nodes;
            J.ctr[kCtrDone] = resume >= J.num_nodes ? 1 : 0;
        }
        J.ctr[kCtrResume] = J.num_nodes;
        J.ctr[kCtrValidEnd] = J.ucap;
    }
}

template <int D, typename T>
static cudaError_t launch_couple_round_t(const CoupleJob *jobs, int num_jobs, int blocks_per_job, bool seed,
                                        cudaStream_t stream) {
    const size_t smem = static_cast<size_t>(kCoupleFS) * sizeof(PackedPt<D, T>);
    using Cfg = SfsCfg<D, T>;
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(couple_prune_kernel<D, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(couple_sfs_kernel<D, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(Cfg::kSmem));
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    if (seed) couple_seed_kernel<D, T><<<dim3(blocks_per_job, num_jobs), kCoupleThreads, 0, stream>>>(jobs);
    else couple_prune_kernel<D, T><<<dim3(blocks_per_job, num_jobs), kCoupleThreads, smem, stream>>>(jobs);
    couple_sfs_kernel<D, T><<<num_jobs, Cfg::kThreads, Cfg::kSmem, stream>>>(jobs, seed ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_couple_round(int d, bool wide, const CoupleJob *jobs, int num_jobs, int blocks_per_job, bool seed,
                                cudaStream_t stream) {
    if (num_jobs <= 0) return cudaSuccess;
    if (wide) {
        PMDD_DISPATCH_D(d, (launch_couple_round_t<DD, int64_t>(jobs, num_jobs, blocks_per_job, seed, stream)));
    }
    PMDD_DISPATCH_D(d, (launch_couple_round_t<DD, int32_t>(jobs, num_jobs, blocks_per_job, seed, stream)));
}

}  // namespace dev
}  // namespace pmdd
