// sm_100a kernels for method 3 (dynamic layer cutset) and DD preparation:
//  - out-arc CSR (transpose of the in-arc CSR) for the bottom-up direction;
//  - the cutset join  F = ND( U_v { t + b : t in TD_v, b in BU_v } )  of
//    src/pmdd/enum/gpu/couple.cu:340-498 / src/pmdd/enum/cpu/enum.cpp:333-398, done in
//    rounds without ever materialising all products.  A seed round builds a first
//    running frontier from a few extreme products per cutset node; each product round
//    streams the remaining products against the whole running frontier F (its first
//    points from shared memory, the rest from L2; per-node and per-row ideal-point bounds
//    discard whole groups of products first) and appends the survivors S behind F.  As
//    no survivor is weakly dominated by a point of F, the next running frontier is
//    {f in F : no s in S dominates f} + the maxima of S: F + S are bucketed by
//    decreasing objective sum (a dominator's sum is never smaller), one GPU-wide mark
//    pass sweeps tiles of F + S against the survivors up to the end of each point's
//    bucket, staged in shared memory, and a compaction writes the next F in bucket
//    order.  The product round uses that order: a product stops sweeping F once the
//    buckets left cannot reach its sum.
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

// Order of the running frontier: F is in decreasing sum-bucket order under (mx, width,
// nb), so every point from position j on has a sum <= top(F_j).  width 0: no order.
struct FOrder {
    int64_t mx, width, nb;
    template <int D, typename T>
    __device__ __forceinline__ int64_t top(const T *q) const {
        if (width <= 0) return INT64_MAX;
        const int64_t sm = point_sum<D, T>(q);
        if (sm > mx) return INT64_MAX;
        const int64_t b = (mx - sm) / width;
        return mx - (b < nb ? b : nb - 1) * width;
    }
};

// Is a single point weakly dominated by a point of F?  Lanes split F: the staged points
// in shared memory first, then the rest of F in global memory; the sweep ends where the
// remaining buckets cannot reach the point's sum.
template <int D, typename T>
__device__ __forceinline__ bool warp_point_dominated(const PackedPt<D, T> *fs, int nf, const T *F, int64_t fn,
                                                     const FOrder &ord, const T (&p)[D], int lane) {
    const int64_t ps = point_sum<D, T>(p);
    bool hit = false;
    for (int j = lane; j < nf && !hit; j += 32) {
        if (ord.top<D, T>(fs[j].v) < ps) break;
        hit = ge_all<D, T>(fs[j], p);
    }
    if (__any_sync(0xffffffffu, hit)) return true;
    for (int64_t j0 = nf; j0 < fn; j0 += 32) {
        if (ord.top<D, T>(F + j0 * D) < ps) break;  // warp-uniform
        const int64_t j = j0 + lane;
        if (j < fn) hit = ge_all<D, T>(load_global_pt<D, T>(F, j), p);
        if (__any_sync(0xffffffffu, hit)) return true;
    }
    return false;
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
    const FOrder ord{J.ctr[kCtrFMax], J.ctr[kCtrFWidth], J.ctr[kCtrFBuckets]};
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
        if (warp_point_dominated<D, T>(fs, nf, U, fn, ord, ub, lane)) continue;
        bool overflowed = false;
        for (int t = 0; t < nt && !overflowed; ++t) {
            T tp[D], rub[D];
#pragma unroll
            for (int o = 0; o < D; ++o) {
                tp[o] = tdv[static_cast<int64_t>(t) * D + o];
                rub[o] = tp[o] + mb[o];
            }
            if (warp_point_dominated<D, T>(fs, nf, U, fn, ord, rub, lane)) continue;
            for (int b0 = 0; b0 < nb; b0 += 32) {
                const int b = b0 + lane;
                const bool valid = b < nb;
                T p[D];
#pragma unroll
                for (int o = 0; o < D; ++o) p[o] = valid ? tp[o] + buv[static_cast<int64_t>(b) * D + o] : T(0);
                bool dom = !valid;
                // `done`: no point of F from here on can reach this product's sum
                bool done = false;
                const int64_t ps = point_sum<D, T>(p);
                // warp-uniform sweep of the staged frontier
                int j = 0, it = 0;
                for (; j + 4 <= nf; j += 4) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) dom |= ge_all<D, T>(fs[j + u], p);
                    if ((++it & 7) == 0) {
                        if (j + 4 < nf) done |= ord.top<D, T>(fs[j + 4].v) < ps;
                        if (__all_sync(0xffffffffu, dom || done)) break;
                    }
                }
                if (!__all_sync(0xffffffffu, dom || done))
                    for (; j < nf; ++j) dom |= ge_all<D, T>(fs[j], p);
                // the rest of F from global memory (warp-uniform, broadcast loads)
                if (fn > nf && !__all_sync(0xffffffffu, dom || done))
                    for (int64_t g = nf; g < fn; ++g) {
                        dom |= ge_all<D, T>(load_global_pt<D, T>(U, g), p);
                        if ((g & 31) == 31) {
                            if (g + 1 < fn) done |= ord.top<D, T>(U + (g + 1) * D) < ps;
                            if (__all_sync(0xffffffffu, dom || done)) break;
                        }
                    }
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

// Points of U at the start of a refilter: F = [0, fn) then this round's survivors S,
// clamped to what was written.
__device__ __forceinline__ void couple_extent(const CoupleJob &J, int64_t *fn, int64_t *n) {
    *fn = J.ctr[kCtrF];
    int64_t m = *fn + J.ctr[kCtrB];
    if (m > J.ctr[kCtrValidEnd]) m = J.ctr[kCtrValidEnd];
    if (m > J.ucap) m = J.ucap;
    *n = m;
}

constexpr int kMarkThreads = 256;
constexpr int kMarkStage = 2048;  // survivors staged in shared memory at a time

// Sum bucket of a point (bucket 0 holds the largest sums): -1 above the top bucket.
__device__ __forceinline__ int64_t sum_bucket(int64_t sum, int64_t mx, int64_t width, int64_t nb) {
    if (sum > mx) return -1;
    const int64_t b = (mx - sum) / width;
    return b < nb ? b : nb - 1;
}

// Largest sum a point in the same bucket as `sum` can have (INT64_MAX without an order).
__device__ __forceinline__ int64_t bucket_top(int64_t sum, int64_t mx, int64_t width, int64_t nb) {
    if (width <= 0) return INT64_MAX;
    const int64_t b = sum_bucket(sum, mx, width, nb);
    return b < 0 ? INT64_MAX : mx - b * width;
}

// Refilter step 1 (one block per job): the sum range of F + S, the bucket count and
// width, and zeroed bucket counts (all points and survivors apart).
template <int D, typename T>
__global__ void __launch_bounds__(1024) couple_bucket_prep_kernel(const CoupleJob *__restrict__ jobs) {
    __shared__ int64_t red_min[32], red_max[32];
    const CoupleJob &J = jobs[blockIdx.x];
    const T *U = static_cast<const T *>(J.U);
    int64_t fn, n;
    couple_extent(J, &fn, &n);
    int64_t mn = INT64_MAX, mx = INT64_MIN;
    for (int64_t i = threadIdx.x; i < n; i += 1024) {
        const int64_t sm = point_sum<D, T>(U + i * D);
        mn = min(mn, sm);
        mx = max(mx, sm);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = min(mn, static_cast<int64_t>(__shfl_xor_sync(0xffffffffu, mn, o)));
        mx = max(mx, static_cast<int64_t>(__shfl_xor_sync(0xffffffffu, mx, o)));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        red_min[warp] = mn;
        red_max[warp] = mx;
    }
    __syncthreads();
    int64_t nb = n / 64;
    nb = nb < 1 ? 1 : (nb > kMaxBuckets ? kMaxBuckets : nb);
    if (threadIdx.x == 0) {
        for (int w = 1; w < 32; ++w) {
            mn = min(mn, red_min[w]);
            mx = max(mx, red_max[w]);
        }
        if (n <= 0) {
            mn = 0;
            mx = 0;
        }
        J.ctr[kCtrSumMax] = mx;
        J.ctr[kCtrWidth] = (mx - mn) / nb + 1;
        J.ctr[kCtrBuckets] = nb;
    }
    for (int64_t b = threadIdx.x; b <= nb; b += 1024) {
        J.sc_hist[b] = 0;
        J.sc_hist[kMaxBuckets + 1 + b] = 0;
    }
}

// Refilter step 2 (grid): points per bucket, all of F + S and survivors alone.
template <int D, typename T>
__global__ void __launch_bounds__(kMarkThreads) couple_bucket_count_kernel(const CoupleJob *__restrict__ jobs) {
    const CoupleJob &J = jobs[blockIdx.y];
    const T *U = static_cast<const T *>(J.U);
    int64_t fn, n;
    couple_extent(J, &fn, &n);
    const int64_t mx = J.ctr[kCtrSumMax], width = J.ctr[kCtrWidth], nb = J.ctr[kCtrBuckets];
    int32_t *hc = J.sc_hist, *hs = J.sc_hist + kMaxBuckets + 1;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kMarkThreads + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * kMarkThreads) {
        const int64_t b = max(static_cast<int64_t>(0), sum_bucket(point_sum<D, T>(U + i * D), mx, width, nb));
        atomicAdd(&hc[b], 1);
        if (i >= fn) atomicAdd(&hs[b], 1);
    }
}

// Refilter step 3 (one block per job): bucket counts -> bucket starts, both arrays.
__global__ void __launch_bounds__(1024) couple_bucket_scan_kernel(const CoupleJob *__restrict__ jobs) {
    __shared__ int32_t warp_buf[32];
    __shared__ int32_t total;
    const CoupleJob &J = jobs[blockIdx.x];
    const int64_t nb = J.ctr[kCtrBuckets];
    const int64_t chunk = (nb + 1023) / 1024;
    const int64_t b0 = threadIdx.x * chunk, b1 = min(nb, b0 + chunk);
    for (int h = 0; h < 2; ++h) {
        int32_t *a = J.sc_hist + h * (kMaxBuckets + 1);
        int32_t sum = 0;
        for (int64_t b = b0; b < b1; ++b) sum += a[b];
        int32_t run = block_exclusive_scan<int32_t, 1024>(sum, warp_buf, &total);
        for (int64_t b = b0; b < b1; ++b) {
            const int32_t c = a[b];
            a[b] = run;
            run += c;
        }
    }
}

// Refilter step 4 (grid): F + S into sc_pts2 in bucket order with a byte per point saying
// whether it is a survivor, and the survivors alone into sc_surv in bucket order with their
// sc_pts2 positions (order inside a bucket arbitrary).  Afterwards the histograms hold
// the bucket ends.
template <int D, typename T>
__global__ void __launch_bounds__(kMarkThreads) couple_bucket_scatter_kernel(const CoupleJob *__restrict__ jobs) {
    const CoupleJob &J = jobs[blockIdx.y];
    const T *U = static_cast<const T *>(J.U);
    T *C = static_cast<T *>(J.sc_pts2);
    T *Sp = static_cast<T *>(J.sc_surv);
    int64_t fn, n;
    couple_extent(J, &fn, &n);
    const int64_t mx = J.ctr[kCtrSumMax], width = J.ctr[kCtrWidth], nb = J.ctr[kCtrBuckets];
    int32_t *hc = J.sc_hist, *hs = J.sc_hist + kMaxBuckets + 1;
    uint8_t *origin = reinterpret_cast<uint8_t *>(J.sc_idx) + J.ucap;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kMarkThreads + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * kMarkThreads) {
        const int64_t b = max(static_cast<int64_t>(0), sum_bucket(point_sum<D, T>(U + i * D), mx, width, nb));
        const int64_t pos = atomicAdd(&hc[b], 1);
#pragma unroll
        for (int o = 0; o < D; ++o) C[pos * D + o] = U[i * D + o];
        origin[pos] = i >= fn ? 1 : 0;
        if (i >= fn) {
            const int64_t sp = atomicAdd(&hs[b], 1);
#pragma unroll
            for (int o = 0; o < D; ++o) Sp[sp * D + o] = U[i * D + o];
            J.sc_sidx[sp] = static_cast<int32_t>(pos);
        }
    }
}

// Refilter step 5: a keep byte for every point of F + S (in bucket order, sc_idx).  A
// point of F is dropped when a survivor is >= on every objective (no survivor equals a
// point of F: the product round drops products weakly dominated by F); a survivor is
// dropped when another survivor is >= and differs, or equals it and comes first.  A
// dominator's sum is never smaller, so it sits in the point's bucket or an earlier one:
// each point sweeps the survivors up to the end of its own bucket.  Tiles of 256 points,
// persistent over gridDim.x blocks per job; a tile stops once all its points are dropped.
template <int D, typename T>
__global__ void __launch_bounds__(kMarkThreads) couple_mark_kernel(const CoupleJob *__restrict__ jobs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PackedPt<D, T> *sp = reinterpret_cast<PackedPt<D, T> *>(smem_raw);                   // [kMarkStage]
    int32_t *spos = reinterpret_cast<int32_t *>(smem_raw + sizeof(PackedPt<D, T>) * kMarkStage);  // [kMarkStage]
    __shared__ int32_t tile_end;
    const CoupleJob &J = jobs[blockIdx.y];
    const T *C = static_cast<const T *>(J.sc_pts2);
    const T *Sp = static_cast<const T *>(J.sc_surv);
    int64_t fn, n;
    couple_extent(J, &fn, &n);
    const int64_t mx = J.ctr[kCtrSumMax], width = J.ctr[kCtrWidth], nb = J.ctr[kCtrBuckets];
    const int32_t *ends = J.sc_hist + kMaxBuckets + 1;  // survivor bucket ends
    uint8_t *keep = reinterpret_cast<uint8_t *>(J.sc_idx);
    const uint8_t *origin = keep + J.ucap;
    for (int64_t t0 = static_cast<int64_t>(blockIdx.x) * kMarkThreads; t0 < n;
         t0 += static_cast<int64_t>(gridDim.x) * kMarkThreads) {
        const int64_t i = t0 + threadIdx.x;
        const bool valid = i < n;
        const bool in_s = valid && origin[i] != 0;
        T p[D];
#pragma unroll
        for (int o = 0; o < D; ++o) p[o] = valid ? C[i * D + o] : T(0);
        int32_t my_end = 0;
        if (valid && n > fn) my_end = ends[max(static_cast<int64_t>(0), sum_bucket(point_sum<D, T>(p), mx, width, nb))];
        if (threadIdx.x == 0) tile_end = 0;
        __syncthreads();
        atomicMax(&tile_end, my_end);
        bool dom = !valid;
        __syncthreads();
        const int64_t limit = tile_end;
        for (int64_t c0 = 0; c0 < limit; c0 += kMarkStage) {
            if (__syncthreads_and(dom || c0 >= my_end)) break;
            const int cn = static_cast<int>(limit - c0 < kMarkStage ? limit - c0 : static_cast<int64_t>(kMarkStage));
            for (int k = threadIdx.x; k < cn; k += kMarkThreads) {
                sp[k] = load_global_pt<D, T>(Sp, c0 + k);
                spos[k] = J.sc_sidx[c0 + k];
            }
            __syncthreads();
            if (!dom) {
                const int64_t rem = my_end - c0;
                const int kn = static_cast<int>(rem < cn ? (rem > 0 ? rem : 0) : cn);
                for (int k = 0; k < kn; ++k) {
                    if (!ge_all<D, T>(sp[k], p)) continue;
                    if (!in_s || (spos[k] != i && (!eq_all<D, T>(sp[k], p) || spos[k] < i))) {
                        dom = true;
                        break;
                    }
                }
            }
        }
        __syncthreads();  // the stage and tile_end are rewritten by the next tile
        if (valid) keep[i] = dom ? 0 : 1;
    }
}

// Refilter step 6: compacts the kept points into U_alt in bucket order -- the next
// running frontier, ordered by decreasing sum bucket under the parameters it records --
// and does the round's bookkeeping.  One block per job.
template <int D, typename T>
__global__ void __launch_bounds__(1024) couple_compact_kernel(const CoupleJob *__restrict__ jobs, int seed) {
    __shared__ int64_t warp_buf[32];
    __shared__ int64_t total;
    const CoupleJob &J = jobs[blockIdx.x];
    const T *C = static_cast<const T *>(J.sc_pts2);
    T *out = static_cast<T *>(J.U_alt);
    int64_t fn, n;
    couple_extent(J, &fn, &n);
    const uint8_t *keep = reinterpret_cast<const uint8_t *>(J.sc_idx);
    constexpr int ITEMS = 8;
    int64_t base = 0;
    for (int64_t c0 = 0; c0 < n; c0 += 1024 * ITEMS) {
        const int64_t b = c0 + static_cast<int64_t>(threadIdx.x) * ITEMS;
        int64_t mine = 0;
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) mine += (b + k < n && keep[b + k]) ? 1 : 0;
        int64_t pos = base + block_exclusive_scan<int64_t, 1024>(mine, warp_buf, &total);
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
            if (b + k < n && keep[b + k]) {
#pragma unroll
                for (int o = 0; o < D; ++o) out[pos * D + o] = C[(b + k) * D + o];
                ++pos;
            }
        }
        base += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const int64_t resume = J.ctr[kCtrResume];
        J.ctr[kCtrF] = base;
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
        J.ctr[kCtrFMax] = J.ctr[kCtrSumMax];
        J.ctr[kCtrFWidth] = J.ctr[kCtrWidth];
        J.ctr[kCtrFBuckets] = J.ctr[kCtrBuckets];
    }
}

template <int D, typename T>
static cudaError_t launch_couple_round_t(const CoupleJob *jobs, int num_jobs, int blocks_per_job, bool seed,
                                        cudaStream_t stream) {
    const size_t smem = static_cast<size_t>(kCoupleFS) * sizeof(PackedPt<D, T>);
    const size_t mark_smem = static_cast<size_t>(kMarkStage) * (sizeof(PackedPt<D, T>) + sizeof(int32_t));
    {
        cudaError_t e = ensure_smem_limit(reinterpret_cast<const void *>(couple_prune_kernel<D, T>), smem);
        if (e != cudaSuccess) return e;
        e = ensure_smem_limit(reinterpret_cast<const void *>(couple_mark_kernel<D, T>), mark_smem);
        if (e != cudaSuccess) return e;
    }
    if (seed) couple_seed_kernel<D, T><<<dim3(blocks_per_job, num_jobs), kCoupleThreads, 0, stream>>>(jobs);
    else couple_prune_kernel<D, T><<<dim3(blocks_per_job, num_jobs), kCoupleThreads, smem, stream>>>(jobs);
    const dim3 grid(blocks_per_job, num_jobs);
    couple_bucket_prep_kernel<D, T><<<num_jobs, 1024, 0, stream>>>(jobs);
    couple_bucket_count_kernel<D, T><<<grid, kMarkThreads, 0, stream>>>(jobs);
    couple_bucket_scan_kernel<<<num_jobs, 1024, 0, stream>>>(jobs);
    couple_bucket_scatter_kernel<D, T><<<grid, kMarkThreads, 0, stream>>>(jobs);
    couple_mark_kernel<D, T><<<grid, kMarkThreads, mark_smem, stream>>>(jobs);
    couple_compact_kernel<D, T><<<num_jobs, 1024, 0, stream>>>(jobs, seed ? 1 : 0);
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
