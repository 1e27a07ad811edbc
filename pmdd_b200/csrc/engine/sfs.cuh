// Block-wide maxima of one point set by a bucketed sort-filter-skyline sweep
// (presorting by a monotone score, after Chomicki, Godfrey, Gryz and Liang, "Skyline
// with presorting", ICDE 2003).  Points are grouped into buckets of decreasing
// objective sum; a dominator of p has a sum >= p's, so it lies in p's bucket or an
// earlier one.  For each bucket, in order:
//   a. every point is checked against K, the maxima of earlier buckets;
//   b. the bucket's survivors are checked against each other (of equal points the
//      one with the smallest input index is kept);
//   c. the bucket's maxima are appended to K, which is the output.
// Comparisons are warp-uniform sweeps: a warp holds 32 points and reads the
// comparison set once, broadcast to every lane.
//
// Used for oversized destinations (big.cu) and for standalone point sets (pareto.cu).
#pragma once

#include <climits>

#include "scan.cuh"

namespace pmdd {
namespace dev {

template <int D, typename T, int kThreads_, int kMaxBuckets_, int kKeepBytes, int kSurvBytes>
struct SfsCfgT {
    static constexpr int kThreads = kThreads_;
    static constexpr int kBucket = 512;        // target points per sum bucket
    static constexpr int kMaxBuckets = kMaxBuckets_;
    static constexpr int kKeepCache = kKeepBytes / static_cast<int>(sizeof(PackedPt<D, T>));
    static constexpr int kSurvCache = kSurvBytes / static_cast<int>(sizeof(PackedPt<D, T>));
    static constexpr size_t kSmem = sizeof(int32_t) * kMaxBuckets + sizeof(PackedPt<D, T>) * kKeepCache +
                                    (sizeof(PackedPt<D, T>) + sizeof(int32_t) + 1) * kSurvCache + 256;
    static_assert(kMaxBuckets % kThreads == 0, "bucket scan layout");
};

// One large block per point set (standalone filter, cutset join): 139 KB of shared
// memory at d=3, so maxima caches hold 4096 points.
template <int D, typename T>
using SfsCfg = SfsCfgT<D, T, 512, 8192, 65536, 32768>;

// Oversized destinations, many side by side: 256 threads and ~60 KB of shared memory at
// d=3, so three blocks share an SM.
template <int D, typename T>
using SfsSmallCfg = SfsCfgT<D, T, 256, 2048, 32768, 16384>;

// Scratch of a point set of n points: P2 and SV hold n points each, I2 and SVI n ints.
template <typename T>
struct SfsScratch {
    T *P2;
    int32_t *I2;
    T *SV;
    int32_t *SVI;
};

template <int D, typename T>
__device__ __forceinline__ PackedPt<D, T> load_global_pt(const T *base, int64_t j) {
    PackedPt<D, T> q;
#pragma unroll
    for (int o = 0; o < PackedPt<D, T>::kPad; ++o) q.v[o] = o < D ? base[j * D + o] : T(0);
    return q;
}

// Maxima of P[0..n) (D values per point) into out[0..k); returns k (all threads).
// Must be called by every thread of a block of Cfg::kThreads threads with Cfg::kSmem
// bytes of dynamic shared memory at smem_raw; n < 2^31.
template <int D, typename T, class Cfg = SfsCfg<D, T>>
__device__ int32_t sfs_block(unsigned char *smem_raw, const T *__restrict__ P, int64_t n, SfsScratch<T> s,
                             T *__restrict__ out) {
    using Pt = PackedPt<D, T>;
    constexpr int NT = Cfg::kThreads, NW = NT / 32, KS = Cfg::kKeepCache, SC = Cfg::kSurvCache;
    Pt *kc = reinterpret_cast<Pt *>(smem_raw);                  // [KS]
    Pt *sc = kc + KS;                                           // [SC]
    int32_t *hist = reinterpret_cast<int32_t *>(sc + SC);       // [kMaxBuckets]
    int32_t *sidx = hist + Cfg::kMaxBuckets;                    // [SC]
    uint8_t *sflag = reinterpret_cast<uint8_t *>(sidx + SC);    // [SC]
    __shared__ int64_t red_min[NW], red_max[NW];
    __shared__ int32_t warp_i[32];
    __shared__ int32_t tot_i;
    __shared__ int64_t s_min, s_max;
    __shared__ int32_t s_kn, s_m;
    T *P2 = s.P2, *SV = s.SV;
    int32_t *I2 = s.I2, *SVI = s.SVI;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // 1. range of point sums
    int64_t mn = INT64_MAX, mx = INT64_MIN;
    for (int64_t i = tid; i < n; i += NT) {
        const int64_t sm = point_sum<D, T>(P + i * D);
        mn = min(mn, sm);
        mx = max(mx, sm);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (lane == 0) {
        red_min[warp] = mn;
        red_max[warp] = mx;
    }
    __syncthreads();
    if (tid == 0) {
        int64_t a = red_min[0], b = red_max[0];
        for (int w = 1; w < NW; ++w) {
            a = min(a, red_min[w]);
            b = max(b, red_max[w]);
        }
        s_min = a;
        s_max = b;
        s_kn = 0;
    }
    __syncthreads();
    if (n == 0) return 0;
    // 2. counting sort into buckets of decreasing sum (bucket 0 = largest sums)
    const int64_t nb64 = n / Cfg::kBucket < 1 ? 1 : n / Cfg::kBucket;
    const int nb = static_cast<int>(nb64 < Cfg::kMaxBuckets ? nb64 : static_cast<int64_t>(Cfg::kMaxBuckets));
    const int64_t width = (s_max - s_min) / nb + 1;
    for (int b = tid; b < nb; b += NT) hist[b] = 0;
    __syncthreads();
    for (int64_t i = tid; i < n; i += NT) {
        const int b = static_cast<int>((s_max - point_sum<D, T>(P + i * D)) / width);
        atomicAdd(&hist[b], 1);
    }
    __syncthreads();
    {
        constexpr int PER = Cfg::kMaxBuckets / NT;
        int32_t loc[PER];
        int32_t run = 0;
#pragma unroll
        for (int r = 0; r < PER; ++r) {
            const int b = tid * PER + r;
            loc[r] = b < nb ? hist[b] : 0;
            run += loc[r];
        }
        int32_t ex = block_exclusive_scan<int32_t, NT>(run, warp_i, &tot_i);
#pragma unroll
        for (int r = 0; r < PER; ++r) {
            const int b = tid * PER + r;
            if (b < nb) hist[b] = ex;
            ex += loc[r];
        }
    }
    __syncthreads();
    for (int64_t i = tid; i < n; i += NT) {
        const T *p = P + i * D;
        const int b = static_cast<int>((s_max - point_sum<D, T>(p)) / width);
        const int pos = atomicAdd(&hist[b], 1);
#pragma unroll
        for (int o = 0; o < D; ++o) P2[static_cast<int64_t>(pos) * D + o] = p[o];
        I2[pos] = static_cast<int32_t>(i);
    }
    __syncthreads();  // hist[b] is now the end of bucket b

    // 3. sweep the buckets
    for (int b = 0; b < nb; ++b) {
        const int32_t lo = b == 0 ? 0 : hist[b - 1], hi = hist[b];
        if (lo == hi) continue;
        if (tid == 0) s_m = 0;
        __syncthreads();
        const int32_t kn = s_kn;
        // 3a. against K, the maxima of earlier buckets
        for (int32_t c0 = lo + warp * 32; c0 < hi; c0 += NW * 32) {
            const int32_t i = c0 + lane;
            const bool valid = i < hi;
            T p[D];
            int32_t pidx = 0;
            if (valid) {
#pragma unroll
                for (int o = 0; o < D; ++o) p[o] = P2[static_cast<int64_t>(i) * D + o];
                pidx = I2[i];
            } else {
#pragma unroll
                for (int o = 0; o < D; ++o) p[o] = T(0);
            }
            bool dom = !valid;
            {
                const int32_t kn_s = kn < KS ? kn : KS;
                int32_t j = 0;
                int it = 0;
                for (; j + 4 <= kn_s; j += 4) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) dom |= ge_all<D, T>(kc[j + u], p);
                    if ((++it & 7) == 0 && __all_sync(0xffffffffu, dom)) break;
                }
                if (!__all_sync(0xffffffffu, dom)) {
                    for (; j < kn_s; ++j) dom |= ge_all<D, T>(kc[j], p);
                    for (j = KS; j < kn; ++j) {
                        dom |= ge_all<D, T>(load_global_pt<D, T>(out, j), p);
                        if ((j & 31) == 31 && __all_sync(0xffffffffu, dom)) break;
                    }
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, !dom);
            int32_t base = 0;
            if (lane == 0 && m) base = atomicAdd(&s_m, __popc(m));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (!dom) {
                const int32_t k = base + __popc(m & ((1u << lane) - 1u));
                if (k < SC) {
                    Pt sp;
#pragma unroll
                    for (int o = 0; o < Pt::kPad; ++o) sp.v[o] = o < D ? p[o] : T(0);
                    sc[k] = sp;
                    sidx[k] = pidx;
                } else {
#pragma unroll
                    for (int o = 0; o < D; ++o) SV[static_cast<int64_t>(k) * D + o] = p[o];
                    SVI[k] = pidx;
                }
            }
        }
        __syncthreads();
        const int32_t m = s_m;
        // 3b. survivors of this bucket against each other (first duplicate kept)
        for (int32_t c0 = warp * 32; c0 < m; c0 += NW * 32) {
            const int32_t k = c0 + lane;
            const bool valid = k < m;
            T p[D];
            int32_t pidx = 0;
            if (valid) {
                const Pt me = k < SC ? sc[k] : load_global_pt<D, T>(SV, k);
#pragma unroll
                for (int o = 0; o < D; ++o) p[o] = me.v[o];
                pidx = k < SC ? sidx[k] : SVI[k];
            } else {
#pragma unroll
                for (int o = 0; o < D; ++o) p[o] = T(0);
            }
            bool dom = !valid;
            for (int32_t j = 0; j < m; ++j) {
                const Pt q = j < SC ? sc[j] : load_global_pt<D, T>(SV, j);
                if (!dom && j != k && ge_all<D, T>(q, p)) {
                    const int32_t qidx = j < SC ? sidx[j] : SVI[j];
                    if (!eq_all<D, T>(q, p) || qidx < pidx) dom = true;
                }
                if ((j & 31) == 31 && __all_sync(0xffffffffu, dom)) break;
            }
            if (valid) {
                if (k < SC) sflag[k] = dom ? 0 : 1;
                else I2[lo + k] = dom ? 0 : 1;  // bucket entries [lo, hi) were consumed in 3a
            }
        }
        __syncthreads();
        // 3c. append the bucket's maxima to K (the output) and the K cache
        for (int32_t c0 = warp * 32; c0 < m; c0 += NW * 32) {
            const int32_t k = c0 + lane;
            const bool keep = k < m && (k < SC ? sflag[k] != 0 : I2[lo + k] != 0);
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            int32_t base = 0;
            if (lane == 0 && bal) base = atomicAdd(&s_kn, __popc(bal));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (keep) {
                const int32_t dst = base + __popc(bal & ((1u << lane) - 1u));
                const Pt x = k < SC ? sc[k] : load_global_pt<D, T>(SV, k);
#pragma unroll
                for (int o = 0; o < D; ++o) out[static_cast<int64_t>(dst) * D + o] = x.v[o];
                if (dst < KS) kc[dst] = x;
            }
        }
        __syncthreads();
    }
    return s_kn;
}

}  // namespace dev
}  // namespace pmdd
