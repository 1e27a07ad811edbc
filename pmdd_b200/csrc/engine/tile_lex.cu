// Fused expand + dominance filter for three objectives, in lexicographic order.
//
// Every node's frontier is kept in descending lexicographic order (objective 0, then 1,
// then 2).  Adding an arc's weight vector to every point of a frontier keeps that order,
// so the candidates of one arc ("a run") arrive sorted, and a destination's candidates
// are a few sorted runs.  In that order a point can only be dominated by a point before
// it, and since every point before q has objective 0 >= q's, q is dominated (or a later
// copy of an equal point) iff some earlier point has objectives 1 and 2 both >= q's: a
// two-dimensional "staircase" question.  The staircase of a destination's first points
// -- the two-dimensional maxima of (objective 1, objective 2) among them -- stays small
// (a few to a few dozen entries on the workloads measured), so one warp can answer it
// for a whole destination in one ordered pass.
//
//   stage:   as the pairwise tile kernel (tile.cu): destinations and their arcs, with
//            each arc's parent flag "frontier sorted";
//   expand:  candidate = parent point + arc weight, in run order;
//   merge:   each candidate's position in its destination's lexicographic order is its
//            index in its run plus, per other run, a binary search for how many of that
//            run's points come before it (equal points: the lower run first); a
//            destination with a run from an unsorted parent counts the points before it
//            instead;
//   filter:  destinations of at most J.pair_max candidates: each candidate is checked
//            against the points before it in the merged order; larger destinations:
//            one warp walks the merged order 32 candidates at a time -- each candidate
//            is looked up in the staircase so far (a binary search over objective 1),
//            the chunk's survivors are checked against each other with warp ballots and
//            shuffles, and the staircase is rebuilt from its survivors and the chunk's
//            new two-dimensional maxima;
//   write:   survivors go to the destination's slot in merged order, so the next
//            layer's runs are sorted again (out_sorted = 1).
//
// The keep rule is the reference GPU filter's (src/pmdd/enum/gpu/dominance_utils.cuh:
// 10-23): q is dropped iff another candidate p of the destination has p >= q on every
// objective and (p != q or p comes first).  Of equal points the first in the merged order
// stays; which copy stays does not change the frontier.  Oversized destinations are
// left to big.cu, whose output is not in this order (out_sorted = 0): their children
// merge by counting.
#include "bulk.cuh"
#include "kernels.cuh"
#include "scan.cuh"
#include "stair.cuh"

#include <algorithm>

namespace pmdd {
namespace dev {

namespace {

constexpr int kLT = kTileThreads;
constexpr int kLexWarps = kLT / 32;
constexpr int kStairCap = 64;      // staircase entries a warp keeps; beyond it: pairwise
// Destinations walked by staircase warps are split into segments of at most kLexSeg
// candidates, one warp each; a segment's staircase never outgrows kStairCap.
constexpr int kLexSeg = 64;
constexpr int kLexSlots = kTileCap / kLexSeg;  // staircases kept for the segments after them
constexpr unsigned kFull = 0xffffffffu;
constexpr int kWaitIters = 1 << 22;  // bulk-copy barrier: try_wait rounds before giving up

template <int D, typename T>
struct LexSmem {
    PackedPt<D, T> pts[kTileCap];        // candidates in run order; staircases after the merge
    PackedPt<D, T> mpts[kTileCap];       // candidates in merged (descending) order
    int16_t tag[kTileCap];               // staged arc of each run-order candidate
    uint16_t item_of[kTileCap];          // staged destination of each candidate (either order)
    uint8_t keep[kTileCap];              // by merged position
    int16_t keep_ex[kTileCap + 1];       // exclusive scan of keep
    int16_t item_s[kTileItemCap + 1];    // staged destination -> first candidate position
    int16_t item_arc0[kTileItemCap + 1]; // staged destination -> first staged arc
    int32_t item_a0g[kTileItemCap];      // staged destination -> first arc (global id)
    int64_t item_c0[kTileItemCap];       // staged destination -> job-local candidate start
    uint8_t item_count[kTileItemCap];    // 1: merge by counting
    int32_t big[kTileItemCap + kLexSlots];  // staircase segments: destination | segment << 16
    int8_t item_slot0[kTileItemCap];     // segmented destination -> slot of its first segment
    int16_t slot_m[kLexSlots];           // entries of each kept staircase (-1: not kept)
    int16_t arc_pos[kTileArcCap + 1];    // staged arc -> first candidate position
    int16_t arc_item[kTileArcCap];       // staged arc -> staged destination
    int32_t arc_w[kTileArcCap];          // staged arc -> weight row
    int64_t arc_src[kTileArcCap];        // staged arc -> parent slot start (points)
    int32_t arc_stage[kTileArcCap];      // bulk staging: byte offset of the run's first point (in mpts)
    uint64_t bar;                        // bulk staging barrier
    int32_t warp_i[32];
    int32_t tot_i, tot_a, i0, i1, job;
    int32_t n_big, next_big, next_chunk, tot_stage, n_slot;
    int64_t tile;                        // tile taken from the launch's queue
};

// Phase clock (J.phase_clk, a diagnostic): thread 0 adds the cycles its block spent in
// each phase of a pass (stage destinations, stage arcs, arc assignment, expand, merge,
// filter, scan and write) to the job's counters.
struct PhaseClock {
    unsigned long long *out;
    long long t;
    __device__ __forceinline__ void start() {
        if (out) t = clock64();
    }
    __device__ __forceinline__ void lap(int phase) {
        if (out) {
            const long long now = clock64();
            atomicAdd(out + phase, static_cast<unsigned long long>(now - t));
            t = now;
        }
    }
};

// Per-warp staircase storage, laid over pts once the merge has read it, followed by the
// final staircases of the segments that later segments are checked against.
template <typename T>
using Stair = StairBuf<T, kStairCap>;
template <typename T>
struct SegStair {
    T v1[kStairCap];  // objective 1, descending
    T v2[kStairCap];  // objective 2, ascending
};

// Segments of a destination of c candidates walked by staircase warps (c > pair_max).
__device__ __forceinline__ int lex_segments(int c) { return (c + kLexSeg - 1) / kLexSeg; }

// Largest x over the threads before this one (-1 for thread 0); every thread calls it.
template <int THREADS>
__device__ __forceinline__ int32_t block_exclusive_max(int32_t x, int32_t *warp_buf) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc = max(inc, y);
    }
    int32_t exc = __shfl_up_sync(kFull, inc, 1);
    if (lane == 0) exc = -1;
    if (lane == 31) warp_buf[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int32_t w = lane < THREADS / 32 ? warp_buf[lane] : -1;
        int32_t winc = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(kFull, winc, o);
            if (lane >= o) winc = max(winc, y);
        }
        int32_t wexc = __shfl_up_sync(kFull, winc, 1);
        if (lane == 0) wexc = -1;
        if (lane < THREADS / 32) warp_buf[lane] = wexc;
    }
    __syncthreads();
    const int32_t r = max(exc, warp_buf[warp]);
    __syncthreads();  // warp_buf may be reused right after
    return r;
}

template <typename T>
__device__ __forceinline__ bool lex_gt(const PackedPt<3, T> &a, const PackedPt<3, T> &b) {
    if (a.v[0] != b.v[0]) return a.v[0] > b.v[0];
    if (a.v[1] != b.v[1]) return a.v[1] > b.v[1];
    return a.v[2] > b.v[2];
}

template <typename T>
__device__ __forceinline__ bool lex_eq(const PackedPt<3, T> &a, const PackedPt<3, T> &b) {
    return a.v[0] == b.v[0] && a.v[1] == b.v[1] && a.v[2] == b.v[2];
}

// The frontier order: three objectives, descending lexicographic; four (int32 points),
// descending objective sum, ties descending lexicographic.  Both keep a shifted run in
// order, and in both a point that dominates another comes before it.
template <int D, typename T>
__device__ __forceinline__ bool ord_gt(const PackedPt<D, T> &a, const PackedPt<D, T> &b) {
    if constexpr (D == 3) {
        return lex_gt(a, b);
    } else {
        int64_t sa = 0, sb = 0;
#pragma unroll
        for (int o = 0; o < D; ++o) {
            sa += a.v[o];
            sb += b.v[o];
        }
        if (sa != sb) return sa > sb;
#pragma unroll
        for (int o = 0; o < D; ++o)
            if (a.v[o] != b.v[o]) return a.v[o] > b.v[o];
        return false;
    }
}

template <int D, typename T>
__device__ __forceinline__ bool ord_eq(const PackedPt<D, T> &a, const PackedPt<D, T> &b) {
    bool e = true;
#pragma unroll
    for (int o = 0; o < D; ++o) e &= a.v[o] == b.v[o];
    return e;
}

// Candidates at merged positions [s, e) (one segment of a destination) walked by one
// warp from an empty staircase; with `save` the final staircase is kept there (its entry
// count in *save_m, -1 if it outgrew kStairCap).
template <typename T>
__device__ void stair_filter(LexSmem<3, T> &S, Stair<T> &sb, int s, int e, int lane, SegStair<T> *save,
                             int16_t *save_m) {
    StairState st;
    for (int c0 = s; c0 < e; c0 += 32) {
        const int p = c0 + lane;
        const bool valid = p < e;
        T q1 = 0, q2 = 0;
        if (valid) {
            q1 = S.mpts[p].v[1];
            q2 = S.mpts[p].v[2];
        }
        bool dom = !valid;
        if (st.overflow) {
            // staircase given up: every point before p, chunk-mates included
            const int hi = min(e, c0 + 32) - 1;
            for (int j = s; j < hi; ++j) {
                const PackedPt<3, T> c = S.mpts[j];
                if (j < p) dom |= (c.v[1] >= q1) & (c.v[2] >= q2);
                if (((j - s) & 15) == 15 && __all_sync(kFull, dom)) break;
            }
        } else {
            dom = stair_chunk<T, kStairCap>(sb, st, valid, q1, q2, save != nullptr || c0 + 32 < e);
        }
        if (valid) S.keep[p] = dom ? 0 : 1;
    }
    if (save != nullptr) {
        for (int i = lane; i < st.m && !st.overflow; i += 32) {
            save->v1[i] = sb.v1[st.cur][i];
            save->v2[i] = sb.v2[st.cur][i];
        }
        if (lane == 0) *save_m = st.overflow ? -1 : static_cast<int16_t>(st.m);
    }
}

}  // namespace

template <int D, typename T>
__global__ void __launch_bounds__(kLT) expand_tile_lex_kernel(const ExpandJob *__restrict__ jobs,
                                                              const int64_t *__restrict__ tile_bases, int num_jobs,
                                                              int64_t total_tiles, unsigned long long *queue,
                                                              const int64_t *tiles_dev) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    LexSmem<D, T> &S = *reinterpret_cast<LexSmem<D, T> *>(smem_raw);
    Stair<T> *stairs = reinterpret_cast<Stair<T> *>(&S.pts[0]);
    SegStair<T> *slots = reinterpret_cast<SegStair<T> *>(stairs + kLexWarps);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned bar_phase = 0;
    bool aborted = false;
    if (tid == 0) mbar_init(&S.bar, 1);
    __syncthreads();
    // tiles are handed out by an atomic counter over all the launch's jobs, so a block
    // that drew cheap tiles takes more
    auto next_tile = [&]() -> int64_t {
        if (tid == 0) S.tile = static_cast<int64_t>(atomicAdd(queue, 1ull));
        __syncthreads();
        return S.tile;
    };
    // jobs sized on the device (chain.cu) publish their tiles' total there
    if (tiles_dev != nullptr) total_tiles = min(total_tiles, *tiles_dev);
    for (int64_t tile = next_tile(); tile < total_tiles && !aborted; tile = next_tile()) {
        if (tid == 0) {
            const int j = find_base(tile_bases, num_jobs, tile);
            const ExpandJob &J = jobs[j];
            const int64_t t = tile - tile_bases[j];
            S.job = j;
            // a job sized on the device may have fewer tiles than the launch allows for
            S.i0 = t < J.num_tiles ? J.tile_first[t] : 0;
            S.i1 = t < J.num_tiles ? J.tile_first[t + 1] : 0;
        }
        __syncthreads();
        const ExpandJob &J = jobs[S.job];
        const int32_t i0 = S.i0, i1 = S.i1;
        const T *__restrict__ prev = static_cast<const T *>(J.prev_pts);
        T *__restrict__ outp = static_cast<T *>(J.out_pts);
        const int pair_max = J.pair_max;
        PhaseClock clk{tid == 0 ? J.phase_clk : nullptr, 0};
        clk.start();
        int32_t ic = i0;
        while (ic < i1) {
            const int n_stage = min(kTileItemCap, i1 - ic);
            // --- stage destinations: candidate starts and sizes, arc ranges
            constexpr int PER = kTileItemCap / kLT;
            static_assert(PER >= 1, "one destination per thread at least");
            int32_t cnt[PER], narc[PER];
            int32_t local = 0, local_a = 0;
#pragma unroll
            for (int r = 0; r < PER; ++r) {
                const int k = tid * PER + r;
                cnt[r] = 0;
                narc[r] = 0;
                if (k < n_stage) {
                    const int32_t i = ic + k;
                    const int32_t v = J.item_base + i;
                    const int32_t a0 = J.item_arc_off[v], a1 = J.item_arc_off[v + 1];
                    const int64_t s = J.arc_cand_off[a0 - J.arc_base];
                    const int64_t c = J.arc_cand_off[a1 - J.arc_base] - s;
                    J.out_off[i] = s;
                    const bool resident = c > 0 && tile_resident(c, a1 - a0);
                    if (c == 0) J.out_size[i] = 0;
                    if (J.out_sorted) J.out_sorted[i] = (c == 0 || resident) ? 1 : 0;
                    S.item_c0[k] = s;
                    S.item_a0g[k] = a0;
                    S.item_count[k] = 0;
                    if (resident) {
                        cnt[r] = static_cast<int32_t>(c);
                        narc[r] = a1 - a0;
                    }
                }
                local += cnt[r];
                local_a += narc[r];
            }
            const int32_t ex = block_exclusive_scan<int32_t, kLT>(local, S.warp_i, &S.tot_i);
            const int32_t exa = block_exclusive_scan<int32_t, kLT>(local_a, S.warp_i, &S.tot_a);
            // this pass takes the longest prefix of staged destinations whose arcs fit
            int32_t fit = 0;
            int32_t end_s[PER], end_a[PER];  // where this thread's destinations end
            {
                int32_t run = ex, runa = exa;
#pragma unroll
                for (int r = 0; r < PER; ++r) {
                    const int k = tid * PER + r;
                    if (k < n_stage) {
                        S.item_s[k] = static_cast<int16_t>(run);
                        S.item_arc0[k] = static_cast<int16_t>(runa);
                        if (runa + narc[r] <= kTileArcCap) ++fit;
                    }
                    run += cnt[r];
                    runa += narc[r];
                    end_s[r] = run;
                    end_a[r] = runa;
                }
            }
            (void)block_exclusive_scan<int32_t, kLT>(fit, S.warp_i, &S.tot_i);
            const int n_it = S.tot_i;  // >= 1: one destination has at most kTileArcCap / 2 arcs
            if (n_it == 0) {           // impossible for well-formed plans; skip defensively
                if (tid == 0) atomicOr(J.err, kErrBounds);
                break;
            }
            __syncthreads();
            // end markers of this pass, from the thread that staged its last destination
#pragma unroll
            for (int r = 0; r < PER; ++r) {
                if (tid * PER + r == n_it - 1) {
                    S.item_s[n_it] = static_cast<int16_t>(end_s[r]);
                    S.item_arc0[n_it] = static_cast<int16_t>(end_a[r]);
                    S.tot_i = end_s[r];
                    S.tot_a = end_a[r];
                }
            }
            if (tid == 0) {
                S.n_big = 0;
                S.next_big = 0;
                S.next_chunk = 0;
                S.n_slot = 0;
            }
            __syncthreads();
            const int32_t total = S.tot_i, total_a = S.tot_a;
            if (total > kTileCap || total_a > kTileArcCap) {  // impossible for well-formed offsets
                if (tid == 0) atomicOr(J.err, kErrBounds);
                break;
            }
            clk.lap(0);
            // --- stage the arcs of the small destinations (and whether each parent is sorted)
            for (int x = tid; x < total_a; x += kLT) {
                int lo = 0, hi = n_it - 1;  // destination owning staged arc x
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (S.item_arc0[mid] <= x) lo = mid;
                    else hi = mid - 1;
                }
                const int k = lo;
                const int32_t a = S.item_a0g[k] + (x - S.item_arc0[k]);
                const int64_t c0 = J.arc_cand_off[a - J.arc_base];
                const int32_t nb = J.arc_nbr[a] - J.prev_base;
                S.arc_pos[x] = static_cast<int16_t>(S.item_s[k] + (c0 - S.item_c0[k]));
                S.arc_src[x] = J.prev_off[nb];
                S.arc_w[x] = J.arc_wrow[a];
                S.arc_item[x] = static_cast<int16_t>(k);
                if (J.prev_sorted == nullptr || J.prev_sorted[nb] == 0) S.item_count[k] = 1;
            }
            if (tid == 0) S.arc_pos[total_a] = static_cast<int16_t>(total);
            for (int q = tid; q < total; q += kLT) S.tag[q] = -1;
            __syncthreads();
            if constexpr (D != 3) {  // a run from an unsorted parent leaves its destination unsorted
                if (J.out_sorted)
                    for (int k = tid; k < n_it; k += kLT)
                        if (S.item_count[k]) J.out_sorted[ic + k] = 0;
            }
            // --- bulk staging (J.lex_bulk): each parent run, widened to 16-byte boundaries,
            // goes to shared memory (the mpts area, unused until the merge) by one
            // cp.async.bulk completing on the block's barrier, while the arc assignment
            // below runs.  Frontier blocks are arena blocks (256-byte aligned, sizes
            // rounded up to 256 bytes), so the widened range stays inside the block.
            unsigned char *stage = reinterpret_cast<unsigned char *>(&S.mpts[0]);
            bool bulk = false;
            if (J.lex_bulk) {
                constexpr int AP = kTileArcCap / kLT;
                int32_t padded[AP];
                uintptr_t lo_addr[AP];
                int32_t local = 0;
#pragma unroll
                for (int r = 0; r < AP; ++r) {
                    const int x = tid * AP + r;
                    padded[r] = 0;
                    lo_addr[r] = 0;
                    if (x < total_a) {
                        const int len = S.arc_pos[x + 1] - S.arc_pos[x];
                        if (len > 0) {
                            const uintptr_t a = reinterpret_cast<uintptr_t>(prev + S.arc_src[x] * D);
                            const uintptr_t lo = a & ~static_cast<uintptr_t>(15);
                            const uintptr_t hi = (a + static_cast<uintptr_t>(len) * D * sizeof(T) + 15) &
                                                 ~static_cast<uintptr_t>(15);
                            padded[r] = static_cast<int32_t>(hi - lo);
                            lo_addr[r] = lo;
                        }
                    }
                    local += padded[r];
                }
                const int32_t ex = block_exclusive_scan<int32_t, kLT>(local, S.warp_i, &S.tot_stage);
                bulk = S.tot_stage <= static_cast<int32_t>(sizeof(S.mpts));
                if (bulk) {
                    int32_t run = ex;
#pragma unroll
                    for (int r = 0; r < AP; ++r) {
                        const int x = tid * AP + r;
                        if (x < total_a && padded[r] > 0) {
                            const uintptr_t a = reinterpret_cast<uintptr_t>(prev + S.arc_src[x] * D);
                            S.arc_stage[x] = run + static_cast<int32_t>(a - lo_addr[r]);
                        }
                        run += padded[r];
                    }
                    fence_proxy_async_smem();  // the last pass's reads and writes of mpts come first
                    __syncthreads();
                    if (tid == 0) mbar_arrive_expect_tx(&S.bar, static_cast<unsigned>(S.tot_stage));
                    __syncthreads();
                    run = ex;
#pragma unroll
                    for (int r = 0; r < AP; ++r) {
                        const int x = tid * AP + r;
                        if (x < total_a && padded[r] > 0)
                            bulk_g2s(stage + run, reinterpret_cast<const void *>(lo_addr[r]),
                                     static_cast<unsigned>(padded[r]), &S.bar);
                        run += padded[r];
                    }
                }
            }
            clk.lap(1);
            // --- each candidate's arc: mark every non-empty run's first position, then a
            // block-wide running maximum carries the arc over its run
            for (int x = tid; x < total_a; x += kLT)
                if (S.arc_pos[x + 1] > S.arc_pos[x]) S.tag[S.arc_pos[x]] = static_cast<int16_t>(x);
            __syncthreads();
            {
                constexpr int QP = kTileCap / kLT;
                int32_t run = -1, seen[QP];
#pragma unroll
                for (int r = 0; r < QP; ++r) {
                    const int q = tid * QP + r;
                    if (q < total) run = max(run, static_cast<int32_t>(S.tag[q]));
                    seen[r] = run;
                }
                const int32_t before = block_exclusive_max<kLT>(run, S.warp_i);
#pragma unroll
                for (int r = 0; r < QP; ++r) {
                    const int q = tid * QP + r;
                    if (q < total) S.tag[q] = static_cast<int16_t>(max(before, seen[r]));
                }
            }
            __syncthreads();
            if (bulk) {
                bool ok = false;
                for (int it = 0; it < kWaitIters && !ok; ++it) ok = mbar_try_wait(&S.bar, bar_phase);
                bar_phase ^= 1u;
                if (__syncthreads_or(!ok)) {
                    // the copies did not arrive: report, give them one more bounded wait, stop
                    if (tid == 0) atomicOr(J.err, kErrTimeout);
                    for (int it = 0; it < kWaitIters && !ok; ++it) ok = mbar_try_wait(&S.bar, bar_phase ^ 1u);
                    aborted = true;
                    break;
                }
            }
            clk.lap(2);
            // --- expand: candidate = parent point + arc weight (run order)
            for (int q = tid; q < total; q += kLT) {
                const int x = S.tag[q];
                const int k = S.arc_item[x];
                const int64_t idx = q - S.arc_pos[x];
                const T *src = bulk ? reinterpret_cast<const T *>(stage + S.arc_stage[x]) + idx * D
                                    : prev + (S.arc_src[x] + idx) * D;
                const int32_t *w = J.weights + static_cast<int64_t>(S.arc_w[x]) * D;
                PackedPt<D, T> pt;
#pragma unroll
                for (int o = 0; o < PackedPt<D, T>::kPad; ++o) pt.v[o] = o < D ? src[o] + static_cast<T>(w[o]) : T(0);
                S.pts[q] = pt;
                S.item_of[q] = static_cast<uint16_t>(k);
            }
            __syncthreads();
            clk.lap(3);
            // --- merge: each candidate's position in its destination's lexicographic order
            for (int q = tid; q < total; q += kLT) {
                const int k = S.item_of[q];
                const int x = S.tag[q];
                const int js = S.item_s[k], je = S.item_s[k + 1];
                const PackedPt<D, T> me = S.pts[q];
                int rank = 0;
                if (S.item_count[k] == 0) {
                    rank = q - S.arc_pos[x];
                    const int y0 = S.item_arc0[k], y1 = S.item_arc0[k + 1];
                    for (int y = y0; y < y1; ++y) {
                        if (y == x) continue;
                        const int lo = S.arc_pos[y], hi = (y + 1 < y1) ? S.arc_pos[y + 1] : je;
                        // points of run y before me: larger, or equal in a lower run; a prefix
                        const bool tie_first = y < x;
                        int a = lo, b = hi;
                        while (a < b) {
                            const int mid = (a + b) >> 1;
                            const PackedPt<D, T> c = S.pts[mid];
                            const bool before = ord_gt<D, T>(c, me) || (tie_first && ord_eq<D, T>(c, me));
                            if (before) a = mid + 1;
                            else b = mid;
                        }
                        rank += a - lo;
                    }
                } else if constexpr (D == 3) {
                    for (int j = js; j < je; ++j) {
                        const PackedPt<3, T> c = S.pts[j];
                        rank += (lex_gt(c, me) || (j < q && lex_eq(c, me))) ? 1 : 0;
                    }
                } else {
                    rank = q - js;  // a run from an unsorted parent: run order, swept in full below
                }
                S.mpts[js + rank] = me;
            }
            if constexpr (D == 3) {
                // segments for the staircase warps, those of the largest destinations first (three
                // tiers); a destination of more than kLexSeg candidates gets one slot per segment
                // but its last for the staircases the later segments are checked against
                for (int tier = 0; tier < 3; ++tier) {
                    const int lo_c = tier == 0 ? 512 : (tier == 1 ? 128 : pair_max);
                    const int hi_c = tier == 0 ? kTileCap : (tier == 1 ? 512 : 128);
                    for (int k = tid; k < n_it; k += kLT) {
                        const int c = S.item_s[k + 1] - S.item_s[k];
                        if (c > lo_c && c <= hi_c && c > pair_max) {
                            const int nseg = lex_segments(c);
                            const int at = atomicAdd(&S.n_big, nseg);
                            for (int g = 0; g < nseg; ++g) S.big[at + g] = k | (g << 16);
                            if (nseg > 1) S.item_slot0[k] = static_cast<int8_t>(atomicAdd(&S.n_slot, nseg - 1));
                        }
                    }
                    __syncthreads();
                }
                clk.lap(4);
                // --- filter, big destinations: one staircase warp per segment
                const long long f0 = (J.phase_clk && lane == 0) ? clock64() : 0;
                while (true) {
                    int b = 0;
                    if (lane == 0) b = atomicAdd(&S.next_big, 1);
                    b = __shfl_sync(kFull, b, 0);
                    if (b >= S.n_big) break;
                    const int k = S.big[b] & 0xffff, g = S.big[b] >> 16;
                    const int js = S.item_s[k], c = S.item_s[k + 1] - js;
                    const int nseg = lex_segments(c), len = (c + nseg - 1) / nseg;
                    if (g == 0 && lane == 0 && J.tile_surv != nullptr)
                        atomicAdd(J.tile_surv + 1, static_cast<unsigned long long>(c));
                    const int slot = g + 1 < nseg ? S.item_slot0[k] + g : -1;
                    stair_filter<T>(S, stairs[warp], js + g * len, js + min(c, (g + 1) * len), lane,
                                    slot >= 0 ? slots + slot : nullptr, slot >= 0 ? S.slot_m + slot : nullptr);
                }
                const long long f1 = (J.phase_clk && lane == 0) ? clock64() : 0;
                // --- filter, small destinations: every candidate against the points before it
                while (true) {
                    int c0 = 0;
                    if (lane == 0) c0 = atomicAdd(&S.next_chunk, 1) * 32;
                    c0 = __shfl_sync(kFull, c0, 0);
                    if (c0 >= total) break;
                    const int q = c0 + lane;
                    int js = q, len = 0;
                    if (q < total) {
                        const int k = S.item_of[q];
                        const int s0 = S.item_s[k], s1 = S.item_s[k + 1];
                        if (s1 - s0 <= pair_max) {
                            js = s0;
                            len = q - s0;
                        }
                    }
                    const bool mine = q < total && (S.item_s[S.item_of[q] + 1] - S.item_s[S.item_of[q]]) <= pair_max;
                    if (!__any_sync(kFull, mine)) continue;
                    T q1 = 0, q2 = 0;
                    if (mine) {
                        q1 = S.mpts[q].v[1];
                        q2 = S.mpts[q].v[2];
                    }
                    bool dom = !mine;
                    const int maxlen = warp_max_i(len);
                    for (int t = 0; t < maxlen; ++t) {
                        if (t < len) {
                            const PackedPt<3, T> c = S.mpts[js + t];
                            dom |= (c.v[1] >= q1) & (c.v[2] >= q2);
                        }
                        if ((t & 7) == 7 && __all_sync(kFull, dom)) break;
                    }
                    if (mine) S.keep[q] = dom ? 0 : 1;
                }
                if (J.phase_clk && lane == 0) {  // warp busy cycles: staircase loop, pairwise loop
                    const long long f2 = clock64();
                    atomicAdd(J.phase_clk + 7, static_cast<unsigned long long>(f1 - f0));
                    atomicAdd(J.phase_clk + 8, static_cast<unsigned long long>(f2 - f1));
                }
                __syncthreads();
                // --- filter, segmented destinations: a survivor of its own segment is checked
                // against the staircases of the segments before it (every point of a segment is
                // covered by an entry of its staircase), or their points if a staircase was not kept
                if (S.n_slot > 0) {
                    for (int q = tid; q < total; q += kLT) {
                        if (!S.keep[q]) continue;
                        const int k = S.item_of[q];
                        const int js = S.item_s[k], c = S.item_s[k + 1] - js;
                        if (c <= pair_max || c <= kLexSeg) continue;
                        const int nseg = lex_segments(c), len = (c + nseg - 1) / nseg;
                        const int g = (q - js) / len;
                        const T q1 = S.mpts[q].v[1], q2 = S.mpts[q].v[2];
                        bool dom = false;
                        for (int t = 0; t < g && !dom; ++t) {
                            const int slot = S.item_slot0[k] + t;
                            const int m = S.slot_m[slot];
                            if (m >= 0) {
                                int a = 0, b = m;  // entries with objective 1 >= q1
                                while (a < b) {
                                    const int mid = (a + b) >> 1;
                                    if (slots[slot].v1[mid] >= q1) a = mid + 1;
                                    else b = mid;
                                }
                                dom = a > 0 && slots[slot].v2[a - 1] >= q2;
                            } else {
                                for (int j = js + t * len; j < js + (t + 1) * len && !dom; ++j)
                                    dom = (S.mpts[j].v[1] >= q1) & (S.mpts[j].v[2] >= q2);
                            }
                        }
                        if (dom) S.keep[q] = 0;
                    }
                    __syncthreads();
                }
            } else {
                // --- filter, four objectives: a candidate is dominated only by a point before
                // it in sum order (a dominating point has the larger sum, an equal one comes
                // first), so each sweeps the points before it -- the likeliest dominators
                // first -- unless its destination has a run from an unsorted parent, which it
                // sweeps in full by the keep rule (another point >= and (different or first))
                __syncthreads();  // the merged order is complete
                clk.lap(4);
                while (true) {
                    int c0 = 0;
                    if (lane == 0) c0 = atomicAdd(&S.next_chunk, 1) * 32;
                    c0 = __shfl_sync(kFull, c0, 0);
                    if (c0 >= total) break;
                    const int q = c0 + lane;
                    const bool valid = q < total;
                    int js = INT_MAX, end = INT_MIN;
                    T p[D];
#pragma unroll
                    for (int o = 0; o < D; ++o) p[o] = T(0);
                    if (valid) {
                        const int k = S.item_of[q];
                        js = S.item_s[k];
                        end = S.item_count[k] ? S.item_s[k + 1] : q;
                        const PackedPt<D, T> me = S.mpts[q];
#pragma unroll
                        for (int o = 0; o < D; ++o) p[o] = me.v[o];
                    }
                    const int J0 = warp_min_i(js), J1 = warp_max_i(end);
                    bool dom = !valid;
                    for (int j = J0; j < J1; ++j) {
                        const PackedPt<D, T> c = S.mpts[j];
                        if (!dom && j >= js && j < end && j != q && ge_all<D, T>(c, p) &&
                            (j < q || !eq_all<D, T>(c, p)))
                            dom = true;
                        if (((j - J0) & 31) == 31 && __all_sync(kFull, dom)) break;
                    }
                    if (valid) S.keep[q] = dom ? 0 : 1;
                }
                __syncthreads();
            }
            clk.lap(5);
            // --- exclusive scan of keep flags (merged order)
            constexpr int QPER = kTileCap / kLT;
            int32_t kept_local = 0;
#pragma unroll
            for (int r = 0; r < QPER; ++r) {
                const int q = tid * QPER + r;
                if (q < total) kept_local += S.keep[q];
            }
            const int32_t kex = block_exclusive_scan<int32_t, kLT>(kept_local, S.warp_i, &S.tot_i);
            {
                int32_t run = kex;
#pragma unroll
                for (int r = 0; r < QPER; ++r) {
                    const int q = tid * QPER + r;
                    if (q < total) {
                        S.keep_ex[q] = static_cast<int16_t>(run);
                        run += S.keep[q];
                    }
                }
                if (tid == kLT - 1) S.keep_ex[total] = static_cast<int16_t>(run);
            }
            __syncthreads();
            if (tid == 0 && J.tile_surv != nullptr && S.keep_ex[total] > 0)
                atomicAdd(J.tile_surv, static_cast<unsigned long long>(S.keep_ex[total]));
            // --- write survivors into each destination's slot, in merged order
            for (int q = tid; q < total; q += kLT) {
                if (!S.keep[q]) continue;
                const int k = S.item_of[q];
                const int64_t dst = S.item_c0[k] + (S.keep_ex[q] - S.keep_ex[S.item_s[k]]);
                T *o_ = outp + dst * D;
                const PackedPt<D, T> me = S.mpts[q];
#pragma unroll
                for (int o = 0; o < D; ++o) o_[o] = me.v[o];
            }
            for (int k = tid; k < n_it; k += kLT) {
                const int js = S.item_s[k], je = S.item_s[k + 1];
                if (je > js) J.out_size[ic + k] = S.keep_ex[je] - S.keep_ex[js];
            }
            __syncthreads();
            clk.lap(6);
            ic += n_it;
        }
        __syncthreads();  // tile bookkeeping in shared memory is rewritten next iteration
    }
}

namespace {

template <int D, typename T>
cudaError_t launch_lex_t(const ExpandJob *jobs, const int64_t *tile_bases, int num_jobs, int64_t total_tiles, int grid,
                         unsigned long long *queue, const int64_t *tiles_dev, cudaStream_t stream) {
    if constexpr (D == 3)
        static_assert(sizeof(Stair<T>) * kLexWarps + sizeof(SegStair<T>) * kLexSlots <= sizeof(PackedPt<3, T>) * kTileCap,
                      "staircases fit over pts");
    const size_t smem = sizeof(LexSmem<D, T>);
    const cudaError_t e = ensure_smem_limit(reinterpret_cast<const void *>(expand_tile_lex_kernel<D, T>), smem);
    if (e != cudaSuccess) return e;
    if (total_tiles <= 0) return cudaSuccess;
    const int64_t g = std::min<int64_t>(total_tiles, grid);
    expand_tile_lex_kernel<D, T><<<static_cast<unsigned>(g), kLT, smem, stream>>>(jobs, tile_bases, num_jobs,
                                                                                 total_tiles, queue, tiles_dev);
    return cudaGetLastError();
}

}  // namespace

bool lex_tiles_cover(int d, bool wide) { return d == 3 || (d == 4 && !wide); }

cudaError_t launch_expand_tiles_lex(int d, bool wide, const ExpandJob *jobs, const int64_t *tile_bases, int num_jobs,
                                    int64_t total_tiles, int grid, unsigned long long *queue,
                                    const int64_t *tiles_dev, cudaStream_t stream) {
    if (d == 3 && wide)
        return launch_lex_t<3, int64_t>(jobs, tile_bases, num_jobs, total_tiles, grid, queue, tiles_dev, stream);
    if (d == 3) return launch_lex_t<3, int32_t>(jobs, tile_bases, num_jobs, total_tiles, grid, queue, tiles_dev, stream);
    if (d == 4 && !wide)
        return launch_lex_t<4, int32_t>(jobs, tile_bases, num_jobs, total_tiles, grid, queue, tiles_dev, stream);
    return cudaErrorInvalidValue;
}

}  // namespace dev
}  // namespace pmdd
