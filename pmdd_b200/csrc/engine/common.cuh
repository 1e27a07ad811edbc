// Shared device-side definitions of the enumeration engine.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <utility>

namespace pmdd {
namespace dev {

// Raises a kernel's dynamic shared-memory limit on the current device, once per
// (kernel, device).  The attribute belongs to the device's context, so a process that
// drives several GPUs, or calls in with another device current, sets it on each; the
// registry is shared by every host thread.
inline cudaError_t ensure_smem_limit(const void *func, size_t bytes) {
    static std::mutex mu;
    static std::set<std::pair<const void *, int>> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if (done.count({func, dev})) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    if (e == cudaSuccess) done.insert({func, dev});
    return e;
}

// Fused expand+filter tiles: a tile owns every destination whose candidate range
// starts inside its window of at most kTileWindow candidates; destinations of at most
// kSmallMax candidates are filtered in shared memory, larger ones take the
// global-memory ("big") path.  A tile therefore holds < 2*kTileWindow candidates.  The
// window shrinks (to kTileWindowMin) for steps with few candidates, so that a small
// step still spreads over the SMs.
constexpr int kTileThreads = 512;
constexpr int kTileWindow = 1024;
constexpr int kTileWindowMin = 128;
constexpr int kSmallMax = 1024;
constexpr int kTileCap = 2 * kTileWindow;
// Per-pass staging caps, sized so that a tile's shared memory (about 70 KB at d=3) lets
// three 512-thread blocks share an SM.
constexpr int kTileItemCap = 512;    // destinations staged per pass inside one tile
constexpr int kTileArcCap = 1024;    // arcs staged per pass inside one tile

// Destinations filtered inside a tile; every other destination takes the oversized
// path.  Both the counting pass and the tile kernel decide with this one rule.
__host__ __device__ constexpr bool tile_resident(int64_t candidates, int64_t arcs) {
    return candidates <= kSmallMax && arcs <= kTileArcCap / 2;
}

// Oversized three-objective destinations in lexicographic order (big_lex.cu): up to
// kBigDirectArcs runs each candidate is ranked against the other runs directly; beyond,
// ceil(log2(runs)) merge rounds of neighbouring run groups sort the destination; more
// than ExpandJob::lex_max_arcs (at most kBigLexMaxArcs) runs take the pivot/mark path.
constexpr int kBigDirectArcs = 16;
constexpr int kBigLexMaxArcs = 4096;
__host__ __device__ inline int lex_merge_rounds(int arcs) {
    int r = 0;
    if (arcs > kBigDirectArcs)
        while ((1 << r) < arcs) ++r;
    return r;
}

constexpr int kCountThreads = 1024;
constexpr int kBigThreads = 256;
constexpr int kBigJTile = 1024;       // candidates per shared-memory comparison tile

// Device error word bits (written with atomicOr; read back once per step).
constexpr uint32_t kErrBounds = 1u;        // an index check failed (work skipped)
constexpr uint32_t kErrCoupleOverflow = 2u;
constexpr uint32_t kErrTimeout = 4u;       // a bounded wait (bulk-copy barrier) gave up

// One layer expansion of one instance in one direction.  "Items" are the destination
// nodes of the layer; each has a contiguous range of arcs whose neighbour (the arc's
// other end, in the previous layer of this direction) carries a frontier.
struct ExpandJob {
    const int32_t *item_arc_off;   // [global node id] -> first arc; range end at v+1
    const int32_t *arc_nbr;        // neighbour node (global id)
    const int32_t *arc_wrow;       // weight row per arc
    const int32_t *weights;        // [rows * D]
    const int64_t *arc_cand_off;   // [arc - arc_base] -> first candidate of the arc; A+1 entries
    int32_t arc_base;
    int32_t item_base;             // global id of the first destination node
    int32_t num_items;
    int32_t prev_base;             // global id of the first neighbour-layer node
    const void *prev_pts;          // neighbour frontiers (slot layout, D values per point)
    const int64_t *prev_off;       // [local neighbour] -> slot start (points)
    const int32_t *prev_size;      // [local neighbour] -> live points in slot
    void *out_pts;                 // destination slots: total_cand points
    int64_t *out_off;              // [local item] -> slot start
    int32_t *out_size;             // [local item] -> survivors
    int64_t total_cand;
    int64_t tile_base;             // first global tile index of this job
    int64_t num_tiles;
    int64_t tile_window;           // candidates per tile window (kTileWindowMin..kTileWindow)
    int32_t *tile_first;           // [num_tiles+1]: first destination of each tile (tile_plan_kernel)
    const int64_t *big_list;       // (local item, scratch offset) pairs
    int32_t num_big;
    int32_t pivot_rule;            // pivots per mark-path destination of n candidates:
                                   // 1: 4*sqrt(n) within [32, 4096]; 0: n/64 within [512, 4096]
    void *big_pts;                 // scratch: candidates of oversized destinations (AoS)
    void *big_pts2;                // scratch: the same candidates in sum-bucket order
    void *big_surv;                // scratch: survivors of one bucket that overflow shared memory
    int32_t *big_idx;              // scratch: candidate index of each bucket-ordered point
    int32_t *big_surv_idx;         // scratch: candidate index of each overflowing survivor
    int64_t big_mark_min;          // oversized destinations of at least this many candidates take the mark path
    int64_t big_window;            // pass p takes the destinations whose scratch offset is in
                                   // [p * big_window, (p + 1) * big_window) (--max-cand)
    int64_t big_rows;              // scratch rows (candidates) one pass can use
    uint32_t *err;
    unsigned long long *tile_surv; // [0]: survivors written by the tile kernel, [1]: candidates of
                                   // destinations filtered by staircase warps (both added to)
    // Lexicographic order (three objectives): a node whose flag is 1 holds its frontier in
    // descending lexicographic order.  prev_sorted is indexed like prev_size; the tile
    // kernels write out_sorted for every destination they stage (1 only when they wrote
    // it in that order); nullptr when the job keeps no flags.
    const uint8_t *prev_sorted;
    uint8_t *out_sorted;
    int32_t pair_max;              // lexicographic tiles: destinations of at most this many
                                   // candidates are checked pairwise, larger ones by a staircase warp
    int32_t lex_big;               // 1: oversized destinations with sorted runs take big_lex.cu
    int32_t lex_bulk;              // 1: lexicographic tiles stage parent runs by bulk copies
    int32_t lex_max_arcs;          // oversized destinations of at most this many runs (and at
                                   // most kBigLexMaxArcs) take big_lex.cu
    unsigned long long *phase_clk; // diagnostic: cycles per tile phase (lexicographic tiles), or nullptr
};

// Bytes of oversized-destination scratch per candidate point.
constexpr size_t big_scratch_bytes_per_point(int d, size_t elem) { return 3 * d * elem + 2 * sizeof(int32_t); }

// Counting pass for the next layer of one direction.
struct CountJob {
    const int32_t *item_arc_off;
    const int32_t *arc_nbr;
    int32_t arc_base;
    int32_t num_arcs;
    int32_t item_base;
    int32_t num_items;
    int32_t cur_base;              // global id of the first node of the current layer
    int32_t cur_nodes;             // nodes in the current layer
    const int32_t *cur_size;       // [local current node] -> frontier size
    int64_t *arc_cand_off;         // out: num_arcs + 1 entries
    int64_t *big_list;             // out: (local item, scratch offset) pairs, capacity num_items
    struct CountResult *result;    // out
    // Chained layers (chain.cu): nothing to count while *stop != 0.  With `next`, the block
    // then sizes and plans this request's next chained expansion from the counts (what
    // chain_prep_kernel and tile_plan_kernel do for a chain's first layer), and the last
    // block of the launch to finish writes every request's first tile.
    int32_t *stop;
    int32_t *stopped_at;
    struct ExpandJob *next;        // nullptr: no next chained expansion
    int64_t *next_tiles;           // [chain_n] tiles of each request's next expansion (0: stopped)
    int64_t *next_bases;           // [chain_n] out: exclusive prefix of next_tiles
    int64_t *next_total;           // out: their sum
    unsigned int *done;            // zeroed: blocks of the launch that have finished
    int64_t cap;                   // candidates the next expansion's buffers hold
    int32_t next_layer;            // the next expansion's chained layer, from 1
    int32_t last;                  // the request's last chained layer
    int32_t slot;                  // the request's index in the launch (= block)
    int32_t chain_n;               // requests (blocks) in the launch
    int32_t bu;                    // the chained side is the bottom-up one (method 3)
    int64_t other_score;           // the other side's score (ChainPrep::other_score)
};

// Whether a chained side goes on after a count of `total` candidates (see ChainPrep).
__host__ __device__ inline bool chain_side_goes_on(int64_t total, int64_t other_score, bool bu) {
    return bu ? other_score > static_cast<int64_t>(1.5 * static_cast<double>(total)) : total <= other_score;
}

struct CountResult {
    int64_t total;       // candidates of the next layer
    int64_t max_item;    // largest destination
    int64_t big_total;   // candidates in destinations above kSmallMax
    int64_t cur_total;   // points of the current layer's frontiers (survivor statistics)
    int32_t num_big;
    int32_t max_big_arcs;  // most arcs of an oversized destination
};

// One chained layer of a group of requests (chain.cu): sizes that layer's expansions from
// the counts before them, on the device, so that the host need not read them back.
constexpr int kChainThreads = 1024;  // most requests one chain group takes
struct ChainPrep {
    struct ExpandJob *jobs;        // [n] this layer's expansions: total_cand, num_tiles written
    int64_t *tile_bases;           // [n] written: first tile of each expansion
    int64_t *tiles_total;          // written: the expansions' tiles in total
    const CountResult *prev;       // the counts these expansions read, slot i at prev[prev_idx[i]]
    const int32_t *prev_idx;       // nullptr: slot i reads prev[i]
    int32_t *stop;                 // [n] per request, sticky: 1 once its chain has stopped
    int32_t *stopped_at;           // [n] the layer at which it stopped (0: never)
    const int64_t *cap;            // [n] candidates its chained frontier buffers hold
    const int32_t *last;           // [n] its last chained layer
    // [n] method 3: a chain goes on while the host would pick the same side again, its
    // new score against the other side's (other_score; INT64_MAX for method 1): top-down
    // (bu 0) while candidates <= other_score, bottom-up (bu 1) while other_score >
    // 1.5 * candidates (the engine's side rule, Engine::step)
    const int64_t *other_score;
    const int32_t *bu;
    int32_t layer;                 // this layer, from 1
    int32_t n;
};

// Big-path work entry: one oversized destination of one job.
struct BigWork {
    int32_t job;
    int32_t big;       // index into the job's big_list
};

}  // namespace dev
}  // namespace pmdd
