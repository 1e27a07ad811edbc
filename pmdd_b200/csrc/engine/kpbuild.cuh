// Exact knapsack BDDs built on the device (kpbuild.cu), one thread block per instance.
//
// Same DD as the host constructor (pmdd_b200/csrc/host/dd_build.cpp: build_knapsack_bdd,
// after the reference's KnapsackBDDConstructor::generate_exact, BDDAlg::reduce and
// update_node_weights, src/pmdd/bdd/knapsack_bdd.cpp:10-150, src/pmdd/bdd/bdd_alg.hpp:24-93),
// array for array: same node numbering, same incoming-arc order, same min_weight.
// Single constraint with non-negative weights and capacity, so a layer's states are
// used capacities 0..cap and every per-layer structure is a dense array over them:
//
//  kp_reduce_kernel   top-down: state s' of layer l+1 is numbered by the first place it
//                     is seen when the parents are walked in index order (0-arc, then
//                     1-arc) -- rank of min(2*idx(s'), 2*idx(s'-w)+1) among the layer's keys;
//                     bottom-up: the states of a layer whose (0-child, 1-child) classes
//                     agree merge.  Completion sets shrink as s grows, so the merged states
//                     form runs of consecutive reachable states; a class is numbered by the
//                     smallest old index among its states (first occurrence).
//  kp_flatten_kernel  top-down again over the classes: in-arc CSR (1-arcs, then 0-arcs,
//                     each by parent id; the parents of one child through one arc type are
//                     a run of consecutive classes in state order), min_weight (min over
//                     in-arcs), the weight table, and the min_weight order per layer
//                     (descending; min_weight is the smallest state of a class, so it is
//                     the reverse state order -- checked).
#pragma once

#include "common.cuh"

namespace pmdd {
namespace dev {

constexpr int kKpThreads = 1024;

struct KpBuildJob {
    int32_t n;               // items; the BDD has n+1 layers
    int32_t cap;             // capacity, >= 0
    int32_t nobjs;
    int32_t pad;
    const int32_t *w;        // [n] item weights, >= 0
    const int32_t *profit;   // [nobjs][n]
    // scratch, S = cap+1 ints per row
    int32_t *idx;            // [(n+1)*S] index of each reachable state, -1 elsewhere
    int32_t *tmp;            // [10*S]
    int32_t *cls_new;        // [(n+1)*S] per layer: class (state order) -> node id
    int32_t *cls_c0;         // [(n+1)*S] per layer: class -> 0-child node id
    int32_t *cls_c1;         // [(n+1)*S] per layer: class -> 1-child node id or -1
    // header (kp_reduce_kernel)
    int32_t *width;          // [n+1] unreduced layer sizes
    int32_t *classes;        // [n+1] reduced layer sizes
    int32_t *arcs_into;      // [n+1] arcs into each layer
    int32_t *err;            // 0 ok; 1 inconsistent counts; 2 min_weight order check failed
    // the flat DD (kp_flatten_kernel), pmdd_dd layout
    int32_t *layer_offsets, *in_arc_offsets, *arc_src, *arc_weight, *weights, *min_weight, *sd_order;
};

// Scratch ints of one job.
inline int64_t kp_scratch_ints(int32_t n, int32_t cap) {
    const int64_t S = static_cast<int64_t>(cap) + 1;
    return (4 * (static_cast<int64_t>(n) + 1) + 10) * S;
}

cudaError_t launch_kp_reduce(const KpBuildJob *jobs, int count, cudaStream_t stream);
cudaError_t launch_kp_flatten(const KpBuildJob *jobs, int count, int max_layers, cudaStream_t stream);

}  // namespace dev
}  // namespace pmdd
