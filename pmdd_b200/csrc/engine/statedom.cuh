// Knapsack state dominance on the device (statedom.cu).
//
// After a top-down layer of a knapsack BDD has been expanded and filtered, the nodes of
// the layer that hold labels are taken in order of decreasing min_weight (ties by
// ascending node id).  A label of node i is removed when a label of one of the next two
// such nodes is >= on every objective; a partner is skipped when both nodes have a single
// incoming arc, from the same parent, of different arc types.  All comparisons read the
// labels as they were before the pass.  This is the rule of the reference's GPU pass
// (src/pmdd/enum/gpu/topdown.cu:256-521, applied per layer at :966-988) and of its CPU
// pass (src/pmdd/enum/cpu/dominance.cpp:24-86).
#pragma once

#include "common.cuh"

namespace pmdd {
namespace dev {

struct StateDomJob {
    const int32_t *order;     // layer-local node ids by min_weight descending, ties by id (num_nodes)
    const int32_t *in_off;    // the DD's incoming-arc offsets (global node ids)
    const int32_t *arc_src;   // tail of each incoming arc (global node id)
    const int32_t *arc_w;     // weight row of each arc; row 0 is the 0-arc row
    void *pts;                // the layer's frontier in slot layout
    const int64_t *off;       // slot start of each node (points)
    int32_t *size;            // live labels of each node (rewritten)
    uint8_t *keep;            // scratch: one flag per slot position of the layer
    int64_t *removed;         // labels removed by this pass (added to)
    int32_t node_base;        // global id of the layer's first node
    int32_t num_nodes;
};

// Marks, then compacts; `node_bases` is the exclusive prefix sum of num_nodes over the
// jobs and `total_nodes` its total.
cudaError_t launch_state_dominance(int d, bool wide, const StateDomJob *jobs, const int64_t *node_bases, int num_jobs,
                                   int64_t total_nodes, int sms, cudaStream_t stream);

}  // namespace dev
}  // namespace pmdd
