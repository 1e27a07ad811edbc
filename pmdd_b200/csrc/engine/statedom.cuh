// State dominance between the nodes of one top-down layer, on the device (statedom.cu).
// It runs after the layer has been expanded and filtered, and removes labels only: the
// final frontier is unchanged.  All comparisons read the labels as they were before the
// pass (in the reference's sequential loops a node is only ever compared with nodes that
// it has not pruned yet, so the order of the passes does not matter).
//
// Knapsack (kind 1).  The nodes of the layer that hold labels are taken in order of
// decreasing min_weight (ties by ascending node id).  A label of node i is removed when a
// label of one of the next two such nodes is >= on every objective; a partner is skipped
// when both nodes have a single incoming arc, from the same parent, of different arc
// types.  This is the rule of the reference's GPU pass
// (src/pmdd/enum/gpu/topdown.cu:256-521, applied per layer at :966-988) and of its CPU
// pass (src/pmdd/enum/cpu/dominance.cpp:24-86).
//
// Set packing (kind 2).  Every node of the layer (labels or not) sits in the bucket of
// its state size.  A node whose bucket holds two or more nodes takes as partner the first
// node, in layer order, of the next non-empty bucket whose state has the same lowest
// vertex, is not its single-parent sibling (as above), and contains its state; a label
// of the node is removed when a label of the partner is >= on every objective.  This is
// the reference's CPU pass (src/pmdd/enum/cpu/dominance.cpp:88-173); the reference's GPU
// path has none.
#pragma once

#include "common.cuh"

namespace pmdd {
namespace dev {

struct StateDomJob {
    const int32_t *order;     // layer-local node ids in the kind's order (num_nodes)
    const int32_t *next;      // kind 2: per order position, the [begin, end) order range of its partner bucket
    const uint64_t *state;    // kind 2: the DD's node states (global ids, state_words words each)
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
    int32_t kind;             // 1 knapsack, 2 set packing
    int32_t state_words;
};

// Marks, then compacts; `node_bases` is the exclusive prefix sum of num_nodes over the
// jobs and `total_nodes` its total.
cudaError_t launch_state_dominance(int d, bool wide, const StateDomJob *jobs, const int64_t *node_bases, int num_jobs,
                                   int64_t total_nodes, int sms, cudaStream_t stream);

}  // namespace dev
}  // namespace pmdd
