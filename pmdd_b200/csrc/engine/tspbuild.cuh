// The TSP MDD of n cities built on the device (tspbuild.cu).
//
// The host constructor (pmdd_b200/csrc/host/dd_build.cpp: build_tsp_mdd, after the
// reference's MDDTSPConstructor::generate_exact, src/pmdd/mdd/tsp_mdd.cpp:21-196) makes
// layers 0..n+1: the root, ({0}, 0), then one layer per further city over every state
// (S, last) with 0 in S and last in S \ {0}, then the terminal.  Every such state is
// reachable, so the layers, the node numbering and the arcs depend on n alone; only the
// weight table (negated costs) depends on the instance.  The structure is therefore built
// once per n and shared by every TSP instance of that size.
//
// Numbering (first sighting, parents in id order, cities ascending): child (S, v) of
// layer l+1 gets the rank of n * min_u id(S \ {v}, u) + v among the layer's keys, u over
// the parent states' last cities.  Incoming arcs of a child are its parents in id order,
// one per u, with weight row 1 + u*n + v; every node of layer l >= 3 has l - 2 of them.
// States are dense: (S, last) -> (S >> 1) * n + last, S < 2^n.
#pragma once

#include <cstdint>
#include <vector>

#include "common.cuh"

namespace pmdd {
namespace dev {

constexpr int kTspMinCities = 2;
constexpr int kTspMaxCities = 20;

// Layer sizes and incoming-arc counts of the n-city MDD (layers 0..n+1), from the
// combinatorics above: layer l >= 2 holds C(n-1, l-1) * (l-1) states.
struct TspShape {
    std::vector<int32_t> layer_off;  // n+3
    std::vector<int32_t> arc_at;     // n+3: in-arcs of layers < l
    int32_t max_width = 0;
};
TspShape tsp_shape(int n);

// Builds layer_offsets / in_arc_offsets / arc_src / arc_weight of the n-city MDD into
// the given device arrays (sized by tsp_shape).  `scratch` must hold
// tsp_scratch_bytes(n) bytes; `err` (device int) is set non-zero if a layer's size
// differs from tsp_shape's.  Launches 4 kernels per layer on `stream`.
size_t tsp_scratch_bytes(int n);
cudaError_t launch_tsp_structure(int n, const TspShape &shape, int32_t *layer_offsets, int32_t *in_arc_offsets,
                                 int32_t *arc_src, int32_t *arc_weight, void *scratch, int32_t *err, int sms,
                                 cudaStream_t stream, int64_t *launches);

}  // namespace dev
}  // namespace pmdd
