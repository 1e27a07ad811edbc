// Layer chaining: a small engine step lets its requests expand several more layers before
// the host reads anything back.
//
// An ordinary step ends with one device->host copy of the counts of the next layer, from
// which the host sizes that layer's frontier slots and tiles.  When a step has few
// candidates, that round trip (and the host's planning) costs more than the kernels, so
// a request expanding by method 1 without state dominance is chained: the host stages
// every further layer's expansion and count descriptors up front, with ping-pong frontier
// buffers of a fixed capacity, and the sizes it would have read back are filled in on the
// device -- the candidates from the count before, the tiles they need, each tile's first
// destination and each request's first tile.  For a chain's first layer (after the
// step's own counts) chain_prep_kernel below and tile_plan_kernel do that; every later
// layer is sized and planned by the count kernel of the layer before it (count.cu), so a
// chained layer costs two launches, the tiles and the counts.  A request stops, for good
// within the step, at a layer that has an oversized destination (the oversized path
// needs host-sized scratch), whose candidates exceed its buffers, or past its last
// chained layer; its expansion then has no tiles and its count returns at once, and the
// host resumes it from the last layer it finished.
#include "kernels.cuh"
#include "scan.cuh"

namespace pmdd {
namespace dev {

__global__ void __launch_bounds__(kChainThreads) chain_prep_kernel(ChainPrep P) {
    __shared__ int64_t warp_buf[32];
    __shared__ int64_t s_total;
    const int i = threadIdx.x;
    int64_t tiles = 0;
    if (i < P.n) {
        const CountResult r = P.prev[P.prev_idx != nullptr ? P.prev_idx[i] : i];
        ExpandJob &J = P.jobs[i];
        const bool stop = P.stop[i] != 0 || P.layer > P.last[i] || r.num_big > 0 || r.total > P.cap[i] ||
                          !chain_side_goes_on(r.total, P.other_score[i], P.bu[i] != 0);
        if (stop) {
            if (P.stop[i] == 0) {
                P.stop[i] = 1;
                P.stopped_at[i] = P.layer;
            }
            J.total_cand = 0;
            J.num_tiles = 0;
        } else {
            tiles = r.total > 0 ? (r.total + J.tile_window - 1) / J.tile_window : 1;
            J.total_cand = r.total;
            J.num_tiles = tiles;
        }
    }
    const int64_t ex = block_exclusive_scan<int64_t, kChainThreads>(tiles, warp_buf, &s_total);
    if (i < P.n) P.tile_bases[i] = ex;
    if (i == 0) *P.tiles_total = s_total;
}

cudaError_t launch_chain_prep(const ChainPrep &P, cudaStream_t stream) {
    if (P.n <= 0 || P.n > kChainThreads) return cudaErrorInvalidValue;
    chain_prep_kernel<<<1, kChainThreads, 0, stream>>>(P);
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace pmdd
