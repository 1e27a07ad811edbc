// Launchers of the enumeration kernels (kernels.cu, couple.cu).  `d` selects the
// objective count (1..8), `wide` the int64 point type.
#pragma once

#include "common.cuh"

namespace pmdd {
namespace dev {

cudaError_t launch_count_scan(const CountJob *jobs, int num_jobs, cudaStream_t stream);
cudaError_t launch_expand_tiles(int d, bool wide, const ExpandJob *jobs, const int64_t *tile_bases, int num_jobs,
                                int64_t total_tiles, int grid, cudaStream_t stream);
// Fills every job's tile_first (destination i belongs to tile min(start_i / kTileWindow,
// num_tiles - 1)); one thread per destination over all jobs.
cudaError_t launch_tile_plan(const ExpandJob *jobs, const int64_t *item_bases, int num_jobs, int64_t total_items,
                             cudaStream_t stream);
// Oversized destinations of scratch pass `pass` (see ExpandJob::big_window): expand,
// then the single-block SFS for those below ExpandJob::big_mark_min candidates;
// `with_mark` also launches the GPU-wide mark and write passes for the larger ones.
cudaError_t launch_big(int d, bool wide, const ExpandJob *jobs, const BigWork *work, int num_work, int64_t max_item,
                       bool with_mark, int64_t pass, cudaStream_t stream);

}  // namespace dev
}  // namespace pmdd
