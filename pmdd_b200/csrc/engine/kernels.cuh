// Launchers of the enumeration kernels (kernels.cu, couple.cu).  `d` selects the
// objective count (1..8), `wide` the int64 point type.
#pragma once

#include "common.cuh"

namespace pmdd {
namespace dev {

cudaError_t launch_count_scan(const CountJob *jobs, int num_jobs, cudaStream_t stream);
// One chained layer's sizes from the counts before it (chain.cu); one block, P.n <= kChainThreads.
cudaError_t launch_chain_prep(const ChainPrep &P, cudaStream_t stream);
// `queue`: a zeroed device counter from which the launch's blocks draw tiles;
// `tiles_dev` (or nullptr): the jobs' tiles in total, written on the device before the
// launch, when total_tiles is only a bound (chained layers).
cudaError_t launch_expand_tiles(int d, bool wide, const ExpandJob *jobs, const int64_t *tile_bases, int num_jobs,
                                int64_t total_tiles, int grid, unsigned long long *queue, const int64_t *tiles_dev,
                                cudaStream_t stream);
// Three objectives (frontiers in descending lexicographic order) and four with int32
// points (descending objective sum) (tile_lex.cu); lex_tiles_cover says which.
bool lex_tiles_cover(int d, bool wide);
cudaError_t launch_expand_tiles_lex(int d, bool wide, const ExpandJob *jobs, const int64_t *tile_bases, int num_jobs,
                                    int64_t total_tiles, int grid, unsigned long long *queue,
                                    const int64_t *tiles_dev, cudaStream_t stream);
// Fills every job's tile_first (destination i belongs to tile min(start_i / kTileWindow,
// num_tiles - 1)); one thread per destination over all jobs.
cudaError_t launch_tile_plan(const ExpandJob *jobs, const int64_t *item_bases, int num_jobs, int64_t total_items,
                             cudaStream_t stream);
// One scratch pass (see ExpandJob::big_window) of the oversized destinations of one
// (d, wide) group.
struct BigLaunch {
    const ExpandJob *jobs;
    const BigWork *work;         // every oversized destination of the group
    int num_work;
    const int64_t *job_bases;    // exclusive prefix of the jobs' big_rows (flat candidate space)
    int num_jobs;
    int64_t total;               // sum of the jobs' big_rows
    int64_t pass;
    int sms;
    bool with_sfs;               // launch the SFS blocks (destinations below big_mark_min)
    void *plan;                  // big_plan_bytes(mark_cap) of scratch for the mark path
    int mark_cap;                // upper bound on mark-path destinations in the pass; 0: none
    int32_t *order;              // num_work ints: SFS blocks largest destination first; nullptr: list order
    bool lex_big;                // three objectives: destinations with sorted runs take big_lex.cu
    int lex_rounds;              // merge rounds the destinations with the most runs need
};
// Most oversized destinations whose SFS blocks are put in size order (one block sorts them).
constexpr int kBigOrderMax = 4096;
size_t big_plan_bytes(int cap);
cudaError_t launch_big(int d, bool wide, const BigLaunch &L, cudaStream_t stream);
// The lexicographic oversized path (big_lex.cu), three objectives: the rank kernel takes
// the place of the materialising expansion, the filter runs after the other paths.
cudaError_t launch_big_lex_rank(bool wide, const BigLaunch &L, cudaStream_t stream);
cudaError_t launch_big_lex_merge(bool wide, const BigLaunch &L, int round, cudaStream_t stream);
cudaError_t launch_big_lex_filter(bool wide, const BigLaunch &L, cudaStream_t stream);

}  // namespace dev
}  // namespace pmdd
