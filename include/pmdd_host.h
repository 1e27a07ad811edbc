/*
 * pmdd_host.h -- C ABI of the host-side front end (libpmdd_host.so): instance
 * parsers and exact decision-diagram constructors that feed the GPU engine.
 *
 * These replace the reference's CPU-side producers of the DD that its GPU seam
 * consumes; they emit the flat layout of pmdd_dd (pmdd.h) directly instead of the
 * reference's pointer graph:
 *
 *   problem 1 (knapsack BDD)   KnapsackInstance::read        src/pmdd/instances/knapsack_instance.cpp:17-47
 *                              KnapsackBDDConstructor::generate_exact / update_node_weights
 *                                                            src/pmdd/bdd/knapsack_bdd.cpp:10-150
 *                              BDDAlg::reduce                src/pmdd/bdd/bdd_alg.hpp:24-93
 *                              (two reduce + weight passes, src/pmdd/main.cpp:120-153)
 *   problem 2 (set packing ->  SetPackingInstance(...)       src/pmdd/instances/setpacking_instance.hpp:49-126
 *    independent-set BDD)      IndepSetBDDConstructor::generate_exact
 *                                                            src/pmdd/bdd/indepset_bdd.cpp:50-165
 *                              min-in-state vertex ordering  src/pmdd/bdd/indepset_bdd.hpp:89-114
 *   problem 3 (TSP MDD)        TSPInstance::read             src/pmdd/instances/tsp_instance.cpp:11-39
 *                              MDDTSPConstructor::generate_exact
 *                                                            src/pmdd/mdd/tsp_mdd.cpp:21-196
 *
 * Layer sizes, node counts and arc counts equal the reference's for the same file
 * (node numbering inside a layer may differ: the reference numbers nodes in hash
 * iteration order).
 */
#ifndef PMDD_HOST_H_
#define PMDD_HOST_H_

#include <stddef.h>
#include <stdint.h>

#include "pmdd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pmdd_host_dd pmdd_host_dd;

/* Structure summary, same meaning as the reference's DDStats
 * (src/pmdd/util/stats.hpp:88-109); -1 where the reference reports -1 (TSP). */
typedef struct pmdd_dd_info {
    int64_t original_width;
    int64_t reduced_width;
    int64_t original_num_nodes;
    int64_t reduced_num_nodes;
    int64_t max_num_in_arcs;     /* largest per-layer incoming-arc total */
    int64_t total_num_in_arcs;
    int32_t num_layers;
    int32_t problem_type;
} pmdd_dd_info;

/* Parses an instance in the reference's text format from `path` (or from the
 * NUL-terminated `text`) and compiles the exact DD for `nobjs` objectives
 * (the first `nobjs` objectives of the file, as the reference's NOBJS build does).
 * Returns NULL and writes `err` on failure. */
pmdd_host_dd *pmdd_build_from_file(const char *path, int32_t problem_type, int32_t nobjs,
                                   char *err, size_t errlen);
pmdd_host_dd *pmdd_build_from_text(const char *text, int32_t problem_type, int32_t nobjs,
                                   char *err, size_t errlen);

/* Borrowed view of the flat DD (valid until pmdd_host_dd_free). */
int pmdd_host_dd_view(const pmdd_host_dd *h, pmdd_dd *view);
int pmdd_host_dd_info(const pmdd_host_dd *h, pmdd_dd_info *info);
/* Copies the per-layer node counts (num_layers values) into `out`. */
int pmdd_host_dd_layer_sizes(const pmdd_host_dd *h, int64_t *out, int32_t cap);
void pmdd_host_dd_free(pmdd_host_dd *h);

/* Sorts `num_points` points of `nobjs` int32 values ascending lexicographically,
 * in place (the reference's ParetoFrontier::sort_lexicographic_ascending,
 * src/pmdd/enum/pareto_frontier.hpp:418-433). */
void pmdd_sort_points_lex_ascending(int32_t *points, int64_t num_points, int32_t nobjs);

/* ------------------------------------------------------------------ output writers
 * The frontier CSV.gz of the reference (write_frontier_gzip_csv,
 * src/pmdd/util/output_utils.cpp:87-152): one point per line, objectives as decimal
 * integers separated by ',', '\n' line ends, gzip-compressed (here by zlib in process
 * instead of a `gzip -c` child per file; the decompressed bytes are the reference's).
 * `points` holds num_points*nobjs values of elem_bytes (4: int32, 8: int64) bytes, as in
 * pmdd_frontier; with `sort` they are written ascending lexicographically, as the
 * reference's main sorts before writing (src/pmdd/main.cpp:267).  The caller's array is
 * not modified.  Returns PMDD_OK, PMDD_ERR_INVALID or PMDD_ERR_IO (text in err). */
int pmdd_write_frontier_csv_gz(const void *points, int64_t num_points, int32_t nobjs, int32_t elem_bytes,
                               int32_t sort, const char *path, char *err, size_t errlen);

/* Asynchronous writer: a pool of `threads` writer threads (<= 0: up to 4) fed by a queue,
 * so that a serving loop hands each result over and goes on.  No counterpart in the
 * reference, which writes from the enumerating thread. */
typedef struct pmdd_writer pmdd_writer;
pmdd_writer *pmdd_writer_create(int32_t threads, char *err, size_t errlen);
/* Queues one result: the frontier (copied now; sorted, then written to csv_gz_path as
 * above) and/or one JSONL record (a single line without '\n', appended to jsonl_path as
 * the reference's write_stats_jsonl appends, output_utils.cpp:154-300).  Either path may
 * be NULL or empty, not both.  Returns PMDD_OK or PMDD_ERR_INVALID; never blocks on I/O. */
int pmdd_writer_submit(pmdd_writer *w, const void *points, int64_t num_points, int32_t nobjs, int32_t elem_bytes,
                       const char *csv_gz_path, const char *jsonl_path, const char *jsonl_record);
/* Results queued or being written. */
int64_t pmdd_writer_pending(pmdd_writer *w);
/* Blocks until everything queued so far is written.  Returns the number of results
 * that failed since the last flush (first failure's text in err) and, in *written, the
 * number written. */
int64_t pmdd_writer_flush(pmdd_writer *w, int64_t *written, char *err, size_t errlen);
/* Writes what is queued, then stops the threads and frees the writer. */
void pmdd_writer_destroy(pmdd_writer *w);

#ifdef __cplusplus
}
#endif

#endif /* PMDD_HOST_H_ */
