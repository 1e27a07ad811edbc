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

#ifdef __cplusplus
}
#endif

#endif /* PMDD_HOST_H_ */
