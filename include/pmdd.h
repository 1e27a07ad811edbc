/*
 * pmdd.h -- C ABI of the B200 Pareto-frontier enumeration engine (libpmdd_gpu.so).
 *
 * This is the drop-in boundary for the GPU enumeration seam of rahulptel/PMDD.  The
 * reference exposes four C++ free functions that take its pointer-based BDD / MDD
 * objects (src/pmdd/enum/gpu/cuda_wrappers.hpp:11-21):
 *
 *   topdown_cuda_enumerate(BDD*, maximization, problem_type, state_dominance,
 *                          EnumerationStats*, std::string* reason, max_cand)
 *   topdown_mdd_cuda_enumerate(MDD*, EnumerationStats*, std::string*, max_cand)
 *   coupled_cuda_enumerate(MDD*, EnumerationStats*, std::string*, max_cand, max_prod)
 *   coupled_bdd_cuda_enumerate(BDD*, maximization, problem_type, state_dominance,
 *                              EnumerationStats*, std::string*, max_cand, max_prod)
 *
 * All four collapse to pmdd_enumerate() over a flat, layered DD (pmdd_dd below): the
 * reference's packing step (src/pmdd/enum/gpu/enum.cu:85-158, :438-593) becomes the
 * caller's job, done once, in plain arrays.  Only POD types cross this boundary.
 *
 * Error behaviour mirrors the reference seam: a failed call returns a non-zero status
 * and writes a one-line reason into `err` (the reference returns NULL and sets
 * *reason, src/pmdd/enum/gpu/enum_types.cuh:76-81); it never falls back to the CPU.
 */
#ifndef PMDD_H_
#define PMDD_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
enum pmdd_status {
    PMDD_OK = 0,
    PMDD_ERR_INVALID = 1,        /* malformed DD or options */
    PMDD_ERR_CUDA = 2,           /* CUDA runtime error (text in err) */
    PMDD_ERR_OOM = 3,            /* request cannot fit the device / server budget */
    PMDD_ERR_CAND_OVERFLOW = 4,  /* a single destination exceeds what one pass can hold */
    PMDD_ERR_TIMEOUT = 5,        /* a bounded device wait gave up */
    PMDD_ERR_INTERNAL = 6,       /* device-side consistency check failed */
    PMDD_ERR_CANCELLED = 7,      /* request cancelled before completion */
    PMDD_ERR_NO_DEVICE = 8,      /* no CUDA device / extension not usable */
    PMDD_ERR_RANGE = 9,          /* objective sums exceed the supported integer range, or a
                                    size exceeds a fixed limit (pmdd_pareto_filter_noalloc) */
    PMDD_ERR_IO = 10             /* an output file could not be written (pmdd_host.h writers) */
};

/* ------------------------------------------------------------ the flat DD format
 * Nodes are numbered 0..num_nodes-1 layer by layer; layer l holds nodes
 * [layer_offsets[l], layer_offsets[l+1]).  Layer 0 holds exactly one node (the root)
 * and the last layer exactly one node (the terminal).
 *
 * Arcs are stored once, grouped by their HEAD (destination) node: the incoming arcs
 * of node v are [in_arc_offsets[v], in_arc_offsets[v+1]); arc a runs from node
 * arc_src[a] (which must lie in the layer just above v) to v and carries the weight
 * vector weights[arc_weight[a]*nobjs .. +nobjs).  A BDD uses weight row 0 for every
 * 0-arc (the zero vector) and one further row per layer for its 1-arcs, so an arc's
 * type is (arc_weight[a] != 0); a TSP MDD uses row 0 for the arc into the fixed first
 * city and row 1 + i*n + j for the move from city i to city j.  The bottom-up
 * direction (outgoing arcs) is derived by the engine.
 *
 * min_weight (optional, may be NULL): knapsack used-capacity lower bound per node,
 * required only for state_dominance > 0 with problem_type 1 (the reference's
 * Node::min_weight, src/pmdd/bdd/knapsack_bdd.cpp:123-150).
 *
 * node_state (optional, may be NULL): set-packing state per node, state_words 64-bit
 * words each, bit v of word v/64 set iff vertex v may still be chosen below the node
 * (the reference's Node::setpack_state, src/pmdd/bdd/indepset_bdd.cpp:79-135);
 * required only for state_dominance > 0 with problem_type 2.  state_words is 0 when
 * node_state is NULL.
 */
typedef struct pmdd_dd {
    int32_t nobjs;        /* objectives per point, 1..8 */
    int32_t num_layers;   /* >= 2 */
    int32_t num_nodes;
    int32_t num_arcs;
    int32_t num_weights;  /* rows in `weights` */
    const int32_t *layer_offsets;   /* [num_layers+1] */
    const int32_t *in_arc_offsets;  /* [num_nodes+1] */
    const int32_t *arc_src;         /* [num_arcs] */
    const int32_t *arc_weight;      /* [num_arcs] row index into weights */
    const int32_t *weights;         /* [num_weights*nobjs] */
    const int32_t *min_weight;      /* [num_nodes] or NULL */
    const uint64_t *node_state;     /* [num_nodes*state_words] or NULL */
    int32_t state_words;
    int32_t reserved;               /* must be 0 */
} pmdd_dd;

/* ------------------------------------------------------------------- options */
typedef struct pmdd_options {
    int32_t method;           /* 1 = top-down, 3 = dynamic layer cutset (coupled) */
    int32_t problem_type;     /* 1 knapsack, 2 set packing, 3 TSP */
    int32_t state_dominance;  /* > 0: label pruning between nodes of a top-down layer
                                 (problem 1 by min_weight, problem 2 by state subsets;
                                 methods 1 and 3; ignored for problem 3) */
    int32_t maximization;     /* must be 1 (the reference's main always maximises) */
    int64_t max_cand;         /* candidate points per expansion pass (--max-cand, 20M) */
    int64_t max_prod;         /* pair products per coupling pass (--max-prod, 625K) */
    int32_t device;           /* CUDA device ordinal (the reference always uses 0) */
    int32_t reserved;
} pmdd_options;

/* Fills `o` with the reference CLI defaults (method 1, max_cand 20M, max_prod 625K). */
void pmdd_options_default(pmdd_options *o);

/* -------------------------------------------------------------------- output */
typedef struct pmdd_frontier {
    int32_t nobjs;
    int32_t elem_bytes;   /* 4: int32 points, 8: int64 points (wide objective bound) */
    int64_t num_points;
    void *points;         /* num_points*nobjs values, unsorted; free with pmdd_frontier_free */
} pmdd_frontier;

void pmdd_frontier_free(pmdd_frontier *f);

/* Run statistics: the GPU-side subset of the reference's EnumerationStats
 * (src/pmdd/util/stats.hpp:18-85), same names and meaning. */
typedef struct pmdd_stats {
    double wall_pack_transfer_s;
    double wall_join_s;
    double kernel_expand_td_s;
    double kernel_dominance_s;
    double kernel_total_s;
    int64_t gpu_mem_peak_used_bytes;
    int64_t gpu_mem_peak_reserved_bytes;
    int64_t work_candidates_total;
    int64_t work_candidates_peak;
    int64_t work_frontier_survivors_total;
    int64_t work_frontier_peak_points;
    int64_t work_join_products_total;
    int64_t dominance_filtered_total;
    int32_t layer_coupling;
    int32_t layers_td;
    int32_t layers_bu;
    int32_t cutset_size;
    int64_t gpu_launches;   /* kernels this call launched */
    double device_elapsed_s;  /* CUDA-event time on the engine stream, first to last op of the call */
    int64_t work_tile_candidates_total;  /* candidates filtered in shared-memory tiles */
    int64_t work_tile_survivors_total;   /* survivors the tile kernel wrote */
    int64_t tile_launches;               /* expand+filter tile kernels this call launched */
    int64_t work_stair_candidates_total; /* three objectives: candidates of destinations filtered by a
                                            staircase warp (tiles above the pairwise limit, and
                                            oversized destinations with sorted runs) */
    int64_t work_chained_layers;         /* layers expanded by chained steps (several layers between two
                                            host read-backs, for steps with few candidates) */
} pmdd_stats;

/* ------------------------------------------------------------ one-shot entry
 * Replaces all four reference seam functions.  Synchronous; blocks until the
 * frontier is on the host.  Thread-safe across different devices. */
int pmdd_enumerate(const pmdd_dd *dd, const pmdd_options *opts, pmdd_frontier *out,
                   pmdd_stats *stats, char *err, size_t errlen);

/* Batched entry: enumerates `count` independent DDs in shared launches (one launch
 * per phase per step covers every instance still running).  outs[i] / status[i]
 * receive each instance's frontier and status; stats (optional) aggregates. */
int pmdd_enumerate_batch(const pmdd_dd *dds, int32_t count, const pmdd_options *opts,
                         pmdd_frontier *outs, int32_t *status, pmdd_stats *stats,
                         char *err, size_t errlen);

/* Standalone Pareto filter of one point set on the GPU: writes the maximal points of
 * points[0..num_points) under componentwise >= (one copy of each group of equal
 * points) into `out` (capacity num_points*nobjs) and their count into *out_points.
 * The merge rule of the reference's ParetoFrontier::merge
 * (src/pmdd/enum/pareto_frontier.hpp:237-303) applied to a whole set at once; output
 * order is unspecified.  Host buffers; num_points < 2^31, nobjs 1..8. */
int pmdd_pareto_filter(const int32_t *points, int64_t num_points, int32_t nobjs, int32_t *out, int64_t *out_points,
                       int32_t device, char *err, size_t errlen);

/* Allocation-free variant of pmdd_pareto_filter, for callers that cannot allocate
 * device memory: libraries running beside a framework allocator that has reserved the
 * device's memory, and services that forbid cudaMalloc / cudaFree after start-up
 * because those calls can synchronise the device.  No counterpart in the reference.
 * Device buffers: d_points (num_points*nobjs) in, d_out (same capacity) out;
 * *out_points (host) receives the count; `stream` is a cudaStream_t (NULL: the
 * default stream).  Scratch comes from a fixed device array of about 9.4 MB that every
 * device loading this library holds until exit: at most 131072 points of at most 8
 * objectives per call (larger sets return PMDD_ERR_RANGE).  Calls share that array, so
 * calls that overlap on the GPU race; serialise them.  The first call on a device
 * looks up the array's address and should happen before any stream capture.
 * Allocates nothing; copies the count to the host and synchronises `stream` before
 * returning. */
int pmdd_pareto_filter_noalloc(const int32_t *d_points, int64_t num_points, int32_t nobjs, int32_t *d_out,
                               int64_t *out_points, void *stream, char *err, size_t errlen);

/* Device-resident DD set: uploads `count` DDs once (with both arc directions) into
 * the device engine's memory; pmdd_resident_enumerate then runs a batch over them
 * with no host->device DD traffic.  Frees with pmdd_resident_free. */
typedef struct pmdd_resident pmdd_resident;
pmdd_resident *pmdd_resident_upload(const pmdd_dd *dds, int32_t count, int32_t device, char *err, size_t errlen);
int pmdd_resident_enumerate(pmdd_resident *res, const pmdd_options *opts, pmdd_frontier *outs, int32_t *status,
                            pmdd_stats *stats, char *err, size_t errlen);
/* Sum of the uploaded DDs' device bytes. */
int64_t pmdd_resident_bytes(const pmdd_resident *res);
void pmdd_resident_free(pmdd_resident *res);

/* 0/1 knapsack instance, one constraint (the reference's KnapsackInstance,
 * src/pmdd/instances/knapsack_instance.cpp:17-47, with n_cons = 1). */
typedef struct pmdd_knapsack {
    int32_t n;                 /* items, >= 1 */
    int32_t nobjs;             /* objectives used, 1..8 */
    const int32_t *profits;    /* [nobjs][n], objective-major as in the file */
    const int32_t *weights;    /* [n], >= 0 */
    int32_t capacity;          /* 0 .. 2^24 */
    int32_t reserved;          /* must be 0 */
} pmdd_knapsack;

/* Builds the exact knapsack BDDs of `count` instances on the device -- the DD the host
 * constructor makes (pmdd_build_from_text, problem type 1: the reference's
 * KnapsackBDDConstructor::generate_exact, two BDDAlg::reduce passes and
 * update_node_weights, src/pmdd/bdd/knapsack_bdd.cpp:10-150, src/pmdd/main.cpp:120-153),
 * array for array -- and keeps them resident like pmdd_resident_upload: only the item
 * weights and profits cross the bus.  No counterpart in the reference, which builds its
 * DDs on the CPU. */
pmdd_resident *pmdd_resident_build_knapsack(const pmdd_knapsack *instances, int32_t count, int32_t device, char *err,
                                            size_t errlen);

/* TSP instance: n cities, one cost matrix per objective (the reference's TSPInstance,
 * src/pmdd/instances/tsp_instance.cpp:11-39; arc weights are the negated costs). */
typedef struct pmdd_tsp {
    int32_t n;                 /* cities, 2..20 */
    int32_t nobjs;             /* objectives used, 1..8 */
    const int32_t *cost;       /* [nobjs][n][n], row-major per objective */
} pmdd_tsp;

/* TSP MDDs on the device: every MDD of n cities has the same layers, nodes and arcs (all
 * (visited set, last city) states are reachable; src/pmdd/mdd/tsp_mdd.cpp:21-196), so the
 * engine builds that structure once per n on the GPU and keeps it, and each instance
 * adds only its weight table.  The DDs equal the host constructor's (problem type 3)
 * array for array.  No counterpart in the reference. */
pmdd_resident *pmdd_resident_build_tsp(const pmdd_tsp *instances, int32_t count, int32_t device, char *err,
                                       size_t errlen);

/* Shape of DD i of a resident set: shape = {nobjs, num_layers, num_nodes, num_arcs,
 * num_weights}; widths = {original width, original nodes, reduced width, reduced nodes}
 * for device-built DDs, -1 otherwise (either pointer may be NULL). */
int pmdd_resident_dd_shape(const pmdd_resident *res, int32_t i, int32_t *shape, int64_t *widths);
/* Copies DD i's arrays (pmdd_dd layout, sized by pmdd_resident_dd_shape) to the host;
 * min_weight may be NULL (it is filled only for DDs that carry it). */
int pmdd_resident_dd_copy(pmdd_resident *res, int32_t i, int32_t *layer_offsets, int32_t *in_arc_offsets,
                          int32_t *arc_src, int32_t *arc_weight, int32_t *weights, int32_t *min_weight, char *err,
                          size_t errlen);

/* ---------------------------------------------------------------- serving
 * A device-resident request loop with continuous batching: submitted requests are
 * admitted as slots and HBM budget free up; every admitted request advances one
 * layer per engine step, sharing each launch with the others.  No counterpart in the
 * reference, which enumerates one instance per process (src/pmdd/main.cpp:67-467).
 *
 * Admission: a request is admitted when its predicted peak device footprint fits
 * beside what the running requests hold and are predicted to grow by.  The prediction
 * is the DD's device bytes plus two layers of frontier slots at the predicted largest
 * layer (the larger of the layers the request has shown, its next layer once counted --
 * exact -- and a per-(problem type, objectives, method) ratio of largest layer to DD
 * arcs learned from finished requests), per-layer bookkeeping, and for method 3 the
 * other side's frontier and the coupling block.  A request that does not fit waits;
 * smaller ones behind it may pass until it has been passed over 32 times.  A request
 * whose DD alone exceeds the budget finishes at once with PMDD_ERR_OOM; one that runs
 * out of memory while running finishes with PMDD_ERR_OOM while the others continue
 * (the reference's GPU path returns NULL with a reason and the CLI exits,
 * src/pmdd/main.cpp:338-345, or lets a Thrust allocation exception escape).
 *
 * Lanes: a server runs two engines.  Requests whose DD has at most 2^17 arcs
 * (PMDD_SERVER_HEAVY_ARCS) go to the light lane, on the device's highest-priority
 * stream, which pmdd_server_run steps in the caller's thread; larger ones go to the
 * heavy lane, which a worker thread of the server steps on its own while it has work,
 * so small requests neither wait for a large one's steps nor queue behind its blocks.
 * The light lane gets a quarter of the budget (at least half of it, up to 512 MB), the
 * heavy lane the rest; max_slots applies to each lane.  A budget below 512 MB, or
 * PMDD_SERVER_LANES=1: one engine with the whole budget, stepped by the caller.  A server's functions are called from one
 * thread at a time. */
typedef struct pmdd_server pmdd_server;

typedef struct pmdd_result {
    uint64_t req_id;
    int32_t status;
    int32_t reserved;
    pmdd_frontier frontier;   /* owned by the caller after poll; pmdd_frontier_free */
    double submit_s;          /* host monotonic clock, seconds */
    double admit_s;
    double finish_s;
    char error[160];
} pmdd_result;

pmdd_server *pmdd_server_create(int32_t device, int64_t budget_bytes, int32_t max_slots,
                                char *err, size_t errlen);
/* Copies the DD; the caller's buffers may be reused immediately. */
int pmdd_server_submit(pmdd_server *srv, const pmdd_dd *dd, const pmdd_options *opts,
                       uint64_t req_id);
/* Submits a TSP request by its cost matrices: the server uses its shared n-city MDD
 * structure (built on the device on first use) and uploads only the weight table. */
int pmdd_server_submit_tsp(pmdd_server *srv, const pmdd_tsp *inst, const pmdd_options *opts, uint64_t req_id);
/* Builds the shared n-city MDD structure now (in every lane) instead of at the first
 * request of that size, and returns when it is built.  No counterpart in the reference. */
int pmdd_server_prepare_tsp(pmdd_server *srv, int32_t n);
/* Runs light-lane steps until at least one request completes (in either lane), max_steps
 * light-lane steps have run (0: no limit) or nothing is pending; while the light lane
 * is idle it waits up to 2 ms at a time for the heavy lane.  Returns the number of
 * results now waiting, or -1 after a CUDA failure of either lane. */
int pmdd_server_run(pmdd_server *srv, int32_t max_steps);
/* Non-blocking: 1 and fills *out if a finished result is available, else 0. */
int pmdd_server_poll(pmdd_server *srv, pmdd_result *out);
int pmdd_server_cancel(pmdd_server *srv, uint64_t req_id);
/* Requests submitted and not yet reported by pmdd_server_run (queued, running, or
 * finished in the heavy lane while the caller was away). */
int pmdd_server_pending(const pmdd_server *srv);

/* Serving counters and memory figures since the server was created.  `rejected`:
 * finished with an error before admission (DD above the budget, invalid request);
 * `failed`: finished with an error after admission (cancellations apart). */
typedef struct pmdd_server_info {
    int64_t submitted, admitted, completed, failed, rejected, cancelled;
    int32_t queued, running;            /* now */
    int32_t queued_peak, running_peak;  /* largest seen at an admission pass */
    int64_t budget_bytes;               /* the engine arena's budget */
    int64_t used_bytes;                 /* arena bytes in use now */
    int64_t peak_used_bytes;            /* arena high-water mark */
    int64_t reserved_growth_bytes;      /* predicted growth of the running requests */
    int64_t injected_alloc_failures;    /* allocations failed by the test hook below */
} pmdd_server_info;
int pmdd_server_get_info(const pmdd_server *srv, pmdd_server_info *out);

/* Test hook for the failure paths: after `after` more device-memory allocations of
 * this server's engine, the next `count` fail as if the device were out of memory.
 * Running requests that cannot get memory finish with PMDD_ERR_OOM; the server keeps
 * serving the others.  No counterpart in the reference. */
int pmdd_server_inject_alloc_failures(pmdd_server *srv, int64_t after, int64_t count);
void pmdd_server_destroy(pmdd_server *srv);

/* --------------------------------------------------------------- utilities */
const char *pmdd_version(void);
/* Number of kernels this library has launched in this process (all calls). */
int64_t pmdd_launch_count(void);
/* The oversized-destination crossover (candidates from which a destination is filtered
 * by the GPU-wide pass rather than one sort-filter-skyline block) that the tuning file
 * at `path` holds for (nobjs, problem_type), or 0 if it holds none (engines then use their
 * built-in crossover, 1025: every destination too large for a tile).  path NULL: the file
 * engines read at start-up (PMDD_TUNING_FILE, else the per-user cache written by
 * pmdd_b200.autotune).  No counterpart in the reference, which has one filter path. */
int64_t pmdd_tuned_mark_min(const char *path, int32_t nobjs, int32_t problem_type);
/* The three-objective crossover between the pairwise check and the staircase warp
 * (destinations of at most this many candidates are checked pairwise) that the tuning
 * file holds for (nobjs, problem_type), or -1 if none (engines then use 48).  Same file
 * rules as pmdd_tuned_mark_min.  No counterpart in the reference, whose filter is
 * pairwise at every size (src/pmdd/enum/gpu/topdown.cu:163-240). */
int64_t pmdd_tuned_lex_pair_max(const char *path, int32_t nobjs, int32_t problem_type);
/* The largest tile window (a tile's destinations start within this many candidates) the
 * tuning file holds for (nobjs, problem_type), or -1 if none (engines then use 1024; a
 * step uses its candidates over six tiles per SM, between 128 and this).  Same file rules
 * as pmdd_tuned_mark_min.  No counterpart in the reference. */
int64_t pmdd_tuned_tile_window_max(const char *path, int32_t nobjs, int32_t problem_type);

#ifdef __cplusplus
}
#endif

#endif /* PMDD_H_ */
