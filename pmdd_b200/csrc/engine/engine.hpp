// Host side of the B200 enumeration engine: a device-memory arena, per-request device
// state, and the step scheduler that advances every admitted request by one layer per
// step in shared launches (continuous batching).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "couple.cuh"
#include "statedom.cuh"
#include "kernels.cuh"
#include "pmdd.h"

namespace pmdd {

double now_s();

// Kernels launched by every engine of this process.
extern std::atomic<int64_t> g_total_launches;

// First-fit allocator over device memory taken in a few large cudaMalloc chunks, the
// first of `initial` bytes at start-up and more (doubling, at most 16 GB at a time) when
// a request does not fit, up to `budget` in all.  Bookkeeping is host-side; every kernel
// of the engine runs on one stream, so memory released on the host may be handed out
// again immediately (later work on the stream runs after earlier work).  Free blocks
// never merge across chunks.
class Arena {
  public:
    ~Arena();
    bool init(size_t budget, size_t initial, std::string *err);
    void *alloc(size_t bytes);
    void release(void *p);
    size_t capacity() const { return cap_; }       // the budget
    size_t reserved() const { return reserved_; }  // device memory taken so far
    size_t used() const { return used_; }
    size_t peak() const { return peak_; }
    void reset_peak() { peak_ = used_; }
    double grow_seconds() const { return grow_s_; }  // host time spent in cudaMalloc
    // Fault injection for tests of the failure paths: after `after` more allocation
    // calls, the next `count` calls fail as if the device were out of memory.
    void inject_failures(int64_t after, int64_t count) {
        inj_after_ = after;
        inj_count_ = count;
    }
    int64_t injected_failures() const { return injected_; }

  private:
    bool grow(size_t at_least);
    int64_t inj_after_ = 0, inj_count_ = 0, injected_ = 0;
    size_t cap_ = 0, reserved_ = 0, used_ = 0, peak_ = 0;
    double grow_s_ = 0;
    std::map<uintptr_t, size_t> chunks_;            // cudaMalloc base -> bytes
    std::map<uintptr_t, size_t> free_;              // address -> bytes (free blocks, for coalescing)
    std::set<std::pair<size_t, uintptr_t>> by_size_;  // the same blocks by (bytes, address): best fit
    std::unordered_map<uintptr_t, size_t> live_;    // address -> bytes
    void add_free(uintptr_t a, size_t bytes);
    void drop_free(std::map<uintptr_t, size_t>::iterator it);
};

// Frontiers of one direction at its current layer, in slot layout: node i's points
// live at pts[off[i] .. off[i]+size[i]) (D values each).
struct Side {
    int layer = -1;
    void *pts = nullptr;
    int64_t *off = nullptr;
    int32_t *size = nullptr;
    uint8_t *sorted = nullptr;     // per node: frontier in descending lexicographic order (in the size block)
    // counts for the next layer in this direction
    bool counted = false;
    int64_t *arc_off = nullptr;
    int64_t *big_list = nullptr;
    dev::CountResult res{};
    int64_t score = 0;
    int64_t slot_points = 0;       // candidate slots of the current frontier (its memory)
};

// The shared part of every TSP MDD of n cities (tspbuild.cuh): all arrays but the
// weight table, with the bottom-up CSR, in one device block owned by the engine.
struct TspStructure {
    int n = 0;
    unsigned char *mem = nullptr;
    std::vector<int32_t> layer_off, arc_at;  // host copies, L+1 each
    int32_t N = 0, A = 0;
    const int32_t *in_off = nullptr, *arc_src = nullptr, *arc_w = nullptr;
    int32_t *out_off = nullptr, *out_head = nullptr, *out_w = nullptr, *cursor = nullptr;
};

struct Instance {
    enum Phase { QUEUED, RUNNING, COUPLING, DONE };
    uint64_t id = 0;
    pmdd_options opts{};
    int d = 0;
    bool wide = false;
    int32_t L = 0, N = 0, A = 0, K = 0;
    std::vector<int32_t> layer_off;     // L+1
    std::vector<int32_t> arc_at_layer;  // L+1: in-arcs of layers < l
    std::vector<unsigned char> blob;    // packed DD arrays, uploaded at admission
    const unsigned char *blob_src = nullptr;  // packed arrays in the engine's pinned staging (instead of blob)
    size_t off_layer = 0, off_in = 0, off_src = 0, off_w = 0, off_weights = 0, off_minw = 0, blob_bytes = 0;
    // state dominance (sd_kind 1: knapsack, 2: set packing; 0: none).  sd_order holds, per
    // layer, the layer-local node ids by min_weight descending (kind 1) or by state size
    // ascending (kind 2), ties by id; packed into the blob at off_sdord when present.
    // Kind 2 also packs sd_next (per order position: the order range [begin, end) of the
    // next non-empty state-size bucket, empty when the node takes no partner) at
    // off_sdnext and the DD's node states (state_words words per node) at off_state.
    std::vector<int32_t> sd_order;
    std::vector<int32_t> sd_next;
    size_t off_sdord = 0, off_sdnext = 0, off_state = 0;
    int32_t state_words = 0;
    int sd_kind = 0;
    bool has_sd_order = false;
    const int32_t *d_sd_order = nullptr;
    const int32_t *d_sd_next = nullptr;
    const uint64_t *d_state = nullptr;
    size_t dev_bytes = 0;               // blob + out-arc CSR
    // device DD
    unsigned char *dd = nullptr;
    const int32_t *d_in_off = nullptr, *d_arc_src = nullptr, *d_arc_w = nullptr, *d_weights = nullptr;
    int32_t *d_out_off = nullptr, *d_out_head = nullptr, *d_out_w = nullptr, *d_cursor = nullptr;
    Side td, bu;
    Phase phase = QUEUED;
    // coupling state
    void *cu_mem = nullptr;             // one block: U | U_alt | filter scratch (couple_bytes)
    void *cu_U = nullptr;               // current running frontier (+ this round's survivors)
    void *cu_U_alt = nullptr;           // receives the next running frontier
    void *cu_p2 = nullptr, *cu_sv = nullptr;
    int32_t *cu_i2 = nullptr, *cu_si = nullptr, *cu_hist = nullptr;
    int64_t *cu_ctr = nullptr;
    int64_t cu_ucap = 0;
    int couple_rounds = 0;
    // outcome
    int status = PMDD_OK;
    std::string error;
    std::vector<unsigned char> result;  // num_points * d * elem
    int64_t result_n = 0;
    pmdd_stats stats{};
    double submit_s = 0, admit_s = 0, finish_s = 0;
    // admission: the exact minimum (the DD's device copy) and what the footprint
    // prediction uses -- the largest layers seen so far and the DD's shape
    int64_t min_bytes = 0;
    int64_t peak_cand = 0;              // largest expansion (candidates) so far, either side
    int64_t max_layer_arcs = 0, max_layer_nodes = 0;
    int32_t skipped = 0;                // admission passes this request was passed over
    int32_t chain_len = 0;              // layers its next chained step tries (0: the engine's base)
    int32_t chain_skip = 0;             // eligible steps to pass over before the next chain
    bool external_dd = false;           // DD already resident (owned by a pmdd_resident set)
    const TspStructure *tsp = nullptr;  // TSP MDD: structure shared, I.dd holds the weight table only
    bool with_out_csr = false;          // device copy carries the bottom-up CSR

    size_t elem() const { return wide ? 8 : 4; }
    int32_t nodes_in(int l) const { return layer_off[l + 1] - layer_off[l]; }
};

// Validates a flat DD and lays it out in an Instance (host side only).  The device copy
// gets the bottom-up CSR when the method needs it or `with_out_csr` asks for it, and the
// state-dominance data when the DD carries it (min_weight for knapsack, node_state for
// set packing) and either the options ask for state dominance or `with_out_csr` is set
// (resident sets, which serve any options).  With
// `pack` the arrays are also copied into inst->blob; without it the caller packs them
// later with pack_instance (e.g. straight into pinned staging memory).
int prepare_instance(const pmdd_dd &dd, const pmdd_options &opts, uint64_t id, Instance *inst, std::string *err,
                     bool with_out_csr = false, bool pack = true);
// Writes the DD arrays of a prepared instance into dst (inst.blob_bytes bytes, laid out
// at the instance's offsets; the alignment gaps are left as they are).
void pack_instance(const pmdd_dd &dd, const Instance &inst, unsigned char *dst);

// Host metadata and blob layout of a knapsack BDD built on the device (kpbuild.cu): layer
// offsets and the incoming-arc offsets at layer starts (both L+1), K weight rows; the
// blob holds the pmdd_dd arrays, min_weight and the min_weight order, then the
// bottom-up CSR.
void layout_built_knapsack(Instance *I, int d, bool wide, const std::vector<int32_t> &layer_off,
                           const std::vector<int32_t> &arc_at_layer, int32_t K);

// A TSP request over a shared structure: host metadata and the blob, which is the weight
// table alone (row 0 zero, row 1 + i*n + j = -cost[o][i][j]; `cost` is [nobjs][n][n]).
// The path-sum bound follows prepare_instance's rule layer by layer.
void prepare_tsp_instance(const TspStructure &S, int nobjs, const int32_t *cost, const pmdd_options &opts,
                          uint64_t id, Instance *I);

// Tuned oversized-path crossovers, (objectives, problem type) -> big_mark_min, from the
// tuning file pmdd_b200.autotune writes (see Engine::mark_min_for); empty when absent.
std::string default_tuning_path();
std::map<std::pair<int, int>, int64_t> read_tuning(const std::string &path, const char *key = "big_mark_min");

// Runs fn(i) for i in [0, n) on up to `threads` host threads (PMDD_HOST_THREADS caps
// the default, which is the hardware concurrency, at most 32).
void parallel_for(int64_t n, int threads, const std::function<void(int64_t)> &fn);
int host_threads();

// Accumulated kernel time of an engine (seconds, CUDA events on its stream): the fused
// expand+filter tiles, the oversized-destination path, and everything else (counting,
// coupling, DD preparation).
struct KernelTimes {
    double expand = 0, big = 0, rest = 0;
    int64_t tile_launches = 0;
};

class Engine {
  public:
    // stream_priority: the engine stream's CUDA priority (0: default; lower numbers are
    // higher priorities, as cudaDeviceGetStreamPriorityRange gives them).
    Engine(int device, int64_t budget_bytes, int max_slots, int stream_priority = 0);
    ~Engine();
    bool ok() const { return ok_; }
    const std::string &error() const { return error_; }

    // Takes ownership; the instance waits in the queue until it fits.
    void submit(std::unique_ptr<Instance> inst);
    // One engine step; returns the number of requests that finished during it, or -1
    // on an engine-wide CUDA failure.
    int step();
    bool idle() const { return queued_.empty() && active_.empty(); }
    size_t queued() const { return queued_.size(); }
    size_t running() const { return active_.size(); }
    std::deque<std::unique_ptr<Instance>> &finished() { return finished_; }
    // Hands a request that failed before reaching the queue (its status and error set)
    // straight to the finished list, counting it as rejected.
    void finish_rejected(std::unique_ptr<Instance> I) {
        I->phase = Instance::DONE;
        I->finish_s = now_s();
        counters_.rejected++;
        finished_.push_back(std::move(I));
    }
    bool cancel(uint64_t id);
    int64_t launches() const { return launches_; }
    const Arena &arena() const { return arena_; }
    // Restarts the arena's high-water mark (gpu_mem_peak_used_bytes of later requests).
    void reset_mem_peak() { arena_.reset_peak(); }
    int device() const { return device_; }
    cudaStream_t stream() const { return stream_; }
    // Serving counters (requests since the engine started).
    struct Counters {
        int64_t admitted = 0, rejected = 0, completed = 0, failed = 0, cancelled = 0;
        int64_t queued_peak = 0, running_peak = 0;
    };
    const Counters &counters() const { return counters_; }
    // Device bytes the admission model predicts for the request at its peak (its DD, two
    // layers of frontier slots at the predicted largest layer, per-layer bookkeeping,
    // and for method 3 the other side's frontier and the coupling block), and the
    // bytes it holds now.
    int64_t predicted_bytes(const Instance &I) const;
    int64_t current_bytes(const Instance &I) const;
    // Predicted growth of the running requests (sum of predicted minus current bytes).
    int64_t reserved_growth() const;
    void inject_alloc_failures(int64_t after, int64_t count) { arena_.inject_failures(after, count); }
    KernelTimes kernel_times() const { return ktimes_; }
    // Device copy of a prepared request's DD (with the bottom-up CSR) that stays in
    // the arena until release_dd(); requests then share it via external_dd.
    bool upload_dd(Instance &I);
    // Makes this engine's device current on the calling thread (a thread may drive the
    // engines of several devices); every entry below that launches work calls it.
    bool make_current();
    // Device pointers of a DD whose arrays are in I.dd (uploaded or built on the device),
    // and its bottom-up CSR when the instance carries one.
    bool bind_dd(Instance &I);
    // The structure of n-city TSP MDDs on this engine's device, built on first use and
    // kept for the engine's life; nullptr (with *err) if it cannot be built.
    const TspStructure *tsp_structure(int n, std::string *err);
    void release_dd(Instance &I);
    // Pinned host memory for packing DD uploads (grow-only, kept across calls); nullptr
    // when it cannot be had.  Contents must stay untouched until the uploads that read
    // them have completed on the stream.
    unsigned char *staging(size_t bytes) {
        return h_stage_.reserve(bytes) ? static_cast<unsigned char *>(h_stage_.p) : nullptr;
    }
    // Raw arena memory for standalone operations run on this engine's stream.
    void *alloc(size_t bytes) { return arena_.alloc(bytes); }
    void release(void *p) { arena_.release(p); }
    void count_launches(int64_t n) {
        launches_ += n;
        g_total_launches += n;
    }

  private:
    struct Pinned {
        void *p = nullptr;
        size_t cap = 0;
        bool reserve(size_t bytes);
        ~Pinned();
    };
    bool admit(Instance &I);
    // (Re)allocates the coupling block for capacity ucap and points U, U_alt and the
    // filter scratch into it; false if it does not fit (old block kept).
    bool carve_couple(Instance &I, int64_t ucap);
    void fail(Instance &I, int status, const std::string &msg);
    void release_instance(Instance &I);
    void release_side(Side &s);
    bool cuda_ok(cudaError_t e, const char *what);
    void *scratch(size_t bytes);  // step-lifetime device memory

    bool ok_ = false;
    std::string error_;
    int device_ = 0;
    int sms_ = 148;
    int max_slots_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev_[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // per-step phase timing, reused
    std::map<int, std::unique_ptr<TspStructure>> tsp_cache_;
    Arena arena_;
    std::deque<std::unique_ptr<Instance>> queued_;
    std::vector<std::unique_ptr<Instance>> active_;
    std::deque<std::unique_ptr<Instance>> finished_;
    std::vector<void *> step_scratch_;
    Pinned h_desc_, h_summary_, h_init_, h_stage_;
    Pinned h_results_;  // the frontiers of the requests a step finishes, fetched together
    static constexpr size_t kSeedTemplate = 256, kSeedBytes = 80;  // seed side template in h_init_

    int64_t launches_ = 0;
    KernelTimes ktimes_;
    bool trace_ = false;  // PMDD_TRACE=1: one stderr line per step
    double last_post_us_ = 0;  // PMDD_TRACE: host time after the last step's synchronisation
    // Oversized destinations of at least mark_min_for(d, problem type) candidates are
    // filtered by the GPU-wide pivot/mark pass instead of one SFS block: PMDD_BIG_MARK_MIN
    // if set, else the tuned value for (d, problem type) from the tuning file, else
    // kSmallMax + 1 (every destination too large for a tile; SFS blocks then take only
    // destinations that leave the tiles for their arc count).
    int64_t mark_min_for(int d, int problem_type) const;
    void load_tuning();
    // Three-objective tiles in lexicographic order (tile_lex.cu): on unless PMDD_LEX_TILES=0.
    // Destinations of at most pair_max_for(d, problem type) candidates are checked
    // pairwise, larger ones by a staircase warp: PMDD_LEX_PAIR_MAX if set, else the tuned
    // value ("lex_pair_max" in the tuning file), else kDefaultPairMax.
    static constexpr int32_t kDefaultPairMax = 48;
    bool lex_tiles_ = true;
    // Four objectives with int32 points: tiles in sum order (tile_lex.cu) with
    // PMDD_SUM_TILES=1; by default the pairwise tile kernel, which measured faster (KP d=4
    // n=60: 29.6 against 31.2 ms, method 1).
    bool sum_tiles_ = false;
    bool lex_tiles_for(int d, bool wide) const {
        return dev::lex_tiles_cover(d, wide) && (d == 3 ? lex_tiles_ : sum_tiles_);
    }
    // Lexicographic tiles stage each arc's parent run into shared memory with one bulk copy
    // (cp.async.bulk on an mbarrier) instead of per-thread loads: PMDD_LEX_BULK=1 / 0.
    bool lex_bulk_ = false;
    // Oversized three-objective destinations of at most this many arc runs, all from
    // sorted frontiers, take the lexicographic path (big_lex.cu); the others the
    // SFS / pivot-mark passes.  PMDD_BIG_LEX_MAX_ARCS, 0 .. kBigLexMaxArcs.
    static constexpr int32_t kDefaultLexMaxArcs = 16;
    // Layer chaining (chain.cu): a request expanding by method 1 without state dominance
    // whose expansion in a step has at most chain_max_cand_ candidates goes on for more
    // layers in the same step, before the host reads back: chain_layers_ the first time,
    // then twice as many after a chain that ran to its end (up to kChainMaxLayers), or
    // one layer past where the last one stopped; beyond chain_layers_ only while the
    // request runs alone (PMDD_CHAIN_GROW=all: always).  Steps expanding more than
    // chain_max_requests_ requests chain none: their host work per request is already
    // shared, and the chained buffers would cost allocations per request.
    // PMDD_CHAIN_LAYERS (0: off), PMDD_CHAIN_MAX_CAND and PMDD_CHAIN_MAX_REQUESTS.
    int32_t chain_layers_ = 8;
    static constexpr int32_t kChainMaxLayers = 64;
    bool chain_grow_all_ = false;
    int64_t chain_max_requests_ = 128;
    // Pivots of a mark-path destination of n candidates (big.cu): about 4*sqrt(n) (1), or
    // n/64 with a floor of 512 (0, PMDD_PIVOT_RULE=n64).
    int32_t pivot_rule_ = 1;
    int64_t chain_max_cand_ = int64_t(1) << 17;
    int64_t chained_layers_total_ = 0;  // layers expanded by chained steps (statistics)
    int32_t lex_max_arcs_ = kDefaultLexMaxArcs;
    int32_t lex_pair_max_fixed_ = -1;
    std::map<std::pair<int, int>, int64_t> tuned_pair_max_;
    int32_t pair_max_for(int d, int problem_type) const;
    // Largest tile window (candidates a tile's destinations start within) for a family:
    // PMDD_TILE_WINDOW_MAX if set, else "tile_window_max" in the tuning file, else
    // kTileWindow; clamped to kTileWindowMin..kTileWindow.  A step's window is its
    // candidates over six tiles per SM, within kTileWindowMin and this.
    int64_t window_max_for(int d, int problem_type) const;
    int64_t window_max_fixed_ = 0;
    std::map<std::pair<int, int>, int64_t> tuned_window_max_;
    int64_t big_mark_min_fixed_ = 0;
    std::map<std::pair<int, int>, int64_t> tuned_mark_min_;
    // Footprint model: largest layer's candidates per DD arc, learned per (problem type,
    // objectives, method) from finished requests (a max that decays by 5 % per finish).
    std::map<std::tuple<int, int, int>, double> cand_per_arc_;
    void learn_footprint(const Instance &I);
    void record_finish(const Instance &I);
    Counters counters_;
};

}  // namespace pmdd
