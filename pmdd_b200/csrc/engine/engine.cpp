// Host side of the enumeration engine: arena, admission, and the step scheduler.
//
// One engine step advances every admitted request by one layer in one direction:
//   H2D of this step's descriptors
//   -> out-arc CSR for newly admitted method-3 requests
//   -> fused expand+filter tiles for all expanding requests (+ the oversized-destination path)
//   -> next-layer counting for every side that moved (and for new requests)
//   -> one coupling round for every request at its cutset
//   -> D2H of a small summary, one stream synchronisation.
// The layer-choice rule of method 3 is the reference GPU driver's
// (src/pmdd/enum/gpu/enum.cu:331-428, :661-738): expand top-down while
// top-down score <= bottom-up score, where the top-down score is the next top-down
// layer's candidate count and the bottom-up score is 1.5x (truncated) the next
// bottom-up layer's candidate count; both start at 0.
#include "engine.hpp"
#include "tspbuild.cuh"

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <tuple>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>

namespace pmdd {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// ------------------------------------------------------------------- Arena
Arena::~Arena() {
    for (auto &c : chunks_) cudaFree(reinterpret_cast<void *>(c.first));
}

bool Arena::init(size_t budget, size_t initial, std::string *err) {
    cap_ = budget & ~static_cast<size_t>(255);
    if (!grow(std::min(std::max<size_t>(initial, 256), cap_))) {
        if (err) *err = "cudaMalloc of the engine arena failed";
        return false;
    }
    return true;
}

bool Arena::grow(size_t at_least) {
    size_t bytes = align256(std::max(at_least, std::min<size_t>(reserved_, size_t(16) << 30)));
    if (reserved_ + bytes > cap_) bytes = align256(at_least);
    if (reserved_ + bytes > cap_) return false;
    void *p = nullptr;
    const double t0 = now_s();
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();  // clear the sticky-free allocation error
        return false;
    }
    grow_s_ += now_s() - t0;
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    chunks_[a] = bytes;
    add_free(a, bytes);
    reserved_ += bytes;
    return true;
}

void *Arena::alloc(size_t bytes) {
    if (inj_count_ > 0) {
        if (inj_after_ > 0) {
            --inj_after_;
        } else {
            --inj_count_;
            ++injected_;
            return nullptr;
        }
    }
    bytes = align256(bytes == 0 ? 1 : bytes);
    for (int attempt = 0; attempt < 2; ++attempt) {
        // best fit: the smallest free block that holds `bytes` (lowest address among equals)
        auto bs = by_size_.lower_bound({bytes, 0});
        if (bs != by_size_.end()) {
            const uintptr_t a = bs->second;
            const size_t rem = bs->first - bytes;
            drop_free(free_.find(a));
            if (rem) add_free(a + bytes, rem);
            live_[a] = bytes;
            used_ += bytes;
            peak_ = std::max(peak_, used_);
            return reinterpret_cast<void *>(a);
        }
        if (attempt == 0 && !grow(bytes)) return nullptr;
    }
    return nullptr;
}

void Arena::add_free(uintptr_t a, size_t bytes) {
    free_[a] = bytes;
    by_size_.insert({bytes, a});
}

void Arena::drop_free(std::map<uintptr_t, size_t>::iterator it) {
    by_size_.erase({it->second, it->first});
    free_.erase(it);
}

void Arena::release(void *p) {
    if (p == nullptr) return;
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    auto lv = live_.find(a);
    if (lv == live_.end()) return;
    uintptr_t start = a;
    size_t bytes = lv->second;
    live_.erase(lv);
    used_ -= bytes;
    // coalesce with free neighbours of the same cudaMalloc chunk only
    auto ch = std::prev(chunks_.upper_bound(a));
    const uintptr_t c0 = ch->first, c1 = ch->first + ch->second;
    auto next = free_.lower_bound(start);
    if (next != free_.end() && next->first == start + bytes && next->first < c1) {
        bytes += next->second;
        auto after = std::next(next);
        drop_free(next);
        next = after;
    }
    if (next != free_.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == start && prev->first >= c0) {
            start = prev->first;
            bytes += prev->second;
            drop_free(prev);
        }
    }
    add_free(start, bytes);
}

bool Engine::Pinned::reserve(size_t bytes) {
    if (bytes <= cap) return true;
    size_t c = std::max<size_t>(bytes, cap * 2);
    c = std::max<size_t>(c, 1 << 16);
    void *np = nullptr;
    if (cudaMallocHost(&np, c) != cudaSuccess) return false;
    if (p) cudaFreeHost(p);
    p = np;
    cap = c;
    return true;
}

Engine::Pinned::~Pinned() {
    if (p) cudaFreeHost(p);
}

// ------------------------------------------------------ request preparation
int host_threads() {
    int t = static_cast<int>(std::thread::hardware_concurrency());
    if (t <= 0) t = 1;
    t = std::min(t, 32);
    const char *env = std::getenv("PMDD_HOST_THREADS");
    if (env && *env && std::atoi(env) > 0) t = std::atoi(env);
    return t;
}

void parallel_for(int64_t n, int threads, const std::function<void(int64_t)> &fn) {
    threads = static_cast<int>(std::min<int64_t>(std::max(threads, 1), n));
    if (threads <= 1) {
        for (int64_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<int64_t> next(0);
    auto worker = [&]() {
        for (int64_t i = next++; i < n; i = next++) fn(i);
    };
    std::vector<std::thread> pool;
    pool.reserve(threads - 1);
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto &th : pool) th.join();
}

void pack_instance(const pmdd_dd &dd, const Instance &I, unsigned char *dst) {
    const size_t N = static_cast<size_t>(I.N), A = static_cast<size_t>(I.A), K = static_cast<size_t>(I.K);
    std::memcpy(dst + I.off_layer, dd.layer_offsets, sizeof(int32_t) * (I.L + 1));
    std::memcpy(dst + I.off_in, dd.in_arc_offsets, sizeof(int32_t) * (N + 1));
    if (A > 0) {
        std::memcpy(dst + I.off_src, dd.arc_src, sizeof(int32_t) * A);
        std::memcpy(dst + I.off_w, dd.arc_weight, sizeof(int32_t) * A);
    }
    std::memcpy(dst + I.off_weights, dd.weights, sizeof(int32_t) * K * I.d);
    if (dd.min_weight) std::memcpy(dst + I.off_minw, dd.min_weight, sizeof(int32_t) * N);
    if (I.has_sd_order) std::memcpy(dst + I.off_sdord, I.sd_order.data(), sizeof(int32_t) * N);
    if (I.sd_kind == 2) {
        std::memcpy(dst + I.off_sdnext, I.sd_next.data(), sizeof(int32_t) * 2 * N);
        std::memcpy(dst + I.off_state, dd.node_state, sizeof(uint64_t) * N * static_cast<size_t>(I.state_words));
    }
}

// Set-packing state-dominance layout (src/pmdd/enum/cpu/dominance.cpp:88-173): per
// layer, nodes bucketed by state size (bucket b < num_layers-1), ordered by (size, id);
// a node whose bucket holds two or more nodes takes its partner from the next non-empty
// bucket only.  Fills I->sd_order and I->sd_next.
static void setpacking_sd_layout(const pmdd_dd &dd, Instance *I) {
    const int32_t N = dd.num_nodes, W = dd.state_words, nb = dd.num_layers - 1;
    I->sd_order.assign(N, 0);
    I->sd_next.assign(2 * static_cast<size_t>(N), 0);
    std::vector<int32_t> pc, first(nb + 1);
    for (int l = 0; l < dd.num_layers; ++l) {
        const int32_t b = dd.layer_offsets[l], e = dd.layer_offsets[l + 1], cnt = e - b;
        pc.assign(cnt, 0);
        for (int32_t i = 0; i < cnt; ++i) {
            const uint64_t *s = dd.node_state + static_cast<size_t>(b + i) * W;
            for (int32_t w = 0; w < W; ++w) pc[i] += __builtin_popcountll(s[w]);
        }
        int32_t *ord = I->sd_order.data() + b;
        for (int32_t i = 0; i < cnt; ++i) ord[i] = i;
        std::stable_sort(ord, ord + cnt, [&pc](int32_t x, int32_t y) { return pc[x] < pc[y]; });
        // first[k] = first order position with size >= k (sizes >= nb take no part)
        int32_t p = 0;
        for (int32_t k = 0; k <= nb; ++k) {
            while (p < cnt && pc[ord[p]] < k) ++p;
            first[k] = p;
        }
        int32_t *nx = I->sd_next.data() + 2 * static_cast<size_t>(b);
        for (int32_t k = 0; k + 1 < nb; ++k) {
            if (first[k + 1] - first[k] < 2) continue;
            int32_t k2 = k + 1;
            while (k2 < nb && first[k2 + 1] == first[k2]) ++k2;
            if (k2 >= nb) continue;
            for (int32_t q = first[k]; q < first[k + 1]; ++q) {
                nx[2 * q] = first[k2];
                nx[2 * q + 1] = first[k2 + 1];
            }
        }
    }
}

// The DD shape the footprint prediction reads: widest layer in arcs and in nodes.
static void set_shape(Instance *I, const std::vector<int32_t> &arc_at) {
    I->max_layer_arcs = 0;
    I->max_layer_nodes = 0;
    for (int l = 0; l < I->L; ++l) {
        I->max_layer_arcs = std::max<int64_t>(I->max_layer_arcs, arc_at[l + 1] - arc_at[l]);
        I->max_layer_nodes = std::max<int64_t>(I->max_layer_nodes, I->layer_off[l + 1] - I->layer_off[l]);
    }
}

int prepare_instance(const pmdd_dd &dd, const pmdd_options &o, uint64_t id, Instance *I, std::string *err,
                     bool with_out_csr, bool pack) {
    auto bad = [&](const std::string &m) {
        if (err) *err = m;
        return static_cast<int>(PMDD_ERR_INVALID);
    };
    if (o.method != 1 && o.method != 3) return bad("method must be 1 (top-down) or 3 (coupled) on the GPU backend");
    if (o.maximization == 0) return bad("only maximisation is supported (the reference's main always maximises)");
    if (dd.nobjs < 1 || dd.nobjs > 8) return bad("nobjs must be in 1..8");
    if (dd.num_layers < 2) return bad("DD needs at least a root and a terminal layer");
    if (dd.num_nodes < 2 || dd.num_arcs < 0 || dd.num_weights < 1) return bad("DD sizes out of range");
    if (!dd.layer_offsets || !dd.in_arc_offsets || !dd.weights || (dd.num_arcs > 0 && (!dd.arc_src || !dd.arc_weight)))
        return bad("DD array pointer is NULL");
    const int32_t L = dd.num_layers, N = dd.num_nodes, A = dd.num_arcs, K = dd.num_weights, d = dd.nobjs;
    if (dd.layer_offsets[0] != 0 || dd.layer_offsets[L] != N) return bad("layer_offsets must run from 0 to num_nodes");
    for (int l = 0; l < L; ++l)
        if (dd.layer_offsets[l + 1] <= dd.layer_offsets[l]) return bad("every layer needs at least one node");
    if (dd.layer_offsets[1] != 1) return bad("layer 0 must hold exactly the root");
    if (dd.layer_offsets[L] - dd.layer_offsets[L - 1] != 1) return bad("the last layer must hold exactly the terminal");
    if (dd.in_arc_offsets[0] != 0 || dd.in_arc_offsets[1] != 0) return bad("the root has no incoming arcs");
    if (dd.in_arc_offsets[N] != A) return bad("in_arc_offsets must end at num_arcs");
    for (int32_t v = 0; v < N; ++v)
        if (dd.in_arc_offsets[v + 1] < dd.in_arc_offsets[v]) return bad("in_arc_offsets must be non-decreasing");
    // every arc runs from the layer right above its head; bound on |path sums|
    std::vector<int64_t> row_max(K, 0);
    for (int32_t r = 0; r < K; ++r)
        for (int k = 0; k < d; ++k)
            row_max[r] = std::max<int64_t>(row_max[r], std::llabs(static_cast<int64_t>(dd.weights[static_cast<int64_t>(r) * d + k])));
    int64_t bound = 0;
    for (int l = 1; l < L; ++l) {
        int64_t layer_max = 0;
        const int32_t lo = dd.layer_offsets[l - 1], hi = dd.layer_offsets[l];
        const int32_t a0 = dd.in_arc_offsets[dd.layer_offsets[l]], a1 = dd.in_arc_offsets[dd.layer_offsets[l + 1]];
        bool bad_src = false, bad_w = false;
        for (int32_t a = a0; a < a1; ++a) {
            const int32_t s = dd.arc_src[a], w = dd.arc_weight[a];
            bad_src |= (s < lo) | (s >= hi);
            const bool wb = (w < 0) | (w >= K);
            bad_w |= wb;
            if (!wb) layer_max = std::max<int64_t>(layer_max, row_max[w]);
        }
        if (bad_src) return bad("arc tail is not in the layer above its head");
        if (bad_w) return bad("arc weight row out of range");
        bound += layer_max;
    }
    I->id = id;
    I->opts = o;
    I->d = d;
    I->wide = bound > static_cast<int64_t>(INT32_MAX);
    I->L = L;
    I->N = N;
    I->A = A;
    I->K = K;
    I->layer_off.assign(dd.layer_offsets, dd.layer_offsets + L + 1);
    I->arc_at_layer.resize(L + 1);
    for (int l = 0; l <= L; ++l) I->arc_at_layer[l] = dd.in_arc_offsets[dd.layer_offsets[l]];
    // pack the DD arrays
    size_t off = 0;
    I->off_layer = off;
    off = align256(off + sizeof(int32_t) * (L + 1));
    I->off_in = off;
    off = align256(off + sizeof(int32_t) * (static_cast<size_t>(N) + 1));
    I->off_src = off;
    off = align256(off + sizeof(int32_t) * static_cast<size_t>(A));
    I->off_w = off;
    off = align256(off + sizeof(int32_t) * static_cast<size_t>(A));
    I->off_weights = off;
    off = align256(off + sizeof(int32_t) * static_cast<size_t>(K) * d);
    const bool has_minw = dd.min_weight != nullptr;
    I->off_minw = has_minw ? off : 0;
    if (has_minw) off = align256(off + sizeof(int32_t) * static_cast<size_t>(N));
    const bool has_state = dd.node_state != nullptr && dd.state_words > 0;
    if (dd.node_state != nullptr && (dd.state_words <= 0 || dd.state_words > (1 << 20)))
        return bad("state_words out of range");
    // state-dominance data: by the requested problem type, or by what the DD carries for
    // resident sets (which serve any options)
    int sd_kind = 0;
    if (o.problem_type == 1 && has_minw) sd_kind = 1;
    else if (o.problem_type == 2 && has_state) sd_kind = 2;
    else if (with_out_csr) sd_kind = has_minw ? 1 : (has_state ? 2 : 0);
    I->sd_kind = (with_out_csr || o.state_dominance > 0) ? sd_kind : 0;
    I->has_sd_order = I->sd_kind != 0;
    I->off_sdord = I->off_sdnext = I->off_state = 0;
    I->state_words = 0;
    if (I->sd_kind == 1) {
        I->off_sdord = off;
        off = align256(off + sizeof(int32_t) * static_cast<size_t>(N));
        I->sd_order.resize(N);
        for (int l = 0; l < L; ++l) {
            const int32_t b = dd.layer_offsets[l], e = dd.layer_offsets[l + 1];
            int32_t *ord = I->sd_order.data() + b;
            for (int32_t i = 0; i < e - b; ++i) ord[i] = i;
            const int32_t *mw = dd.min_weight + b;
            std::stable_sort(ord, ord + (e - b), [mw](int32_t x, int32_t y) { return mw[x] > mw[y]; });
        }
    } else if (I->sd_kind == 2) {
        I->state_words = dd.state_words;
        I->off_sdord = off;
        off = align256(off + sizeof(int32_t) * static_cast<size_t>(N));
        I->off_sdnext = off;
        off = align256(off + sizeof(int32_t) * 2 * static_cast<size_t>(N));
        I->off_state = off;
        off = align256(off + sizeof(uint64_t) * static_cast<size_t>(N) * static_cast<size_t>(dd.state_words));
        setpacking_sd_layout(dd, I);
    }
    I->blob_bytes = off;
    if (pack) {
        I->blob.assign(off, 0);
        pack_instance(dd, *I, I->blob.data());
    }
    size_t dev = off;
    I->with_out_csr = with_out_csr || o.method == 3;
    if (I->with_out_csr) {
        dev = align256(dev + sizeof(int32_t) * (static_cast<size_t>(N) + 1));  // out_off
        dev = align256(dev + sizeof(int32_t) * static_cast<size_t>(A));       // out_head
        dev = align256(dev + sizeof(int32_t) * static_cast<size_t>(A));       // out_w
        dev = align256(dev + sizeof(int32_t) * static_cast<size_t>(N));       // cursor
    }
    I->dev_bytes = dev;
    set_shape(I, I->arc_at_layer);
    I->min_bytes = static_cast<int64_t>(dev);
    I->submit_s = now_s();
    return PMDD_OK;
}

void prepare_tsp_instance(const TspStructure &S, int nobjs, const int32_t *cost, const pmdd_options &opts,
                          uint64_t id, Instance *I) {
    const int n = S.n, d = nobjs;
    const int32_t L = n + 2, K = 1 + n * n;
    I->id = id;
    I->opts = opts;
    I->d = d;
    I->L = L;
    I->N = S.N;
    I->A = S.A;
    I->K = K;
    I->layer_off = S.layer_off;
    I->arc_at_layer = S.arc_at;
    I->tsp = &S;
    I->off_weights = 0;
    I->blob.assign(sizeof(int32_t) * static_cast<size_t>(K) * d, 0);
    int32_t *w = reinterpret_cast<int32_t *>(I->blob.data());
    const size_t nn = static_cast<size_t>(n) * n;
    for (size_t ij = 0; ij < nn; ++ij)
        for (int o = 0; o < d; ++o) w[(1 + ij) * d + o] = -cost[o * nn + ij];
    // |path sum| bound, layer by layer as prepare_instance takes it: the arcs into layer 2
    // use rows (0, v), layers 3..n rows (u, v) with u, v >= 1, the terminal rows (u, 0)
    auto rmax = [&](int i, int j) {
        int64_t m = 0;
        for (int o = 0; o < d; ++o) m = std::max<int64_t>(m, std::llabs(static_cast<int64_t>(cost[o * nn + i * n + j])));
        return m;
    };
    int64_t m2 = 0, m3 = 0, mt = 0;
    for (int v = 1; v < n; ++v) m2 = std::max(m2, rmax(0, v));
    for (int u = 1; u < n; ++u)
        for (int v = 1; v < n; ++v)
            if (u != v) m3 = std::max(m3, rmax(u, v));
    for (int u = 1; u < n; ++u) mt = std::max(mt, rmax(u, 0));
    const int64_t bound = m2 + static_cast<int64_t>(std::max(0, n - 2)) * m3 + mt;
    I->wide = bound > static_cast<int64_t>(INT32_MAX);
    I->blob_bytes = I->blob.size();
    I->dev_bytes = align256(I->blob_bytes);
    I->with_out_csr = true;
    I->sd_kind = 0;
    I->has_sd_order = false;
    set_shape(I, S.arc_at);
    I->min_bytes = static_cast<int64_t>(I->dev_bytes);
    I->submit_s = now_s();
}

const TspStructure *Engine::tsp_structure(int n, std::string *err) {
    auto it = tsp_cache_.find(n);
    if (it != tsp_cache_.end()) return it->second.get();
    if (!make_current()) {
        *err = error_;
        return nullptr;
    }
    if (n < dev::kTspMinCities || n > dev::kTspMaxCities) {
        *err = "TSP structure: n must be in 2..20";
        return nullptr;
    }
    std::unique_ptr<TspStructure> S(new TspStructure);
    const dev::TspShape shape = dev::tsp_shape(n);
    S->n = n;
    S->layer_off = shape.layer_off;
    S->arc_at = shape.arc_at;
    S->N = shape.layer_off.back();
    S->A = shape.arc_at.back();
    const size_t L1 = shape.layer_off.size(), N = static_cast<size_t>(S->N), A = static_cast<size_t>(S->A);
    size_t off = 0;
    auto take = [&](size_t ints) {
        const size_t o = off;
        off = align256(off + sizeof(int32_t) * ints);
        return o;
    };
    const size_t o_lo = take(L1), o_in = take(N + 1), o_src = take(A), o_w = take(A), o_oo = take(N + 1),
                 o_oh = take(A), o_ow = take(A), o_cur = take(N), o_err = take(1);
    S->mem = static_cast<unsigned char *>(arena_.alloc(off));
    void *scratch = arena_.alloc(dev::tsp_scratch_bytes(n));
    if (!S->mem || !scratch) {
        arena_.release(S->mem);
        arena_.release(scratch);
        *err = "TSP structure does not fit the device memory budget";
        return nullptr;
    }
    int32_t *base = reinterpret_cast<int32_t *>(S->mem);
    auto at = [&](size_t o) { return reinterpret_cast<int32_t *>(S->mem + o); };
    int32_t *d_err = at(o_err);
    int32_t h_err = 0;
    (void)base;
    bool ok = cuda_ok(cudaMemsetAsync(d_err, 0, sizeof(int32_t), stream_), "TSP structure");
    int64_t nl = 0;
    ok = ok && cuda_ok(dev::launch_tsp_structure(n, shape, at(o_lo), at(o_in), at(o_src), at(o_w), scratch, d_err,
                                                 sms_, stream_, &nl),
                       "TSP structure");
    S->in_off = at(o_in);
    S->arc_src = at(o_src);
    S->arc_w = at(o_w);
    S->out_off = at(o_oo);
    S->out_head = at(o_oh);
    S->out_w = at(o_ow);
    S->cursor = at(o_cur);
    ok = ok && cuda_ok(dev::launch_build_out_csr(S->in_off, S->arc_src, S->arc_w, S->N, S->A, S->out_off, S->cursor,
                                                 S->out_head, S->out_w, stream_),
                       "TSP out-arc CSR");
    ok = ok && cuda_ok(cudaMemcpyAsync(&h_err, d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, stream_), "TSP check") &&
         cuda_ok(cudaStreamSynchronize(stream_), "TSP structure");
    launches_ += nl + 3;
    g_total_launches += nl + 3;
    arena_.release(scratch);
    if (!ok || h_err != 0) {
        arena_.release(S->mem);
        *err = ok ? "TSP structure: layer sizes differ from the combinatorial count (internal)" : error_;
        return nullptr;
    }
    const TspStructure *r = S.get();
    tsp_cache_[n] = std::move(S);
    return r;
}

void layout_built_knapsack(Instance *I, int d, bool wide, const std::vector<int32_t> &layer_off,
                           const std::vector<int32_t> &arc_at_layer, int32_t K) {
    const int32_t L = static_cast<int32_t>(layer_off.size()) - 1;
    const int32_t N = layer_off.back(), A = arc_at_layer.back();
    I->d = d;
    I->wide = wide;
    I->L = L;
    I->N = N;
    I->A = A;
    I->K = K;
    I->layer_off = layer_off;
    I->arc_at_layer = arc_at_layer;
    size_t off = 0;
    I->off_layer = off;
    off = align256(off + sizeof(int32_t) * (static_cast<size_t>(L) + 1));
    I->off_in = off;
    off = align256(off + sizeof(int32_t) * (static_cast<size_t>(N) + 1));
    I->off_src = off;
    off = align256(off + sizeof(int32_t) * static_cast<size_t>(A));
    I->off_w = off;
    off = align256(off + sizeof(int32_t) * static_cast<size_t>(A));
    I->off_weights = off;
    off = align256(off + sizeof(int32_t) * static_cast<size_t>(K) * d);
    I->off_minw = off;
    off = align256(off + sizeof(int32_t) * static_cast<size_t>(N));
    I->sd_kind = 1;
    I->has_sd_order = true;
    I->off_sdord = off;
    off = align256(off + sizeof(int32_t) * static_cast<size_t>(N));
    I->blob_bytes = off;
    I->with_out_csr = true;
    size_t dev = off;
    dev = align256(dev + sizeof(int32_t) * (static_cast<size_t>(N) + 1));
    dev = align256(dev + sizeof(int32_t) * static_cast<size_t>(A));
    dev = align256(dev + sizeof(int32_t) * static_cast<size_t>(A));
    dev = align256(dev + sizeof(int32_t) * static_cast<size_t>(N));
    I->dev_bytes = dev;
    set_shape(I, arc_at_layer);
    I->min_bytes = static_cast<int64_t>(dev);
    I->submit_s = now_s();
}

// ------------------------------------------------------------------ Engine
Engine::Engine(int device, int64_t budget_bytes, int max_slots, int stream_priority)
    : device_(device), max_slots_(max_slots) {
    const double init_t0 = now_s();
    struct InitTrace {
        const double &t0;
        const bool &ok;
        ~InitTrace() {
            const char *tr = std::getenv("PMDD_TRACE");
            if (tr && tr[0] == '1') std::fprintf(stderr, "[pmdd engine] init_ms=%.1f ok=%d\n", (now_s() - t0) * 1e3, ok);
        }
    } init_trace{init_t0, ok_};
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count <= 0) {
        error_ = e != cudaSuccess ? std::string("cudaGetDeviceCount failed: ") + cudaGetErrorString(e)
                                  : std::string("No CUDA device found");
        return;
    }
    if (device < 0 || device >= count) {
        error_ = "CUDA device ordinal out of range";
        return;
    }
    if (!cuda_ok(cudaSetDevice(device), "cudaSetDevice")) return;
    cudaDeviceProp prop;
    if (!cuda_ok(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties")) return;
    if (prop.major < 10) {
        error_ = "this engine is built for sm_100a (B200); device reports compute capability " +
                 std::to_string(prop.major) + "." + std::to_string(prop.minor);
        return;
    }
    sms_ = prop.multiProcessorCount;
    if (!cuda_ok(cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, stream_priority), "cudaStreamCreate"))
        return;
    for (cudaEvent_t &ev : ev_)
        if (!cuda_ok(cudaEventCreate(&ev), "cudaEventCreate")) return;
    size_t free_b = 0, total_b = 0;
    if (!cuda_ok(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo")) return;
    int64_t budget = budget_bytes;
    const int64_t cap = static_cast<int64_t>(free_b) - (static_cast<int64_t>(1) << 30);
    if (budget <= 0 || budget > cap) budget = static_cast<int64_t>(cap * 0.9);
    if (budget < (static_cast<int64_t>(64) << 20)) {
        error_ = "not enough free device memory for the engine arena";
        return;
    }
    // device memory is taken as it is needed: 2 GB now (PMDD_ARENA_INITIAL), more later
    int64_t initial = static_cast<int64_t>(2) << 30;
    const char *ini = std::getenv("PMDD_ARENA_INITIAL");
    if (ini && *ini && std::atoll(ini) > 0) initial = std::atoll(ini);
    if (!arena_.init(static_cast<size_t>(budget), static_cast<size_t>(std::min(initial, budget)), &error_)) return;
    if (max_slots_ <= 0) max_slots_ = 1 << 20;
    const char *tr = std::getenv("PMDD_TRACE");
    trace_ = tr != nullptr && tr[0] == '1';
    const char *bm = std::getenv("PMDD_BIG_MARK_MIN");
    if (bm && *bm && std::atoll(bm) > 0) big_mark_min_fixed_ = std::atoll(bm);
    load_tuning();
    // constant initial frontier: one zero point (up to 8 int64 values), offset 0, size 1
    if (!h_init_.reserve(512)) {
        error_ = "cudaMallocHost failed";
        return;
    }
    std::memset(h_init_.p, 0, 512);
    *reinterpret_cast<int32_t *>(static_cast<char *>(h_init_.p) + 128) = 1;  // size of the root frontier
    *(static_cast<unsigned char *>(h_init_.p) + 132) = 1;                   // one point is sorted
    // the seed side of an admitted request, one block: the zero point (64 B) | slot offset
    // 0 | size 1 | sorted 1
    *reinterpret_cast<int32_t *>(static_cast<char *>(h_init_.p) + kSeedTemplate + 72) = 1;
    *(static_cast<unsigned char *>(h_init_.p) + kSeedTemplate + 76) = 1;
    const char *lx = std::getenv("PMDD_LEX_TILES");
    if (lx && lx[0] == '0') lex_tiles_ = false;
    const char *sx = std::getenv("PMDD_SUM_TILES");
    if (sx && *sx) sum_tiles_ = sx[0] == '1';
    const char *lb = std::getenv("PMDD_LEX_BULK");
    if (lb && *lb) lex_bulk_ = lb[0] == '1';
    const char *cl = std::getenv("PMDD_CHAIN_LAYERS");
    if (cl && *cl) chain_layers_ = std::max(0, std::min(std::atoi(cl), kChainMaxLayers));
    const char *pr = std::getenv("PMDD_PIVOT_RULE");
    if (pr && *pr) pivot_rule_ = std::strcmp(pr, "n64") == 0 ? 0 : 1;
    const char *cg = std::getenv("PMDD_CHAIN_GROW");
    if (cg && *cg) chain_grow_all_ = std::strcmp(cg, "all") == 0;
    const char *cr = std::getenv("PMDD_CHAIN_MAX_REQUESTS");
    if (cr && *cr) chain_max_requests_ = std::max<int64_t>(0, std::atoll(cr));
    const char *cm = std::getenv("PMDD_CHAIN_MAX_CAND");
    if (cm && *cm) chain_max_cand_ = std::max<int64_t>(0, std::atoll(cm));
    const char *la = std::getenv("PMDD_BIG_LEX_MAX_ARCS");
    if (la && *la) lex_max_arcs_ = std::max(0, std::min(std::atoi(la), dev::kBigLexMaxArcs));
    const char *tw = std::getenv("PMDD_TILE_WINDOW_MAX");
    if (tw && *tw) window_max_fixed_ = std::atoll(tw);
    const char *pm = std::getenv("PMDD_LEX_PAIR_MAX");
    if (pm && *pm && std::atoi(pm) >= 0) lex_pair_max_fixed_ = std::atoi(pm);
    ok_ = true;
}

Engine::~Engine() {
    if (stream_) {
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
    }
    for (cudaEvent_t ev : ev_)
        if (ev) cudaEventDestroy(ev);
}

bool Engine::cuda_ok(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return true;
    error_ = std::string(what) + " failed: " + cudaGetErrorString(e);
    ok_ = false;
    return false;
}

// The tuning file written by pmdd_b200.autotune: {"entries": {"d<D>_p<P>":
// {"big_mark_min": <n>, ...}, ...}} (PMDD_TUNING_FILE, else
// $XDG_CACHE_HOME/pmdd_b200/tuning.json or ~/.cache/pmdd_b200/tuning.json).  Entries
// that do not parse are ignored; a missing file leaves the defaults.
std::string default_tuning_path() {
    if (const char *p = std::getenv("PMDD_TUNING_FILE")) return p;
    if (const char *x = std::getenv("XDG_CACHE_HOME")) return std::string(x) + "/pmdd_b200/tuning.json";
    if (const char *h = std::getenv("HOME")) return std::string(h) + "/.cache/pmdd_b200/tuning.json";
    return std::string();
}

std::map<std::pair<int, int>, int64_t> read_tuning(const std::string &path, const char *key) {
    std::map<std::pair<int, int>, int64_t> out;
    if (path.empty()) return out;
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return out;
    std::string text;
    char buf[4096];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0 && text.size() < (1u << 20)) text.append(buf, got);
    std::fclose(f);
    const std::string quoted = std::string("\"") + key + "\"";
    // entry keys "d<objectives>_p<problem type>"; an entry runs to the next entry key
    std::vector<std::pair<size_t, std::pair<int, int>>> entries;
    size_t pos = 0;
    while ((pos = text.find("\"d", pos)) != std::string::npos) {
        int d = 0, p = 0, used = 0;
        if (std::sscanf(text.c_str() + pos, "\"d%d_p%d\"%n", &d, &p, &used) == 2 && used > 0) {
            entries.push_back({pos, {d, p}});
            pos += used;
        } else {
            ++pos;
        }
    }
    for (size_t i = 0; i < entries.size(); ++i) {
        const size_t begin = entries[i].first;
        const size_t end = i + 1 < entries.size() ? entries[i + 1].first : text.size();
        const size_t k = text.find(quoted, begin);
        if (k == std::string::npos || k >= end) continue;
        long long v = 0;
        const int d = entries[i].second.first;
        if (std::sscanf(text.c_str() + k + quoted.size(), " : %lld", &v) == 1 && v >= 0 && d >= 1 && d <= 8)
            out[entries[i].second] = v;
    }
    return out;
}

void Engine::load_tuning() {
    const std::string path = default_tuning_path();
    tuned_mark_min_ = read_tuning(path, "big_mark_min");
    for (auto it = tuned_mark_min_.begin(); it != tuned_mark_min_.end();)  // 0 is not a crossover
        it = it->second > 0 ? std::next(it) : tuned_mark_min_.erase(it);
    tuned_pair_max_ = read_tuning(path, "lex_pair_max");
    tuned_window_max_ = read_tuning(path, "tile_window_max");
}

int64_t Engine::window_max_for(int d, int problem_type) const {
    int64_t w = dev::kTileWindow;
    if (window_max_fixed_ > 0) w = window_max_fixed_;
    else {
        auto it = tuned_window_max_.find({d, problem_type});
        if (it != tuned_window_max_.end()) w = it->second;
    }
    return std::max<int64_t>(dev::kTileWindowMin, std::min<int64_t>(dev::kTileWindow, w));
}

int64_t Engine::mark_min_for(int d, int problem_type) const {
    if (big_mark_min_fixed_ > 0) return big_mark_min_fixed_;
    auto it = tuned_mark_min_.find({d, problem_type});
    return it != tuned_mark_min_.end() ? it->second : static_cast<int64_t>(dev::kSmallMax) + 1;
}

int32_t Engine::pair_max_for(int d, int problem_type) const {
    if (lex_pair_max_fixed_ >= 0) return lex_pair_max_fixed_;
    auto it = tuned_pair_max_.find({d, problem_type});
    return it != tuned_pair_max_.end() ? static_cast<int32_t>(std::min<int64_t>(it->second, dev::kSmallMax))
                                       : kDefaultPairMax;
}

void *Engine::scratch(size_t bytes) {
    void *p = arena_.alloc(bytes);
    if (p) step_scratch_.push_back(p);
    return p;
}

void Engine::submit(std::unique_ptr<Instance> inst) { queued_.push_back(std::move(inst)); }

int64_t Engine::predicted_bytes(const Instance &I) const {
    const auto key = std::make_tuple(I.opts.problem_type, I.d, I.opts.method);
    auto it = cand_per_arc_.find(key);
    const double ratio = it != cand_per_arc_.end() ? it->second : 1.0;
    // the largest layer of candidates: what the request has shown so far, its next
    // expansion once counted (exact), and the class's learned ratio to the DD's arcs
    int64_t c = std::max<int64_t>(I.peak_cand, static_cast<int64_t>(ratio * static_cast<double>(I.A)));
    for (const Side *s : {&I.td, &I.bu})
        if (s->counted) c = std::max<int64_t>(c, s->res.total);
    const int64_t pb = static_cast<int64_t>(I.d) * static_cast<int64_t>(I.elem());
    int64_t b = I.external_dd ? 0 : static_cast<int64_t>(I.dev_bytes);
    b += 2 * c * pb + 8 * I.max_layer_arcs + 28 * I.max_layer_nodes;
    if (I.opts.method == 3) {
        const int64_t ucap = std::max<int64_t>(1 << 17, I.max_layer_nodes * (I.d + 1) + 4096);
        b += c * pb + static_cast<int64_t>(dev::couple_bytes(ucap, I.d, I.elem()));
    }
    return b;
}

int64_t Engine::current_bytes(const Instance &I) const {
    const int64_t pb = static_cast<int64_t>(I.d) * static_cast<int64_t>(I.elem());
    int64_t b = I.external_dd ? 0 : static_cast<int64_t>(I.dev_bytes);
    for (const Side *s : {&I.td, &I.bu})
        if (s->pts) b += s->slot_points * pb;
    return b;
}

int64_t Engine::reserved_growth() const {
    int64_t r = 0;
    for (const auto &p : active_)
        if (p->phase != Instance::DONE) r += std::max<int64_t>(0, predicted_bytes(*p) - current_bytes(*p));
    return r;
}

void Engine::learn_footprint(const Instance &I) {
    if (I.A <= 0 || I.peak_cand <= 0) return;
    const double seen = static_cast<double>(I.peak_cand) / static_cast<double>(I.A);
    double &r = cand_per_arc_.emplace(std::make_tuple(I.opts.problem_type, I.d, I.opts.method), seen).first->second;
    r = std::max(0.95 * r, seen);
}

void Engine::record_finish(const Instance &I) {
    if (I.status == PMDD_OK) {
        counters_.completed++;
        learn_footprint(I);
    } else if (I.status == PMDD_ERR_CANCELLED) {
        counters_.cancelled++;
    } else if (I.admit_s > 0) {
        counters_.failed++;
    } else {
        counters_.rejected++;
    }
}

void Engine::release_side(Side &s) {
    arena_.release(s.pts);
    arena_.release(s.off);
    arena_.release(s.size);
    arena_.release(s.arc_off);
    arena_.release(s.big_list);
    s.pts = nullptr;
    s.off = nullptr;
    s.size = nullptr;
    s.sorted = nullptr;
    s.arc_off = nullptr;
    s.big_list = nullptr;
    s.counted = false;
}

void Engine::release_instance(Instance &I) {
    release_side(I.td);
    release_side(I.bu);
    if (!I.external_dd) arena_.release(I.dd);
    arena_.release(I.cu_mem);
    arena_.release(I.cu_ctr);
    I.dd = nullptr;
    I.cu_mem = I.cu_U = I.cu_U_alt = I.cu_p2 = I.cu_sv = nullptr;
    I.cu_i2 = I.cu_si = I.cu_hist = nullptr;
    I.cu_ctr = nullptr;
    I.blob.clear();
    I.blob.shrink_to_fit();
    I.blob_src = nullptr;
    std::vector<int32_t>().swap(I.sd_order);
}

void Engine::fail(Instance &I, int status, const std::string &msg) {
    I.status = status;
    I.error = msg;
    I.phase = Instance::DONE;
}

bool Engine::cancel(uint64_t id) {
    for (auto it = queued_.begin(); it != queued_.end(); ++it) {
        if ((*it)->id == id) {
            fail(**it, PMDD_ERR_CANCELLED, "request cancelled");
            (*it)->finish_s = now_s();
            record_finish(**it);
            finished_.push_back(std::move(*it));
            queued_.erase(it);
            return true;
        }
    }
    for (auto &p : active_) {
        if (p && p->id == id && p->phase != Instance::DONE) {
            fail(*p, PMDD_ERR_CANCELLED, "request cancelled");
            return true;  // collected at the end of the next step
        }
    }
    return false;
}

bool Engine::carve_couple(Instance &I, int64_t ucap) {
    void *mem = arena_.alloc(dev::couple_bytes(ucap, I.d, I.elem()));
    if (!mem) return false;
    const size_t pts = align256(static_cast<size_t>(ucap) * I.d * I.elem());
    const size_t idx = align256(static_cast<size_t>(ucap) * sizeof(int32_t));
    char *m = static_cast<char *>(mem);
    void *old_U = I.cu_U, *old_mem = I.cu_mem;
    I.cu_mem = mem;
    I.cu_U = m;
    I.cu_U_alt = m + pts;
    I.cu_p2 = m + 2 * pts;
    I.cu_sv = m + 3 * pts;
    I.cu_i2 = reinterpret_cast<int32_t *>(m + 4 * pts);
    I.cu_si = reinterpret_cast<int32_t *>(m + 4 * pts + idx);
    I.cu_hist = reinterpret_cast<int32_t *>(m + 4 * pts + 2 * idx);
    if (old_U && I.result_n > 0)  // carry the running frontier over (growth)
        cudaMemcpyAsync(I.cu_U, old_U, static_cast<size_t>(I.result_n) * I.d * I.elem(), cudaMemcpyDeviceToDevice,
                        stream_);
    arena_.release(old_mem);  // stream-ordered: the copy above runs first
    I.cu_ucap = ucap;
    return true;
}

bool Engine::make_current() {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur == device_) return true;
    return cuda_ok(cudaSetDevice(device_), "cudaSetDevice");
}

bool Engine::upload_dd(Instance &I) {
    if (!make_current()) return false;
    I.dd = static_cast<unsigned char *>(arena_.alloc(I.dev_bytes));
    if (!I.dd) return false;
    if (!cuda_ok(cudaMemcpyAsync(I.dd, I.blob_src ? I.blob_src : I.blob.data(), I.blob_bytes, cudaMemcpyHostToDevice, stream_), "DD upload"))
        return false;
    return bind_dd(I);
}

bool Engine::bind_dd(Instance &I) {
    if (I.tsp) {  // shared structure: only the weight table is the instance's own
        const TspStructure &S = *I.tsp;
        I.d_in_off = S.in_off;
        I.d_arc_src = S.arc_src;
        I.d_arc_w = S.arc_w;
        I.d_weights = reinterpret_cast<const int32_t *>(I.dd);
        I.d_sd_order = nullptr;
        I.d_sd_next = nullptr;
        I.d_state = nullptr;
        I.d_out_off = S.out_off;
        I.d_out_head = S.out_head;
        I.d_out_w = S.out_w;
        I.d_cursor = S.cursor;
        return true;
    }
    I.d_in_off = reinterpret_cast<const int32_t *>(I.dd + I.off_in);
    I.d_arc_src = reinterpret_cast<const int32_t *>(I.dd + I.off_src);
    I.d_arc_w = reinterpret_cast<const int32_t *>(I.dd + I.off_w);
    I.d_weights = reinterpret_cast<const int32_t *>(I.dd + I.off_weights);
    I.d_sd_order = I.has_sd_order ? reinterpret_cast<const int32_t *>(I.dd + I.off_sdord) : nullptr;
    I.d_sd_next = I.sd_kind == 2 ? reinterpret_cast<const int32_t *>(I.dd + I.off_sdnext) : nullptr;
    I.d_state = I.sd_kind == 2 ? reinterpret_cast<const uint64_t *>(I.dd + I.off_state) : nullptr;
    if (I.with_out_csr) {
        size_t off = I.blob_bytes;
        I.d_out_off = reinterpret_cast<int32_t *>(I.dd + off);
        off = align256(off + sizeof(int32_t) * (static_cast<size_t>(I.N) + 1));
        I.d_out_head = reinterpret_cast<int32_t *>(I.dd + off);
        off = align256(off + sizeof(int32_t) * static_cast<size_t>(I.A));
        I.d_out_w = reinterpret_cast<int32_t *>(I.dd + off);
        off = align256(off + sizeof(int32_t) * static_cast<size_t>(I.A));
        I.d_cursor = reinterpret_cast<int32_t *>(I.dd + off);
        if (!cuda_ok(dev::launch_build_out_csr(I.d_in_off, I.d_arc_src, I.d_arc_w, I.N, I.A, I.d_out_off, I.d_cursor,
                                               I.d_out_head, I.d_out_w, stream_),
                     "out-arc CSR"))
            return false;
        launches_ += 3;
        g_total_launches += 3;
    }
    return true;
}

void Engine::release_dd(Instance &I) {
    arena_.release(I.dd);
    I.dd = nullptr;
}

// Uploads the DD (unless resident), builds the bottom-up CSR and seeds the frontiers.
bool Engine::admit(Instance &I) {
    if (!I.external_dd) {
        if (!upload_dd(I)) {
            arena_.release(I.dd);
            I.dd = nullptr;
            return false;
        }
    }
    auto seed = [&](Side &s, int layer) -> bool {
        s.layer = layer;
        s.slot_points = 1;
        // one block (released through pts; the arena ignores the releases of off and size):
        // the zero point | slot offset | size | sorted flag, written by one copy
        char *b = static_cast<char *>(arena_.alloc(kSeedBytes));
        if (!b) return false;
        s.pts = b;
        s.off = reinterpret_cast<int64_t *>(b + 64);
        s.size = reinterpret_cast<int32_t *>(b + 72);
        s.sorted = reinterpret_cast<uint8_t *>(b + 76);
        cudaMemcpyAsync(b, static_cast<const char *>(h_init_.p) + kSeedTemplate, kSeedBytes, cudaMemcpyHostToDevice,
                        stream_);
        s.counted = false;
        s.score = 0;
        return true;
    };
    if (!seed(I.td, 0) || (I.opts.method == 3 && !seed(I.bu, I.L - 1))) {
        release_instance(I);
        return false;
    }
    if (I.opts.method == 3 && !I.with_out_csr) {
        fail(I, PMDD_ERR_INVALID, "resident DD lacks the bottom-up CSR needed by method 3");
        return true;
    }
    I.blob.clear();
    I.blob.shrink_to_fit();
    I.blob_src = nullptr;
    std::vector<int32_t>().swap(I.sd_order);
    I.phase = Instance::RUNNING;
    I.admit_s = now_s();
    return true;
}

namespace {

struct ExpPlan {
    Instance *I;
    bool td;
    int nl;
    void *out_pts;
    int64_t *out_off;
    int32_t *out_size;
    uint8_t *out_sorted;  // per destination: written in lexicographic order (after the tile plan)
    void *big_mem;    // oversized-destination scratch (one block, carved per use)
    int64_t big_total;
    int64_t cand;       // candidates of this expansion (trace / statistics)
    int64_t max_item;
    int64_t num_big;
    // oversized scratch in passes of whole destinations (--max-cand): pass p holds the
    // destinations whose scratch offset is in [p * big_window, (p + 1) * big_window),
    // so big_rows = min(big_total, big_window + largest destination) rows suffice
    int64_t big_window = 1;
    int64_t window = dev::kTileWindow;  // its tile window
    int64_t big_rows = 0;
};

struct CountPlan {
    Instance *I;
    bool td;
    bool after_expand;  // score update (false for the initial counts at admission)
};

// A request chained within one step (chain.cu): chained layer j (from 1) expands it to
// layer e->nl + j into buffer set j % 2, reading set (j - 1) % 2 (layer 1: the step's own
// expansion and count), and counts the layer after it into the same set.
struct ChainSlot {
    Instance *I = nullptr;
    const ExpPlan *e = nullptr;    // this step's expansion of the request
    size_t count_idx = 0;          // this step's count of the layer after it
    int32_t last = 0;              // chained layers at most (the terminal layer included)
    int32_t dir = 1;               // +1: the top-down side; -1: the bottom-up one (method 3)
    int64_t other_score = INT64_MAX;  // method 3: the other side's score (the side rule)
    int64_t cap = 0;               // candidates a frontier buffer holds
    int64_t ntiles = 0;            // tiles a chained layer may need
    int32_t vmax = 0, amax = 0;    // most nodes / in-arcs of a chained layer
    int32_t cmax = 0;              // most nodes of a layer a chained count counts
    int64_t items[2] = {0, 0};
    void *pts[2] = {nullptr, nullptr};
    int64_t *off[2] = {nullptr, nullptr};
    int32_t *size[2] = {nullptr, nullptr};  // sizes | tile plan | sorted flags (at sorted())
    int64_t *arc[2] = {nullptr, nullptr};
    int64_t *big[2] = {nullptr, nullptr};
    uint8_t *sorted(int b) const { return reinterpret_cast<uint8_t *>(size[b] + vmax + ntiles + 1); }
};

// The chained requests of one (objectives, point type) pair, sharing launches.
struct ChainGroup {
    int d = 0;
    bool wide = false;
    std::vector<ChainSlot> slots;
    int32_t layers = 0;            // most chained layers of a slot
    size_t layer_bytes = 0;        // staging per layer: jobs | tile bases | item bases | count jobs
    size_t st_off = 0;             // staging: layers, then cap | last | count index
    size_t dv_off = 0;             // the group's part of the chain block (layout below)
    size_t dv_bytes = 0;
    size_t first_slot = 0;         // index of its first slot over all groups
    std::vector<int64_t> items, tiles;  // per layer: destinations, tile bound
    size_t r_bytes() const { return align256(sizeof(dev::CountResult) * static_cast<size_t>(layers) * slots.size()); }
    size_t n4() const { return align256(sizeof(int32_t) * slots.size()); }
    size_t ln(size_t each) const { return align256(each * static_cast<size_t>(layers)); }
    // chain block: counts [layers][n] | stop [n] | stopped_at [n] | tile survivors and
    // staircase candidates [layers][n][2] | tile queue [layers] | tiles [layers] |
    // next expansion's tiles [layers][n] | finished count blocks [layers]
    size_t off_stop() const { return r_bytes(); }
    size_t off_stopped() const { return off_stop() + n4(); }
    size_t off_ts() const { return off_stopped() + n4(); }
    size_t off_queue() const { return off_ts() + ln(2 * sizeof(unsigned long long) * slots.size()); }
    size_t off_tiles() const { return off_queue() + ln(sizeof(unsigned long long)); }
    size_t off_nt() const { return off_tiles() + ln(sizeof(int64_t)); }
    size_t off_done() const { return off_nt() + ln(sizeof(int64_t) * slots.size()); }
    size_t bytes() const { return off_done() + ln(sizeof(unsigned int)); }
};

}  // namespace

std::atomic<int64_t> g_total_launches{0};

int Engine::step() {
    if (!ok_ || !make_current()) return -1;
    const double step_t0 = trace_ ? now_s() : 0.0;
    struct LaunchTally {
        const int64_t &n;
        int64_t start;
        ~LaunchTally() { g_total_launches += n - start; }
    } tally{launches_, launches_};
    // ---------------------------------------------------------------- admission
    // A queued request is admitted when its predicted peak footprint fits beside what the
    // running requests hold and are predicted to grow by; a request that does not fit
    // stays queued and smaller ones behind it may pass, until it has been passed over
    // kMaxPassOver times, after which nothing behind it is admitted before it.  With
    // nothing running a request is always tried (its prediction may be pessimistic).  A
    // request whose DD alone exceeds the budget is rejected at once.
    constexpr int32_t kMaxPassOver = 32;
    std::vector<CountPlan> counts;
    const int64_t cap_bytes = static_cast<int64_t>(arena_.capacity());
    int64_t reserved = reserved_growth();
    for (auto it = queued_.begin(); it != queued_.end() && static_cast<int>(active_.size()) < max_slots_;) {
        Instance &I = **it;
        auto reject = [&](const std::string &msg) {
            fail(I, PMDD_ERR_OOM, msg);
            I.finish_s = now_s();
            record_finish(I);
            finished_.push_back(std::move(*it));
            it = queued_.erase(it);
        };
        if (I.min_bytes > cap_bytes) {
            reject("request needs at least " + std::to_string(I.min_bytes) + " device bytes for its DD, above the "
                   "memory budget of " + std::to_string(cap_bytes));
            continue;
        }
        const int64_t pred = predicted_bytes(I);
        const bool fits = static_cast<int64_t>(arena_.used()) + reserved + pred <= cap_bytes;
        if (!fits && !active_.empty()) {
            if (++I.skipped > kMaxPassOver) break;
            ++it;
            continue;
        }
        if (!admit(I)) {
            if (!ok_) return -1;
            if (!active_.empty()) {  // wait for memory to free up
                if (++I.skipped > kMaxPassOver) break;
                ++it;
                continue;
            }
            reject("request does not fit the device memory budget");
            continue;
        }
        counters_.admitted++;
        reserved += std::max<int64_t>(0, pred - current_bytes(I));
        if (I.phase == Instance::RUNNING) {
            counts.push_back({&I, true, false});
            if (I.opts.method == 3) counts.push_back({&I, false, false});
        }
        active_.push_back(std::move(*it));
        it = queued_.erase(it);
    }
    counters_.running_peak = std::max<int64_t>(counters_.running_peak, static_cast<int64_t>(active_.size()));
    counters_.queued_peak = std::max<int64_t>(counters_.queued_peak, static_cast<int64_t>(queued_.size()));

    // ------------------------------------------------------------ expansions
    std::vector<ExpPlan> exps;
    int64_t blocked_need = -1;
    Instance *blocked = nullptr;
    // tile window of this step: full windows when the step has candidates for a few waves
    // of tiles over the SMs, smaller ones (more tiles) when it has not
    int64_t step_cand = 0;
    for (auto &p : active_) {
        const Instance &I = *p;
        if (I.phase != Instance::RUNNING) continue;
        const bool is_td = I.opts.method != 3 || I.td.score <= I.bu.score;
        const Side &s = is_td ? I.td : I.bu;
        if (s.counted) step_cand += s.res.total;
    }
    const int64_t want_tiles = static_cast<int64_t>(sms_) * 6;
    const int64_t step_window = std::max<int64_t>(dev::kTileWindowMin, std::min<int64_t>(dev::kTileWindow,
                                                                                          step_cand / want_tiles));
    for (auto &p : active_) {
        Instance &I = *p;
        if (I.phase != Instance::RUNNING) continue;
        bool is_td = true;
        if (I.opts.method == 3) is_td = I.td.score <= I.bu.score;
        Side &s = is_td ? I.td : I.bu;
        if (!s.counted) continue;
        const int nl = is_td ? s.layer + 1 : s.layer - 1;
        const int64_t C = s.res.total;
        const int32_t V = I.nodes_in(nl);
        ExpPlan e{&I, is_td, nl, nullptr, nullptr, nullptr, nullptr, nullptr, 0, C, s.res.max_item, s.res.num_big};
        e.window = std::min<int64_t>(step_window, window_max_for(I.d, I.opts.problem_type));
        const int64_t window = e.window;
        const size_t pts_bytes = static_cast<size_t>(std::max<int64_t>(C, 1)) * I.d * I.elem();
        // one block: slot offsets | sizes of the new frontier | the tile plan of this
        // expansion | sorted flags | the frontier's points (released through out_off; the
        // arena ignores the releases of out_size and out_pts, which it did not hand out).
        // The points come last, so that a read widened to 16 bytes past their end stays
        // inside the block (the arena rounds blocks up to 256 bytes).
        const int64_t ntiles = std::max<int64_t>(1, (C + window - 1) / window);
        const size_t off_bytes = align256(sizeof(int64_t) * V);
        const size_t size_bytes = align256(sizeof(int32_t) * (V + ntiles + 1) + static_cast<size_t>(V));
        char *ix = static_cast<char *>(arena_.alloc(off_bytes + size_bytes + pts_bytes));
        e.out_off = reinterpret_cast<int64_t *>(ix);
        e.out_size = ix ? reinterpret_cast<int32_t *>(ix + off_bytes) : nullptr;
        e.out_pts = ix ? ix + off_bytes + size_bytes : nullptr;
        if (e.out_size) e.out_sorted = reinterpret_cast<uint8_t *>(e.out_size + V + ntiles + 1);
        bool okay = e.out_pts && e.out_off && e.out_size;
        if (okay && s.res.num_big > 0) {
            const int64_t bt = s.res.big_total;
            const int64_t cap = I.opts.max_cand > 0 ? I.opts.max_cand : bt;
            e.big_total = bt;
            e.big_window = std::max<int64_t>(1, std::min<int64_t>(cap, bt));
            e.big_rows = std::min<int64_t>(bt, e.big_window + s.res.max_item);
            e.big_mem =
                arena_.alloc(static_cast<size_t>(e.big_rows) * dev::big_scratch_bytes_per_point(I.d, I.elem()) + 1024);
            okay = e.big_mem != nullptr;
        }
        if (!okay) {
            for (void *q : {e.out_pts, static_cast<void *>(e.out_off), static_cast<void *>(e.out_size), e.big_mem})
                arena_.release(q);
            const int64_t need = static_cast<int64_t>(pts_bytes);
            if (need > blocked_need) {
                blocked_need = need;
                blocked = &I;
            }
            continue;
        }
        exps.push_back(e);
    }


    // group by (d, wide) and build descriptors
    std::map<std::pair<int, bool>, std::vector<size_t>> groups;
    for (size_t i = 0; i < exps.size(); ++i) groups[{exps[i].I->d, exps[i].I->wide}].push_back(i);

    // staging of every H2D payload of this step
    size_t stage_bytes = 0;
    stage_bytes += align256(sizeof(dev::ExpandJob) * exps.size());
    stage_bytes += align256(sizeof(dev::BigWork) * 1);  // sized below per group
    std::vector<dev::ExpandJob> xjobs(exps.size());
    std::vector<dev::BigWork> bigwork;
    struct GroupLaunch {
        int d;
        bool wide;
        size_t first, count;       // into xjobs
        int64_t tiles;
        size_t big_first, big_count;
        int64_t max_big;
        int32_t max_big_arcs;      // most arcs of an oversized destination (merge rounds)
        int64_t items;             // destinations over the group's jobs
        int64_t big_passes;        // scratch passes of the oversized path
        int64_t big_rows;          // oversized candidate rows over the group's jobs (flat space)
        int64_t mark_cap;          // upper bound on the group's mark-path destinations per pass
    };
    std::vector<GroupLaunch> glaunch;
    std::vector<int64_t> tile_bases(exps.size()), item_bases(exps.size());  // group-relative
    std::vector<int64_t> big_bases(exps.size());                           // group-relative
    {
        size_t pos = 0;
        std::vector<ExpPlan> ordered;
        ordered.reserve(exps.size());
        for (auto &g : groups) {
            GroupLaunch gl{g.first.first, g.first.second, pos, g.second.size(), 0, bigwork.size(), 0, 0, 0, 0, 0, 0, 0};
            for (size_t idx : g.second) {
                const ExpPlan &e = exps[idx];
                Instance &I = *e.I;
                Side &s = e.td ? I.td : I.bu;
                dev::ExpandJob &J = xjobs[pos];
                std::memset(&J, 0, sizeof(J));
                if (e.td) {
                    J.item_arc_off = I.d_in_off;
                    J.arc_nbr = I.d_arc_src;
                    J.arc_wrow = I.d_arc_w;
                    J.arc_base = I.arc_at_layer[e.nl];
                } else {
                    J.item_arc_off = I.d_out_off;
                    J.arc_nbr = I.d_out_head;
                    J.arc_wrow = I.d_out_w;
                    J.arc_base = I.arc_at_layer[e.nl + 1];
                }
                J.weights = I.d_weights;
                J.arc_cand_off = s.arc_off;
                J.item_base = I.layer_off[e.nl];
                J.num_items = I.nodes_in(e.nl);
                J.prev_base = I.layer_off[s.layer];
                J.prev_pts = s.pts;
                J.prev_off = s.off;
                J.prev_size = s.size;
                J.out_pts = e.out_pts;
                J.out_off = e.out_off;
                J.out_size = e.out_size;
                J.total_cand = s.res.total;
                J.tile_window = e.window;
                J.num_tiles = std::max<int64_t>(1, (s.res.total + e.window - 1) / e.window);
                J.tile_first = e.out_size + J.num_items;
                J.prev_sorted = s.sorted;
                J.out_sorted = e.out_sorted;
                J.pair_max = pair_max_for(I.d, I.opts.problem_type);
                J.lex_big = (I.d == 3 && lex_tiles_) ? 1 : 0;
                J.lex_bulk = lex_bulk_ ? 1 : 0;
                J.lex_max_arcs = lex_max_arcs_;
                J.tile_base = gl.tiles;
                tile_bases[pos] = gl.tiles;
                item_bases[pos] = gl.items;
                gl.tiles += J.num_tiles;
                gl.items += J.num_items;
                J.big_list = s.big_list;
                J.num_big = s.res.num_big;
                if (e.big_mem) {
                    const size_t pb = align256(static_cast<size_t>(e.big_rows) * I.d * I.elem());
                    const size_t ib = align256(sizeof(int32_t) * static_cast<size_t>(e.big_rows));
                    char *m = static_cast<char *>(e.big_mem);
                    J.big_pts = m;
                    J.big_pts2 = m + pb;
                    J.big_surv = m + 2 * pb;
                    J.big_idx = reinterpret_cast<int32_t *>(m + 3 * pb);
                    J.big_surv_idx = reinterpret_cast<int32_t *>(m + 3 * pb + ib);
                    J.big_window = e.big_window;
                    J.big_rows = e.big_rows;
                    const int64_t mm = mark_min_for(I.d, I.opts.problem_type);
                    J.big_mark_min = mm;
                    J.pivot_rule = pivot_rule_;
                    if (s.res.max_item >= mm) gl.mark_cap += e.big_rows / mm + 1;
                    gl.big_passes = std::max<int64_t>(gl.big_passes, (e.big_total + e.big_window - 1) / e.big_window);
                }
                big_bases[pos] = gl.big_rows;
                gl.big_rows += J.big_rows;
                for (int b = 0; b < s.res.num_big; ++b) bigwork.push_back({static_cast<int32_t>(pos - gl.first), b});
                if (s.res.num_big > 0) {
                    gl.max_big = std::max(gl.max_big, s.res.max_item);
                    gl.max_big_arcs = std::max(gl.max_big_arcs, s.res.max_big_arcs);
                }
                ordered.push_back(e);
                ++pos;
            }
            gl.big_count = bigwork.size() - gl.big_first;
            glaunch.push_back(gl);
        }
        exps.swap(ordered);
    }
    const double t_p1 = trace_ ? now_s() : 0.0;  // expansions planned and described

    // state dominance on the top-down layers that knapsack and set-packing requests asking
    // for it expand this step, in both methods (jobs follow the expansion order, so
    // (d, wide) groups stay contiguous)
    struct SdGroup {
        int d;
        bool wide;
        size_t first, count;
        int64_t total;  // nodes over the group's jobs
    };
    std::vector<dev::StateDomJob> sdjobs;
    std::vector<int64_t> sd_bases;
    std::vector<Instance *> sd_inst;
    std::vector<SdGroup> sdg;
    bool sd_alloc_failed = false;
    {
        std::vector<size_t> pick;
        size_t keep_bytes = 0;
        for (size_t i = 0; i < exps.size(); ++i) {
            const ExpPlan &e = exps[i];
            const Instance &I = *e.I;
            if (e.td && I.opts.state_dominance > 0 && I.sd_kind != 0 && I.sd_kind == I.opts.problem_type &&
                I.d_sd_order != nullptr && I.nodes_in(e.nl) > 1) {
                pick.push_back(i);
                keep_bytes += align256(static_cast<size_t>(std::max<int64_t>(e.cand, 1)));
            }
        }
        char *keep = pick.empty() ? nullptr : static_cast<char *>(scratch(keep_bytes));
        if (!pick.empty() && !keep) sd_alloc_failed = true;  // rolled back below, before any launch
        if (keep) {
            for (size_t k = 0; k < pick.size(); ++k) {
                const ExpPlan &e = exps[pick[k]];
                Instance &I = *e.I;
                dev::StateDomJob J;
                std::memset(&J, 0, sizeof(J));
                J.order = I.d_sd_order + I.layer_off[e.nl];
                J.kind = I.sd_kind;
                J.next = I.sd_kind == 2 ? I.d_sd_next + 2 * static_cast<size_t>(I.layer_off[e.nl]) : nullptr;
                J.state = I.d_state;
                J.state_words = I.state_words;
                J.in_off = I.d_in_off;
                J.arc_src = I.d_arc_src;
                J.arc_w = I.d_arc_w;
                J.pts = e.out_pts;
                J.off = e.out_off;
                J.size = e.out_size;
                J.keep = reinterpret_cast<uint8_t *>(keep);
                keep += align256(static_cast<size_t>(std::max<int64_t>(e.cand, 1)));
                J.removed = nullptr;  // set once the step's summary block exists
                J.node_base = I.layer_off[e.nl];
                J.num_nodes = I.nodes_in(e.nl);
                if (sdg.empty() || sdg.back().d != I.d || sdg.back().wide != I.wide)
                    sdg.push_back({I.d, I.wide, k, 0, 0});
                SdGroup &g = sdg.back();
                sd_bases.push_back(g.total);
                g.total += J.num_nodes;
                g.count++;
                sdjobs.push_back(J);
                sd_inst.push_back(&I);
            }
        }
    }

    // count plans for sides that move this step
    for (const ExpPlan &e : exps) {
        Instance &I = *e.I;
        if (I.opts.method == 1) {
            if (e.nl < I.L - 1) counts.push_back({&I, true, true});
        } else {
            const int td_layer = e.td ? e.nl : I.td.layer;
            const int bu_layer = e.td ? I.bu.layer : e.nl;
            if (td_layer != bu_layer) counts.push_back({&I, e.td, true});
        }
    }
    std::vector<dev::CountJob> cjobs(counts.size());
    std::vector<int64_t *> new_arc_off(counts.size(), nullptr);
    std::vector<int64_t *> new_big(counts.size(), nullptr);
    // The step's summary block: everything the host reads back after the step, in one
    // device allocation and one copy: count results | tile survivors per expansion |
    // labels removed by state dominance per job | error word.  All but the count
    // results start at zero (one memset).
    const size_t f_ts = sizeof(dev::CountResult) * counts.size();
    const size_t f_sd = f_ts + 2 * sizeof(unsigned long long) * exps.size();  // (survivors, staircase) per expansion
    const size_t f_err = f_sd + sizeof(int64_t) * sdjobs.size();
    const size_t f_clk = f_err + sizeof(uint64_t);  // PMDD_TRACE: tile phase cycles (8 counters)
    const size_t f_q = f_clk + (trace_ ? 10 * sizeof(unsigned long long) : 0);  // tile queue per group
    const size_t f_total = f_q + sizeof(unsigned long long) * glaunch.size();
    char *d_fixed = static_cast<char *>(scratch(f_total));
    dev::CountResult *d_results = counts.empty() ? nullptr : reinterpret_cast<dev::CountResult *>(d_fixed);
    unsigned long long *d_tile_surv = d_fixed ? reinterpret_cast<unsigned long long *>(d_fixed + f_ts) : nullptr;
    int64_t *d_removed = d_fixed ? reinterpret_cast<int64_t *>(d_fixed + f_sd) : nullptr;
    uint32_t *d_err_step = d_fixed ? reinterpret_cast<uint32_t *>(d_fixed + f_err) : nullptr;
    for (size_t k = 0; k < xjobs.size(); ++k) {
        xjobs[k].tile_surv = d_tile_surv ? d_tile_surv + 2 * k : nullptr;
        xjobs[k].err = d_err_step;
        xjobs[k].phase_clk = (trace_ && d_fixed) ? reinterpret_cast<unsigned long long *>(d_fixed + f_clk) : nullptr;
    }
    for (size_t k = 0; k < sdjobs.size(); ++k) sdjobs[k].removed = d_removed ? d_removed + k : nullptr;
    bool count_alloc_ok = d_fixed != nullptr && !sd_alloc_failed;
    // the expansion's new frontier is what the count reads; resolve per plan below

    // ------------------------------------------------------------- staging
    const size_t off_x = 0;
    const size_t off_b = align256(off_x + sizeof(dev::ExpandJob) * xjobs.size());
    const size_t off_c = align256(off_b + sizeof(dev::BigWork) * bigwork.size());
    const size_t off_tb = align256(off_c + sizeof(dev::CountJob) * cjobs.size());
    const size_t off_ib = align256(off_tb + sizeof(int64_t) * tile_bases.size());
    const size_t off_bb = align256(off_ib + sizeof(int64_t) * item_bases.size());
    const size_t off_sd = align256(off_bb + sizeof(int64_t) * big_bases.size());
    const size_t off_sdb = align256(off_sd + sizeof(dev::StateDomJob) * sdjobs.size());
    size_t off_k = align256(off_sdb + sizeof(int64_t) * sd_bases.size());
    // coupling: requests at their cutset
    std::vector<Instance *> couplers;
    for (auto &p : active_)
        if (p->phase == Instance::COUPLING) couplers.push_back(p.get());
    // (requests entering coupling this step are appended after the expansion bookkeeping)

    // --------------------------------------------------- finish planning of counts
    // Counts read the frontier a side will have after this step's expansions.
    // this step's expansion of each (request, direction), looked up per count
    std::unordered_map<const Instance *, std::pair<int32_t, int32_t>> exp_of;  // td, bu index (-1: none)
    exp_of.reserve(exps.size() * 2);
    for (size_t i = 0; i < exps.size(); ++i) {
        auto ins = exp_of.emplace(exps[i].I, std::make_pair(int32_t(-1), int32_t(-1)));
        (exps[i].td ? ins.first->second.first : ins.first->second.second) = static_cast<int32_t>(i);
    }
    auto exp_index = [&](const Instance &I, bool td) -> int32_t {
        auto it = exp_of.find(&I);
        return it == exp_of.end() ? -1 : (td ? it->second.first : it->second.second);
    };
    auto side_after = [&](Instance &I, bool td) -> std::pair<int, int32_t *> {
        const int32_t i = exp_index(I, td);
        if (i >= 0) return {exps[i].nl, exps[i].out_size};
        Side &s = td ? I.td : I.bu;
        return {s.layer, s.size};
    };
    for (size_t k = 0; k < counts.size() && count_alloc_ok; ++k) {
        Instance &I = *counts[k].I;
        const bool td = counts[k].td;
        auto cur = side_after(I, td);
        const int l = cur.first;
        const int nl = td ? l + 1 : l - 1;
        dev::CountJob &J = cjobs[k];
        std::memset(&J, 0, sizeof(J));
        if (td) {
            J.item_arc_off = I.d_in_off;
            J.arc_nbr = I.d_arc_src;
            J.arc_base = I.arc_at_layer[nl];
            J.num_arcs = I.arc_at_layer[nl + 1] - I.arc_at_layer[nl];
        } else {
            J.item_arc_off = I.d_out_off;
            J.arc_nbr = I.d_out_head;
            J.arc_base = I.arc_at_layer[nl + 1];
            J.num_arcs = I.arc_at_layer[nl + 2] - I.arc_at_layer[nl + 1];
        }
        J.item_base = I.layer_off[nl];
        J.num_items = I.nodes_in(nl);
        J.cur_base = I.layer_off[l];
        J.cur_nodes = I.nodes_in(l);
        J.cur_size = cur.second;
        // one block: per-arc candidate offsets | oversized list (released through the offsets)
        const size_t arc_bytes = align256(sizeof(int64_t) * (static_cast<size_t>(J.num_arcs) + 1));
        char *cb = static_cast<char *>(arena_.alloc(arc_bytes + sizeof(int64_t) * 2 * std::max(1, J.num_items)));
        new_arc_off[k] = reinterpret_cast<int64_t *>(cb);
        new_big[k] = cb ? reinterpret_cast<int64_t *>(cb + arc_bytes) : nullptr;
        if (!new_arc_off[k] || !new_big[k]) {
            count_alloc_ok = false;
            break;
        }
        J.arc_cand_off = new_arc_off[k];
        J.big_list = new_big[k];
        J.result = d_results + k;
    }
    // requests whose sides meet this step enter coupling now
    std::vector<Instance *> entering;
    for (const ExpPlan &e : exps) {
        Instance &I = *e.I;
        if (I.opts.method != 3) continue;
        const int td_layer = e.td ? e.nl : I.td.layer;
        const int bu_layer = e.td ? I.bu.layer : e.nl;
        if (td_layer == bu_layer) entering.push_back(&I);
    }

    // coupling descriptors (built after the expansion bookkeeping below swaps sides)
    const size_t n_couple_max = couplers.size() + entering.size();
    const size_t off_u = off_k;  // CoupleJob array
    const size_t off_ctrinit = align256(off_u + sizeof(dev::CoupleJob) * n_couple_max);
    stage_bytes = align256(off_ctrinit + sizeof(int64_t) * dev::kCtrCount * n_couple_max);

    // ------------------------------------------------------------ layer chains
    // A small step lets requests whose next count it computes (method 1, no state
    // dominance, not yet at the terminal) expand further layers before the read-back.
    std::vector<ChainGroup> chains;
    size_t chain_dev_bytes = 0, chain_slots = 0;
    char *d_chain = nullptr;
    auto release_slot = [&](ChainSlot &c) {
        for (int b = 0; b < 2; ++b)
            for (void *q : {c.pts[b], static_cast<void *>(c.off[b]), static_cast<void *>(c.size[b]),
                            static_cast<void *>(c.arc[b]), static_cast<void *>(c.big[b])})
                arena_.release(q);
    };
    auto release_chains = [&]() {
        for (auto &g : chains)
            for (auto &c : g.slots) release_slot(c);
        chains.clear();
    };
    if (chain_layers_ > 0 && count_alloc_ok && static_cast<int64_t>(exps.size()) <= chain_max_requests_) {
        for (size_t k = 0; k < counts.size(); ++k) {
            const CountPlan &cp = counts[k];
            if (!cp.after_expand) continue;
            Instance &I = *cp.I;
            if (I.opts.state_dominance > 0 || I.phase != Instance::RUNNING) continue;
            if (I.opts.method != 1 && I.opts.method != 3) continue;
            if (I.opts.method == 1 && !cp.td) continue;
            const int32_t ei = exp_index(I, cp.td);
            const ExpPlan *e = ei >= 0 ? &exps[ei] : nullptr;
            if (e == nullptr || e->cand > chain_max_cand_) continue;
            if (I.chain_skip > 0) {  // its last chain went nowhere (method 3): wait a little
                --I.chain_skip;
                continue;
            }
            ChainSlot c;
            c.I = &I;
            c.e = e;
            c.count_idx = k;
            c.dir = cp.td ? 1 : -1;
            // longer chains delay whatever else waits for the step: beyond the base length
            // only for a request the engine runs alone
            int32_t want = I.chain_len > 0 ? I.chain_len : (I.opts.method == 3 ? 2 : chain_layers_);
            if (!chain_grow_all_ && !(active_.size() == 1 && queued_.empty())) want = std::min(want, chain_layers_);
            if (I.opts.method == 1) {
                c.last = std::min<int32_t>(want, I.L - 1 - e->nl);
            } else {
                // method 3: the same side while the side rule picks it (checked on the
                // device), and stopping one layer short of the other side (the meeting
                // expansion and the cutset join are ordinary steps)
                const Side &o = cp.td ? I.bu : I.td;
                c.other_score = o.score;
                c.last = std::min<int32_t>(want, (cp.td ? o.layer - e->nl : e->nl - o.layer) - 1);
            }
            if (c.last <= 0) continue;
            c.cap = std::min<int64_t>(std::max<int64_t>(8 * std::max<int64_t>(e->cand, 1), 16384), int64_t(1) << 22);
            c.ntiles = c.cap / e->window + 2;
            for (int j = 1; j <= c.last; ++j) {
                const int x = e->nl + c.dir * j;  // the layer chained layer j writes
                c.vmax = std::max(c.vmax, I.nodes_in(x));
                const int y = x + c.dir;          // the layer its count counts
                if (y >= 0 && y <= I.L - 1) {
                    c.amax = std::max(c.amax, c.dir > 0 ? I.arc_at_layer[y + 1] - I.arc_at_layer[y]
                                                        : I.arc_at_layer[y + 2] - I.arc_at_layer[y + 1]);
                    c.cmax = std::max(c.cmax, I.nodes_in(y));
                }
            }
            bool okc = true;
            for (int b = 0; b < 2; ++b) {
                c.pts[b] = arena_.alloc(static_cast<size_t>(c.cap) * I.d * I.elem());
                c.off[b] = static_cast<int64_t *>(arena_.alloc(sizeof(int64_t) * static_cast<size_t>(c.vmax)));
                c.size[b] = static_cast<int32_t *>(
                    arena_.alloc(sizeof(int32_t) * static_cast<size_t>(c.vmax + c.ntiles + 1) + static_cast<size_t>(c.vmax)));
                c.arc[b] = static_cast<int64_t *>(arena_.alloc(sizeof(int64_t) * static_cast<size_t>(c.amax + 1)));
                c.big[b] = static_cast<int64_t *>(arena_.alloc(sizeof(int64_t) * 2 * static_cast<size_t>(std::max(1, c.cmax))));
                okc = okc && c.pts[b] && c.off[b] && c.size[b] && c.arc[b] && c.big[b];
            }
            if (!okc) {  // no room: this request and the rest take ordinary steps
                release_slot(c);
                break;
            }
            ChainGroup *g = nullptr;
            for (auto &x : chains)
                if (x.d == I.d && x.wide == I.wide) g = &x;
            if (g == nullptr) {
                chains.emplace_back();
                g = &chains.back();
                g->d = I.d;
                g->wide = I.wide;
            }
            if (static_cast<int>(g->slots.size()) >= dev::kChainThreads) {
                release_slot(c);
                continue;
            }
            g->slots.push_back(c);
        }
        for (auto &g : chains) {
            const size_t n = g.slots.size();
            g.first_slot = chain_slots;
            chain_slots += n;
            for (const auto &c : g.slots) g.layers = std::max(g.layers, c.last);
            g.layer_bytes = align256(sizeof(dev::ExpandJob) * n) + 2 * align256(sizeof(int64_t) * n) +
                            align256(sizeof(dev::CountJob) * n);
            g.st_off = stage_bytes;
            stage_bytes += g.layer_bytes * static_cast<size_t>(g.layers) + 2 * align256(sizeof(int64_t) * n) + 3 * g.n4();
            g.dv_off = chain_dev_bytes;
            g.dv_bytes = g.bytes();
            chain_dev_bytes += g.dv_bytes;
        }
        if (chain_dev_bytes > 0) {
            d_chain = static_cast<char *>(scratch(chain_dev_bytes));
            if (d_chain == nullptr) {
                release_chains();
                chain_dev_bytes = chain_slots = 0;
            }
        }
        if (chains.empty()) stage_bytes = align256(off_ctrinit + sizeof(int64_t) * dev::kCtrCount * n_couple_max);
    }
    // Every device and pinned allocation of the step is made here, before any side moves
    // or launch, so that running out of memory rolls the step back and fails one request
    // instead of the engine.
    char *d_stage = nullptr;
    // host summary (D2H): the summary block | coupling ctrs | finishing sizes (bounds:
    // every coupler, every expansion finishing)
    const size_t s_counts = 0, s_ts = f_ts, s_sd = f_sd, s_err = f_err;
    const size_t s_ctr = align256(f_total);
    const size_t s_fin = align256(s_ctr + sizeof(int64_t) * dev::kCtrCount * n_couple_max);
    // ... | the chain block | the terminal sizes of chained requests
    const size_t s_chain = align256(s_fin + sizeof(int32_t) * exps.size());
    const size_t s_chfin = s_chain + chain_dev_bytes;
    const size_t s_total = s_chfin + sizeof(int32_t) * chain_slots;
    // oversized path: per group, the size-order list and the mark-path plan
    std::vector<int32_t *> big_order(glaunch.size(), nullptr);
    std::vector<void *> big_plan(glaunch.size(), nullptr);
    if (count_alloc_ok) {
        if (stage_bytes) d_stage = static_cast<char *>(scratch(stage_bytes));
        if ((stage_bytes && !d_stage) || !h_desc_.reserve(stage_bytes) || !h_summary_.reserve(s_total))
            count_alloc_ok = false;
        for (size_t g = 0; g < glaunch.size() && count_alloc_ok; ++g) {
            const GroupLaunch &gl = glaunch[g];
            if (gl.big_count == 0) continue;
            const int64_t nw = static_cast<int64_t>(gl.big_count);
            if (nw > sms_ * 3 && nw <= dev::kBigOrderMax) {
                big_order[g] = static_cast<int32_t *>(scratch(sizeof(int32_t) * static_cast<size_t>(nw)));
                if (!big_order[g]) count_alloc_ok = false;
            }
            const int mark_cap = static_cast<int>(std::min<int64_t>(gl.mark_cap, nw));
            if (count_alloc_ok && mark_cap > 0) {
                big_plan[g] = scratch(dev::big_plan_bytes(mark_cap));
                if (!big_plan[g]) count_alloc_ok = false;
            }
        }
    }
    if (!count_alloc_ok) {
        // Out of device memory for bookkeeping: give everything back and fail the
        // largest blocked request so the others can progress next step.
        for (size_t k = 0; k < counts.size(); ++k) {
            arena_.release(new_arc_off[k]);
            arena_.release(new_big[k]);
        }
        for (const ExpPlan &e : exps) {
            for (void *q : {e.out_pts, static_cast<void *>(e.out_off), static_cast<void *>(e.out_size), e.big_mem})
                arena_.release(q);
        }
        release_chains();
        for (void *q : step_scratch_) arena_.release(q);
        step_scratch_.clear();
        // the request with the largest expansion of this step (else the last one counted)
        Instance *victim = counts.empty() ? nullptr : counts.back().I;
        int64_t most = -1;
        for (const ExpPlan &e : exps)
            if (e.cand > most) {
                most = e.cand;
                victim = e.I;
            }
        if (victim) fail(*victim, PMDD_ERR_OOM, "device memory budget exhausted");
        int done = 0;
        for (auto it = active_.begin(); it != active_.end();) {
            if ((*it)->phase == Instance::DONE) {
                release_instance(**it);
                (*it)->finish_s = now_s();
                record_finish(**it);
                finished_.push_back(std::move(*it));
                it = active_.erase(it);
                ++done;
            } else {
                ++it;
            }
        }
        return done;
    }

    char *hs = static_cast<char *>(h_desc_.p);
    if (!xjobs.empty()) std::memcpy(hs + off_x, xjobs.data(), sizeof(dev::ExpandJob) * xjobs.size());
    if (!bigwork.empty()) std::memcpy(hs + off_b, bigwork.data(), sizeof(dev::BigWork) * bigwork.size());
    if (!cjobs.empty()) std::memcpy(hs + off_c, cjobs.data(), sizeof(dev::CountJob) * cjobs.size());
    if (!tile_bases.empty()) {
        std::memcpy(hs + off_tb, tile_bases.data(), sizeof(int64_t) * tile_bases.size());
        std::memcpy(hs + off_ib, item_bases.data(), sizeof(int64_t) * item_bases.size());
        std::memcpy(hs + off_bb, big_bases.data(), sizeof(int64_t) * big_bases.size());
    }
    if (!sdjobs.empty()) {
        std::memcpy(hs + off_sd, sdjobs.data(), sizeof(dev::StateDomJob) * sdjobs.size());
        std::memcpy(hs + off_sdb, sd_bases.data(), sizeof(int64_t) * sd_bases.size());
    }
    // chained layers: every descriptor but the sizes the prep kernel fills in
    for (auto &g : chains) {
        const size_t n = g.slots.size();
        char *dv = d_chain + g.dv_off;
        dev::CountResult *dR = reinterpret_cast<dev::CountResult *>(dv);
        int32_t *dstop = reinterpret_cast<int32_t *>(dv + g.off_stop());
        int32_t *dstopped = reinterpret_cast<int32_t *>(dv + g.off_stopped());
        unsigned long long *dts = reinterpret_cast<unsigned long long *>(dv + g.off_ts());
        int64_t *dtiles = reinterpret_cast<int64_t *>(dv + g.off_tiles());
        int64_t *dnt = reinterpret_cast<int64_t *>(dv + g.off_nt());
        unsigned int *ddone = reinterpret_cast<unsigned int *>(dv + g.off_done());
        g.items.assign(static_cast<size_t>(g.layers) + 1, 0);
        g.tiles.assign(static_cast<size_t>(g.layers) + 1, 0);
        for (int j = 1; j <= g.layers; ++j) {
            char *hl = hs + g.st_off + g.layer_bytes * static_cast<size_t>(j - 1);
            dev::ExpandJob *hx = reinterpret_cast<dev::ExpandJob *>(hl);
            int64_t *hib = reinterpret_cast<int64_t *>(hl + align256(sizeof(dev::ExpandJob) * n) +
                                                       align256(sizeof(int64_t) * n));
            dev::CountJob *hc = reinterpret_cast<dev::CountJob *>(hl + align256(sizeof(dev::ExpandJob) * n) +
                                                                 2 * align256(sizeof(int64_t) * n));
            for (size_t i = 0; i < n; ++i) {
                ChainSlot &c = g.slots[i];
                Instance &I = *c.I;
                const int b = j % 2, pb = (j - 1) % 2;
                dev::ExpandJob &J = hx[i];
                dev::CountJob &C = hc[i];
                std::memset(&J, 0, sizeof(J));
                std::memset(&C, 0, sizeof(C));
                hib[i] = g.items[j];
                J.tile_window = c.e->window;
                J.err = d_err_step;
                J.tile_surv = dts + 2 * (static_cast<size_t>(j - 1) * n + i);
                C.stop = dstop + i;
                C.stopped_at = dstopped + i;
                C.result = dR + static_cast<size_t>(j - 1) * n + i;
                if (j < g.layers) {  // the count sizes and plans this request's next chained expansion
                    char *dn = d_stage + g.st_off + g.layer_bytes * static_cast<size_t>(j);
                    C.next = reinterpret_cast<dev::ExpandJob *>(dn) + i;
                    C.next_tiles = dnt + static_cast<size_t>(j - 1) * n;
                    C.next_bases = reinterpret_cast<int64_t *>(dn + align256(sizeof(dev::ExpandJob) * n));
                    C.next_total = dtiles + j;
                    C.done = ddone + (j - 1);
                    C.cap = c.cap;
                    C.next_layer = j + 1;
                    C.last = c.last;
                    C.slot = static_cast<int32_t>(i);
                    C.chain_n = static_cast<int32_t>(n);
                    C.bu = c.dir < 0 ? 1 : 0;
                    C.other_score = c.other_score;
                }
                C.arc_cand_off = c.arc[b];
                C.big_list = c.big[b];
                J.tile_first = c.size[b];
                if (j > c.last) continue;  // past its last layer: the prep stops it
                const int cur = c.e->nl + c.dir * (j - 1), nl = cur + c.dir;
                if (c.dir > 0) {
                    J.item_arc_off = I.d_in_off;
                    J.arc_nbr = I.d_arc_src;
                    J.arc_wrow = I.d_arc_w;
                    J.arc_base = I.arc_at_layer[nl];
                } else {
                    J.item_arc_off = I.d_out_off;
                    J.arc_nbr = I.d_out_head;
                    J.arc_wrow = I.d_out_w;
                    J.arc_base = I.arc_at_layer[nl + 1];
                }
                J.weights = I.d_weights;
                J.arc_cand_off = j == 1 ? new_arc_off[c.count_idx] : c.arc[pb];
                J.item_base = I.layer_off[nl];
                J.num_items = I.nodes_in(nl);
                J.prev_base = I.layer_off[cur];
                J.prev_pts = j == 1 ? c.e->out_pts : c.pts[pb];
                J.prev_off = j == 1 ? c.e->out_off : c.off[pb];
                J.prev_size = j == 1 ? c.e->out_size : c.size[pb];
                J.prev_sorted = j == 1 ? c.e->out_sorted : c.sorted(pb);
                J.out_pts = c.pts[b];
                J.out_off = c.off[b];
                J.out_size = c.size[b];
                J.out_sorted = c.sorted(b);
                J.tile_first = c.size[b] + J.num_items;
                J.big_list = j == 1 ? new_big[c.count_idx] : c.big[pb];
                J.pair_max = pair_max_for(I.d, I.opts.problem_type);
                J.lex_big = (I.d == 3 && lex_tiles_) ? 1 : 0;
                J.lex_bulk = lex_bulk_ ? 1 : 0;
                J.lex_max_arcs = lex_max_arcs_;
                g.items[j] += J.num_items;
                g.tiles[j] += c.ntiles;
                const int y = nl + c.dir;  // the layer after it in this direction
                if (y >= 0 && y <= I.L - 1) {  // its count (none past the terminal)
                    if (c.dir > 0) {
                        C.item_arc_off = I.d_in_off;
                        C.arc_nbr = I.d_arc_src;
                        C.arc_base = I.arc_at_layer[y];
                        C.num_arcs = I.arc_at_layer[y + 1] - I.arc_at_layer[y];
                    } else {
                        C.item_arc_off = I.d_out_off;
                        C.arc_nbr = I.d_out_head;
                        C.arc_base = I.arc_at_layer[y + 1];
                        C.num_arcs = I.arc_at_layer[y + 2] - I.arc_at_layer[y + 1];
                    }
                    C.item_base = I.layer_off[y];
                    C.num_items = I.nodes_in(y);
                    C.cur_base = I.layer_off[nl];
                    C.cur_nodes = I.nodes_in(nl);
                    C.cur_size = c.size[b];
                }
            }
        }
        char *hp = hs + g.st_off + g.layer_bytes * static_cast<size_t>(g.layers);
        int64_t *hcap = reinterpret_cast<int64_t *>(hp);
        int32_t *hlast = reinterpret_cast<int32_t *>(hp + align256(sizeof(int64_t) * n));
        int32_t *hidx = reinterpret_cast<int32_t *>(hp + align256(sizeof(int64_t) * n) + g.n4());
        int64_t *hother = reinterpret_cast<int64_t *>(hp + align256(sizeof(int64_t) * n) + 2 * g.n4());
        int32_t *hbu = reinterpret_cast<int32_t *>(hp + 2 * align256(sizeof(int64_t) * n) + 2 * g.n4());
        for (size_t i = 0; i < n; ++i) {
            hcap[i] = g.slots[i].cap;
            hlast[i] = g.slots[i].last;
            hidx[i] = static_cast<int32_t>(g.slots[i].count_idx);
            hother[i] = g.slots[i].other_score;
            hbu[i] = g.slots[i].dir < 0 ? 1 : 0;
        }
    }

    // ------------------------------------------------- expansion bookkeeping
    // Sides move to their new layer now (host view); device work is stream-ordered.
    std::vector<Instance *> finishing;  // method 1 reached the terminal
    std::vector<void *> to_release;
    for (const ExpPlan &e : exps) {
        Instance &I = *e.I;
        Side &s = e.td ? I.td : I.bu;
        to_release.push_back(s.pts);
        to_release.push_back(s.off);
        to_release.push_back(s.size);
        to_release.push_back(s.arc_off);
        to_release.push_back(s.big_list);
        to_release.push_back(e.big_mem);
        I.stats.work_candidates_total += s.res.total;
        I.stats.work_candidates_peak = std::max(I.stats.work_candidates_peak, s.res.total);
        I.peak_cand = std::max(I.peak_cand, s.res.total);
        s.slot_points = std::max<int64_t>(e.cand, 1);
        s.pts = e.out_pts;
        s.off = e.out_off;
        s.size = e.out_size;
        s.sorted = e.out_sorted;
        s.arc_off = nullptr;
        s.big_list = nullptr;
        s.counted = false;
        s.layer = e.nl;
        if (e.td) I.stats.layers_td++;
        else I.stats.layers_bu++;
        if (I.opts.method == 1 && e.nl == I.L - 1) finishing.push_back(&I);
    }
    for (Instance *I : entering) {
        I->phase = Instance::COUPLING;
        I->stats.layer_coupling = I->td.layer;
        I->stats.cutset_size = I->nodes_in(I->td.layer);
        // running frontier + one round of survivors; the seed round needs d+1 per node
        const int64_t ucap = std::max<int64_t>(1 << 17, static_cast<int64_t>(I->stats.cutset_size) * (I->d + 1) + 4096);
        I->cu_ctr = static_cast<int64_t *>(arena_.alloc(sizeof(int64_t) * dev::kCtrCount));
        if (!I->cu_ctr || !carve_couple(*I, ucap)) {
            fail(*I, PMDD_ERR_OOM, "device memory budget exhausted at the cutset join");
            continue;
        }
        couplers.push_back(I);
    }
    std::vector<dev::CoupleJob> ujobs;
    std::vector<Instance *> ujob_inst;
    std::vector<int> ujob_new;
    for (Instance *I : couplers) {
        if (I->phase != Instance::COUPLING) continue;
        dev::CoupleJob J;
        std::memset(&J, 0, sizeof(J));
        J.td_pts = I->td.pts;
        J.td_off = I->td.off;
        J.td_size = I->td.size;
        J.bu_pts = I->bu.pts;
        J.bu_off = I->bu.off;
        J.bu_size = I->bu.size;
        J.num_nodes = I->nodes_in(I->td.layer);
        J.U = I->cu_U;
        J.U_alt = I->cu_U_alt;
        J.ucap = I->cu_ucap;
        J.sc_pts2 = I->cu_p2;
        J.sc_surv = I->cu_sv;
        J.sc_idx = I->cu_i2;
        J.sc_sidx = I->cu_si;
        J.sc_hist = I->cu_hist;
        J.ctr = I->cu_ctr;
        // the next running frontier lands in U_alt: swap now (host view)
        std::swap(I->cu_U, I->cu_U_alt);
        const bool is_new = std::find(entering.begin(), entering.end(), I) != entering.end();
        int64_t *ci = reinterpret_cast<int64_t *>(hs + off_ctrinit) + dev::kCtrCount * ujobs.size();
        std::memset(ci, 0, sizeof(int64_t) * dev::kCtrCount);
        ci[dev::kCtrResume] = J.num_nodes;
        ci[dev::kCtrValidEnd] = J.ucap;
        ujobs.push_back(J);
        ujob_inst.push_back(I);
        ujob_new.push_back(is_new ? 1 : 0);
    }
    if (!ujobs.empty()) std::memcpy(hs + off_u, ujobs.data(), sizeof(dev::CoupleJob) * ujobs.size());

    // ----------------------------------------------------------- device work
    cudaEvent_t ev0 = ev_[0], ev1 = ev_[1], ev2 = ev_[2], ev3 = ev_[3];
    const double t_issue = trace_ ? now_s() : 0.0;  // host planning done
    if (stage_bytes && !cuda_ok(cudaMemcpyAsync(d_stage, hs, stage_bytes, cudaMemcpyHostToDevice, stream_), "H2D"))
        return -1;
    // coupling counters of requests that just reached their cutset start from the staged init values
    for (size_t k = 0; k < ujobs.size(); ++k) {
        if (!ujob_new[k]) continue;
        cudaMemcpyAsync(ujobs[k].ctr, d_stage + off_ctrinit + sizeof(int64_t) * dev::kCtrCount * k,
                        sizeof(int64_t) * dev::kCtrCount, cudaMemcpyDeviceToDevice, stream_);
    }
    cudaMemsetAsync(d_fixed + f_ts, 0, f_total - f_ts, stream_);
    cudaEventRecord(ev0, stream_);
    for (size_t gi = 0; gi < glaunch.size(); ++gi) {
        const GroupLaunch &gl = glaunch[gi];
        unsigned long long *queue = reinterpret_cast<unsigned long long *>(d_fixed + f_q) + gi;
        const dev::ExpandJob *dj = reinterpret_cast<const dev::ExpandJob *>(d_stage + off_x) + gl.first;
        const int64_t *dtb = reinterpret_cast<const int64_t *>(d_stage + off_tb) + gl.first;
        const int64_t *dib = reinterpret_cast<const int64_t *>(d_stage + off_ib) + gl.first;
        if (!cuda_ok(dev::launch_tile_plan(dj, dib, static_cast<int>(gl.count), gl.items, stream_), "tile_plan_kernel"))
            return -1;
        // blocks beyond the tiles would only be scheduled to exit (several waves of them at
        // the tiles' shared-memory size cost more than a small step's work)
        const int grid = static_cast<int>(std::min<int64_t>(sms_ * 8, std::max<int64_t>(1, gl.tiles)));
        const bool lex = lex_tiles_for(gl.d, gl.wide);
        const cudaError_t te =
            lex ? dev::launch_expand_tiles_lex(gl.d, gl.wide, dj, dtb, static_cast<int>(gl.count), gl.tiles, grid, queue,
                                               nullptr, stream_)
                : dev::launch_expand_tiles(gl.d, gl.wide, dj, dtb, static_cast<int>(gl.count), gl.tiles, grid, queue,
                                           nullptr, stream_);
        if (!cuda_ok(te, lex ? "expand_tile_lex_kernel" : "expand_tile_kernel")) return -1;
        launches_ += 2;
        ktimes_.tile_launches += 1;
    }
    cudaEventRecord(ev1, stream_);
    for (size_t g = 0; g < glaunch.size(); ++g) {
        const GroupLaunch &gl = glaunch[g];
        if (gl.big_count == 0) continue;
        const dev::ExpandJob *dj = reinterpret_cast<const dev::ExpandJob *>(d_stage + off_x) + gl.first;
        dev::BigLaunch L;
        L.jobs = dj;
        L.work = reinterpret_cast<const dev::BigWork *>(d_stage + off_b) + gl.big_first;
        L.num_work = static_cast<int>(gl.big_count);
        L.job_bases = reinterpret_cast<const int64_t *>(d_stage + off_bb) + gl.first;
        L.num_jobs = static_cast<int>(gl.count);
        L.total = gl.big_rows;
        L.sms = sms_;
        L.with_sfs = true;
        L.lex_big = gl.d == 3 && lex_tiles_;
        L.lex_rounds = L.lex_big ? dev::lex_merge_rounds(std::min(gl.max_big_arcs, lex_max_arcs_)) : 0;
        L.mark_cap = static_cast<int>(std::min<int64_t>(gl.mark_cap, static_cast<int64_t>(gl.big_count)));
        L.plan = nullptr;
        // more SFS blocks than fit the SMs at once: start the largest destinations first
        L.order = big_order[g];
        const bool ordered = L.order != nullptr;
        L.plan = big_plan[g];
        for (int64_t pass = 0; pass < gl.big_passes; ++pass) {
            L.pass = pass;
            if (!cuda_ok(dev::launch_big(gl.d, gl.wide, L, stream_), "oversized-destination kernels")) return -1;
            launches_ += (L.mark_cap > 0 ? 9 : 2) + (ordered ? 1 : 0) + (L.lex_big ? 1 + L.lex_rounds : 0);
        }
    }
    if (!sdjobs.empty()) {
        for (const SdGroup &g : sdg) {
            const dev::StateDomJob *dj = reinterpret_cast<const dev::StateDomJob *>(d_stage + off_sd) + g.first;
            const int64_t *db = reinterpret_cast<const int64_t *>(d_stage + off_sdb) + g.first;
            if (!cuda_ok(dev::launch_state_dominance(g.d, g.wide, dj, db, static_cast<int>(g.count), g.total, sms_,
                                                     stream_),
                         "state dominance"))
                return -1;
            launches_ += 2;
        }
    }
    cudaEventRecord(ev2, stream_);
    if (!cjobs.empty()) {
        if (!cuda_ok(dev::launch_count_scan(reinterpret_cast<const dev::CountJob *>(d_stage + off_c),
                                            static_cast<int>(cjobs.size()), stream_),
                     "count_scan_kernel"))
            return -1;
        launches_ += 1;
    }
    // coupling rounds, grouped by (d, wide, seed round)
    {
        std::map<std::tuple<int, bool, bool>, std::vector<size_t>> ug;
        for (size_t k = 0; k < ujobs.size(); ++k)
            ug[std::make_tuple(ujob_inst[k]->d, ujob_inst[k]->wide, ujob_inst[k]->couple_rounds == 0)].push_back(k);
        const dev::CoupleJob *du = reinterpret_cast<const dev::CoupleJob *>(d_stage + off_u);
        // new requests: product statistics once
        for (size_t k = 0; k < ujobs.size(); ++k) {
            if (!ujob_new[k]) continue;
            dev::launch_couple_products(du + k, 1, stream_);
            launches_ += 1;
        }
        for (auto &g : ug) {
            // jobs of one group are contiguous only if sorted; launch per job run
            size_t i = 0;
            while (i < g.second.size()) {
                size_t j = i;
                while (j + 1 < g.second.size() && g.second[j + 1] == g.second[j] + 1) ++j;
                const int n = static_cast<int>(j - i + 1);
                // three 256-thread blocks per SM: the prune kernel's register limit
                const int per = std::max(1, (sms_ * 3) / n);
                if (!cuda_ok(dev::launch_couple_round(std::get<0>(g.first), std::get<1>(g.first), du + g.second[i], n,
                                                      per, std::get<2>(g.first), stream_),
                             "coupling round"))
                    return -1;
                launches_ += 7;
                i = j + 1;
            }
        }
    }
    cudaEventRecord(ev3, stream_);
    // chained layers, per layer and group: the tiles and the counts of the layer after
    // (which size and plan the next layer); the first layer is sized and planned by its own
    // two kernels from the step's counts
    int32_t chain_layers_run = 0;
    if (!chains.empty()) {
        cudaEventRecord(ev_[4], stream_);
        cudaMemsetAsync(d_chain, 0, chain_dev_bytes, stream_);
        for (const auto &g : chains) chain_layers_run = std::max(chain_layers_run, g.layers);
        for (int j = 1; j <= chain_layers_run; ++j) {
            for (const auto &g : chains) {
                if (j > g.layers) continue;
                const size_t n = g.slots.size();
                char *dl = d_stage + g.st_off + g.layer_bytes * static_cast<size_t>(j - 1);
                char *dv = d_chain + g.dv_off;
                char *dp = d_stage + g.st_off + g.layer_bytes * static_cast<size_t>(g.layers);
                dev::ExpandJob *dj = reinterpret_cast<dev::ExpandJob *>(dl);
                int64_t *dtb = reinterpret_cast<int64_t *>(dl + align256(sizeof(dev::ExpandJob) * n));
                const int64_t *dib = dtb + align256(sizeof(int64_t) * n) / sizeof(int64_t);
                const dev::CountJob *dc = reinterpret_cast<const dev::CountJob *>(
                    dl + align256(sizeof(dev::ExpandJob) * n) + 2 * align256(sizeof(int64_t) * n));
                const dev::CountResult *dR = reinterpret_cast<const dev::CountResult *>(dv);
                // chain block after the survivor counters: tile queue per layer, tiles per layer
                unsigned long long *queue = reinterpret_cast<unsigned long long *>(dv + g.off_queue()) + (j - 1);
                int64_t *tiles_dev = reinterpret_cast<int64_t *>(dv + g.off_tiles()) + (j - 1);
                dev::ChainPrep P;
                P.jobs = dj;
                P.tile_bases = dtb;
                P.tiles_total = tiles_dev;
                P.prev = j == 1 ? d_results : dR + static_cast<size_t>(j - 2) * n;
                P.prev_idx = j == 1 ? reinterpret_cast<const int32_t *>(dp + align256(sizeof(int64_t) * n) + g.n4())
                                    : nullptr;
                P.stop = reinterpret_cast<int32_t *>(dv + g.off_stop());
                P.stopped_at = reinterpret_cast<int32_t *>(dv + g.off_stopped());
                P.cap = reinterpret_cast<const int64_t *>(dp);
                P.last = reinterpret_cast<const int32_t *>(dp + align256(sizeof(int64_t) * n));
                P.other_score = reinterpret_cast<const int64_t *>(dp + align256(sizeof(int64_t) * n) + 2 * g.n4());
                P.bu = reinterpret_cast<const int32_t *>(dp + 2 * align256(sizeof(int64_t) * n) + 2 * g.n4());
                P.layer = j;
                P.n = static_cast<int32_t>(n);
                if (j == 1) {  // later layers are sized and planned by the count before them
                    if (!cuda_ok(dev::launch_chain_prep(P, stream_), "chain_prep_kernel")) return -1;
                    if (!cuda_ok(dev::launch_tile_plan(dj, dib, static_cast<int>(n), g.items[j], stream_),
                                 "tile_plan_kernel"))
                        return -1;
                    launches_ += 2;
                }
                const bool lex = lex_tiles_for(g.d, g.wide);
                // the tiles' bound assumes full buffers: one wave of blocks loops over them
                const int grid = static_cast<int>(std::min<int64_t>(sms_ * 2, std::max<int64_t>(1, g.tiles[j])));
                const cudaError_t te =
                    lex ? dev::launch_expand_tiles_lex(g.d, g.wide, dj, dtb, static_cast<int>(n), g.tiles[j], grid, queue,
                                                       tiles_dev, stream_)
                        : dev::launch_expand_tiles(g.d, g.wide, dj, dtb, static_cast<int>(n), g.tiles[j], grid, queue,
                                                   tiles_dev, stream_);
                if (!cuda_ok(te, lex ? "expand_tile_lex_kernel" : "expand_tile_kernel")) return -1;
                if (!cuda_ok(dev::launch_count_scan(dc, static_cast<int>(n), stream_), "count_scan_kernel")) return -1;
                launches_ += 2;
                ktimes_.tile_launches += 1;
            }
        }
        cudaEventRecord(ev_[5], stream_);
    }
    char *hsum = static_cast<char *>(h_summary_.p);
    cudaMemcpyAsync(hsum + s_counts, d_fixed, f_total, cudaMemcpyDeviceToHost, stream_);
    for (size_t k = 0; k < ujobs.size(); ++k)
        cudaMemcpyAsync(hsum + s_ctr + sizeof(int64_t) * dev::kCtrCount * k, ujobs[k].ctr,
                        sizeof(int64_t) * dev::kCtrCount, cudaMemcpyDeviceToHost, stream_);
    for (size_t k = 0; k < finishing.size(); ++k)
        cudaMemcpyAsync(hsum + s_fin + sizeof(int32_t) * k, finishing[k]->td.size, sizeof(int32_t),
                        cudaMemcpyDeviceToHost, stream_);
    if (!chains.empty()) {
        cudaMemcpyAsync(hsum + s_chain, d_chain, chain_dev_bytes, cudaMemcpyDeviceToHost, stream_);
        for (const auto &g : chains)
            for (size_t i = 0; i < g.slots.size(); ++i) {
                const ChainSlot &c = g.slots[i];
                if (c.e->nl + c.last == c.I->L - 1)  // the chain may reach the terminal node
                    cudaMemcpyAsync(hsum + s_chfin + sizeof(int32_t) * (g.first_slot + i), c.size[c.last % 2],
                                    sizeof(int32_t), cudaMemcpyDeviceToHost, stream_);
            }
    }
    const double t_rel = trace_ ? now_s() : 0.0;
    for (void *q : to_release) arena_.release(q);
    const double t_enq = trace_ ? now_s() : 0.0;  // every copy and launch enqueued
    const cudaError_t se = cudaStreamSynchronize(stream_);
    const double t_sync = trace_ ? now_s() : 0.0;
    if (!cuda_ok(se, "engine step")) {
        for (auto &p : active_) fail(*p, PMDD_ERR_CUDA, error_);
        return -1;
    }
    float ms_expand = 0, ms_big = 0, ms_rest = 0;
    cudaEventElapsedTime(&ms_expand, ev0, ev1);
    cudaEventElapsedTime(&ms_big, ev1, ev2);
    cudaEventElapsedTime(&ms_rest, ev2, ev3);
    ktimes_.expand += ms_expand * 1e-3;
    ktimes_.big += ms_big * 1e-3;
    ktimes_.rest += ms_rest * 1e-3;
    float ms_chain = 0;
    if (!chains.empty()) cudaEventElapsedTime(&ms_chain, ev_[4], ev_[5]);
    ktimes_.expand += ms_chain * 1e-3;
    if (trace_) {
        int64_t cand = 0, big_cand = 0, max_item = 0, nbig = 0;
        for (const ExpPlan &e : exps) {
            const Side &s = e.td ? e.I->td : e.I->bu;  // already moved: stats come from the plan
            (void)s;
            cand += e.cand;
            big_cand += e.big_total;
            max_item = std::max(max_item, e.max_item);
            nbig += e.num_big;
        }
        long long step_tiles = 0;
        for (const GroupLaunch &gl : glaunch) step_tiles += gl.tiles;
        unsigned long long tile_surv = 0;
        for (size_t k = 0; k < exps.size(); ++k)
            tile_surv += reinterpret_cast<const unsigned long long *>(static_cast<char *>(h_summary_.p) + s_ts)[2 * k];
        const unsigned long long *pc = reinterpret_cast<const unsigned long long *>(static_cast<char *>(h_summary_.p) + f_clk);
        std::fprintf(stderr,
                     "[pmdd step] jobs=%zu counts=%zu couple=%zu cand=%lld big_items=%lld big_cand=%lld max_item=%lld "
                     "tile_cand=%lld tile_surv=%llu tiles=%lld tiles_ms=%.3f big_ms=%.3f rest_ms=%.3f host_to_sync_us=%.1f "
                     "plan_us=%.1f plan_exp_us=%.1f enqueue_us=%.1f release_us=%.1f wait_us=%.1f prev_post_us=%.1f "
                     "arena_reserved_mb=%.0f arena_grow_ms=%.1f phase_mcyc=%.2f,%.2f,%.2f,%.2f,%.2f,%.2f,%.2f warp_mcyc=%.2f,%.2f\n",
                     exps.size(), counts.size(), ujobs.size(), static_cast<long long>(cand),
                     static_cast<long long>(nbig), static_cast<long long>(big_cand), static_cast<long long>(max_item),
                     static_cast<long long>(cand - big_cand), tile_surv, step_tiles, ms_expand, ms_big, ms_rest,
                     (now_s() - step_t0) * 1e6, (t_issue - step_t0) * 1e6, (t_p1 - step_t0) * 1e6,
                     (t_rel - t_issue) * 1e6, (t_enq - t_rel) * 1e6, (t_sync - t_enq) * 1e6, last_post_us_,
                     arena_.reserved() / 1e6, arena_.grow_seconds() * 1e3,
                     pc[0] * 1e-6, pc[1] * 1e-6, pc[2] * 1e-6, pc[3] * 1e-6, pc[4] * 1e-6, pc[5] * 1e-6, pc[6] * 1e-6,
                     pc[7] * 1e-6, pc[8] * 1e-6);
    }
    for (void *q : step_scratch_) arena_.release(q);
    step_scratch_.clear();

    // ----------------------------------------------------------- host updates
    const uint32_t errw = *reinterpret_cast<uint32_t *>(hsum + s_err);
    if (errw != 0) {
        const bool timeout = (errw & dev::kErrTimeout) != 0 && (errw & ~dev::kErrTimeout) == 0;
        for (auto &p : active_)
            if (p->phase != Instance::DONE) {
                if (timeout) fail(*p, PMDD_ERR_TIMEOUT, "a bounded device wait gave up (bulk-copy staging)");
                else fail(*p, PMDD_ERR_INTERNAL, "device-side index check failed");
            }
    }
    for (size_t k = 0; k < exps.size(); ++k) {
        const ExpPlan &e = exps[k];
        e.I->stats.kernel_expand_td_s += ms_expand * 1e-3;
        e.I->stats.kernel_dominance_s += ms_big * 1e-3;
        e.I->stats.kernel_total_s += (ms_expand + ms_big + ms_rest) * 1e-3;
        e.I->stats.work_tile_candidates_total += e.cand - e.big_total;
        e.I->stats.work_tile_survivors_total +=
            static_cast<int64_t>(reinterpret_cast<const unsigned long long *>(hsum + s_ts)[2 * k]);
        e.I->stats.work_stair_candidates_total +=
            static_cast<int64_t>(reinterpret_cast<const unsigned long long *>(hsum + s_ts)[2 * k + 1]);
    }
    for (size_t k = 0; k < sdjobs.size(); ++k)
        sd_inst[k]->stats.dominance_filtered_total += reinterpret_cast<const int64_t *>(hsum + s_sd)[k];
    const dev::CountResult *hres = reinterpret_cast<const dev::CountResult *>(hsum + s_counts);
    for (size_t k = 0; k < counts.size(); ++k) {
        Instance &I = *counts[k].I;
        Side &s = counts[k].td ? I.td : I.bu;
        s.arc_off = new_arc_off[k];
        s.big_list = new_big[k];
        s.res = hres[k];
        s.counted = true;
        if (counts[k].after_expand) {
            s.score = counts[k].td ? s.res.total : static_cast<int64_t>(1.5 * static_cast<double>(s.res.total));
            I.stats.work_frontier_survivors_total += s.res.cur_total;
            I.stats.work_frontier_peak_points = std::max(I.stats.work_frontier_peak_points, s.res.cur_total);
        }
    }
    // frontiers of the requests this step finishes: fetched together below (one pinned
    // buffer, one synchronisation) instead of one blocking copy each
    std::vector<std::pair<Instance *, const void *>> fetches;
    auto fetch = [&](Instance &I, const void *src) {
        if (!I.result.empty()) fetches.push_back({&I, src});
    };
    for (size_t k = 0; k < finishing.size(); ++k) {
        Instance &I = *finishing[k];
        if (I.phase == Instance::DONE) continue;
        const int32_t n = *reinterpret_cast<const int32_t *>(hsum + s_fin + sizeof(int32_t) * k);
        I.result_n = n;
        I.result.resize(static_cast<size_t>(n) * I.d * I.elem());
        fetch(I, I.td.pts);
        I.stats.work_frontier_survivors_total += n;
        I.stats.work_frontier_peak_points = std::max<int64_t>(I.stats.work_frontier_peak_points, n);
        I.phase = Instance::DONE;
    }
    for (size_t k = 0; k < ujobs.size(); ++k) {
        Instance &I = *ujob_inst[k];
        if (I.phase == Instance::DONE) continue;
        const int64_t *c = reinterpret_cast<const int64_t *>(hsum + s_ctr + sizeof(int64_t) * dev::kCtrCount * k);
        I.couple_rounds++;
        if (ujob_new[k]) I.stats.work_join_products_total = c[dev::kCtrProducts];
        if (c[dev::kCtrDone]) {
            const int64_t n = c[dev::kCtrF];
            I.result_n = n;
            I.result.resize(static_cast<size_t>(n) * I.d * I.elem());
            fetch(I, I.cu_U);
            I.stats.work_frontier_survivors_total += n;
            I.stats.work_frontier_peak_points = std::max<int64_t>(I.stats.work_frontier_peak_points, n);
            I.phase = Instance::DONE;
        } else if (c[dev::kCtrF] > I.cu_ucap / 2) {
            // the running frontier crowds out the survivors of a round: grow the block
            I.result_n = c[dev::kCtrF];
            const bool grown = carve_couple(I, I.cu_ucap * 2);
            I.result_n = 0;
            if (!grown) {
                fail(I, PMDD_ERR_OOM, "device memory budget exhausted growing the cutset frontier");
                continue;
            }
            const int64_t ncap = I.cu_ucap;
            // ValidEnd must follow the capacity
            int64_t *hv = reinterpret_cast<int64_t *>(h_init_.p) + 24;  // scratch slot in the init block
            *hv = ncap;
            cudaMemcpyAsync(I.cu_ctr + dev::kCtrValidEnd, hv, sizeof(int64_t), cudaMemcpyHostToDevice, stream_);
            cudaStreamSynchronize(stream_);
        }
    }
    // chained requests move to the last layer they finished
    int64_t chained_done = 0;
    for (auto &g : chains) {
        const size_t n = g.slots.size();
        const char *hv = hsum + s_chain + g.dv_off;
        const dev::CountResult *R = reinterpret_cast<const dev::CountResult *>(hv);
        const int32_t *stopped = reinterpret_cast<const int32_t *>(hv + g.off_stopped());
        const unsigned long long *ts = reinterpret_cast<const unsigned long long *>(hv + g.off_ts());
        for (size_t i = 0; i < n; ++i) {
            ChainSlot &c = g.slots[i];
            Instance &I = *c.I;
            const int32_t done = stopped[i] == 0 ? c.last : stopped[i] - 1;
            // next chain: twice as long after one that ran to its end, one layer past
            // where it stopped otherwise.  Method 3 grows from its last length and, after a
            // chain that went nowhere (the other side was due at once), skips two steps:
            // its sides alternate, and a chain that stops at once only costs launches.
            if (I.opts.method == 3) {
                I.chain_len = done == c.last ? std::min(kChainMaxLayers, 2 * c.last) : std::max(1, done + 1);
                if (done == 0) I.chain_skip = 2;
            } else {
                I.chain_len = done == c.last ? std::min(kChainMaxLayers, 2 * std::max(c.last, chain_layers_))
                                             : std::max(1, done + 1);
            }
            if (I.phase != Instance::RUNNING || done <= 0) {
                release_slot(c);
                continue;
            }
            Side &s = c.dir > 0 ? I.td : I.bu;
            int64_t C = 0;
            for (int j = 1; j <= done; ++j) {
                C = j == 1 ? hres[c.count_idx].total : R[static_cast<size_t>(j - 2) * n + i].total;
                const size_t t = 2 * (static_cast<size_t>(j - 1) * n + i);
                I.stats.work_candidates_total += C;
                I.stats.work_candidates_peak = std::max(I.stats.work_candidates_peak, C);
                I.peak_cand = std::max(I.peak_cand, C);
                I.stats.work_tile_candidates_total += C;
                I.stats.work_tile_survivors_total += static_cast<int64_t>(ts[t]);
                I.stats.work_stair_candidates_total += static_cast<int64_t>(ts[t + 1]);
                if (c.dir > 0) I.stats.layers_td++;
                else I.stats.layers_bu++;
                I.stats.work_chained_layers++;
                const int y = c.e->nl + c.dir * (j + 1);  // the layer its count counted
                if (y >= 0 && y <= I.L - 1) {
                    const int64_t surv = R[static_cast<size_t>(j - 1) * n + i].cur_total;
                    I.stats.work_frontier_survivors_total += surv;
                    I.stats.work_frontier_peak_points = std::max(I.stats.work_frontier_peak_points, surv);
                }
            }
            I.stats.kernel_expand_td_s += ms_chain * 1e-3;
            I.stats.kernel_total_s += ms_chain * 1e-3;
            chained_done += done;
            const int b = done % 2;
            for (void *q : {s.pts, static_cast<void *>(s.off), static_cast<void *>(s.size), static_cast<void *>(s.arc_off),
                            static_cast<void *>(s.big_list), c.pts[b ^ 1], static_cast<void *>(c.off[b ^ 1]),
                            static_cast<void *>(c.size[b ^ 1]), static_cast<void *>(c.arc[b ^ 1]),
                            static_cast<void *>(c.big[b ^ 1])})
                arena_.release(q);
            s.pts = c.pts[b];
            s.off = c.off[b];
            s.size = c.size[b];
            s.sorted = c.sorted(b);
            s.layer = c.e->nl + c.dir * done;
            s.slot_points = std::max<int64_t>(C, 1);
            if (I.opts.method == 1 && s.layer == I.L - 1) {  // the terminal: its frontier is the result
                arena_.release(c.arc[b]);
                arena_.release(c.big[b]);
                s.arc_off = nullptr;
                s.big_list = nullptr;
                s.counted = false;
                const int32_t rn = *reinterpret_cast<const int32_t *>(hsum + s_chfin + sizeof(int32_t) * (g.first_slot + i));
                I.result_n = rn;
                I.result.resize(static_cast<size_t>(rn) * I.d * I.elem());
                fetch(I, s.pts);
                I.stats.work_frontier_survivors_total += rn;
                I.stats.work_frontier_peak_points = std::max<int64_t>(I.stats.work_frontier_peak_points, rn);
                I.phase = Instance::DONE;
            } else {
                s.arc_off = c.arc[b];
                s.big_list = c.big[b];
                s.res = R[static_cast<size_t>(done - 1) * n + i];
                s.counted = true;
                s.score = c.dir > 0 ? s.res.total : static_cast<int64_t>(1.5 * static_cast<double>(s.res.total));
            }
        }
    }
    chained_layers_total_ += chained_done;
    if (!fetches.empty()) {
        size_t total = 0;
        for (auto &f : fetches) total += align256(f.first->result.size());
        if (!h_results_.reserve(total)) {
            error_ = "cudaMallocHost failed";
            return -1;
        }
        size_t at = 0;
        for (auto &f : fetches) {
            cudaMemcpyAsync(static_cast<char *>(h_results_.p) + at, f.second, f.first->result.size(),
                            cudaMemcpyDeviceToHost, stream_);
            at += align256(f.first->result.size());
        }
        if (!cuda_ok(cudaStreamSynchronize(stream_), "D2H")) return -1;
        at = 0;
        for (auto &f : fetches) {
            std::memcpy(f.first->result.data(), static_cast<char *>(h_results_.p) + at, f.first->result.size());
            at += align256(f.first->result.size());
        }
    }
    if (trace_ && !chains.empty())
        std::fprintf(stderr, "[pmdd chain] requests=%zu layers=%d chained=%lld chain_ms=%.3f\n", chain_slots,
                     chain_layers_run, static_cast<long long>(chained_done), ms_chain);
    if (blocked && exps.empty() && ujobs.empty() && counts.empty()) {
        // nothing could move: the largest blocked request cannot fit next to the others
        fail(*blocked, PMDD_ERR_OOM, "device memory budget exhausted (layer does not fit)");
    }
    int done = 0;
    for (auto it = active_.begin(); it != active_.end();) {
        if ((*it)->phase == Instance::DONE) {
            Instance &I = **it;
            I.stats.gpu_mem_peak_used_bytes = static_cast<int64_t>(arena_.peak());
            I.stats.gpu_mem_peak_reserved_bytes = static_cast<int64_t>(arena_.reserved());
            release_instance(I);
            I.finish_s = now_s();
            record_finish(I);
            finished_.push_back(std::move(*it));
            it = active_.erase(it);
            ++done;
        } else {
            ++it;
        }
    }
    if (trace_) last_post_us_ = (now_s() - t_sync) * 1e6;
    return done;
}

}  // namespace pmdd
