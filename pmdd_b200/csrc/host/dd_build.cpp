// Host front end: instance parsers and exact decision-diagram constructors.
//
// Each constructor reproduces the reference's DD (same layers, same node and arc
// counts, same arc weights) but emits the flat, layer-major arrays of pmdd_dd
// directly.  Node numbering within a layer follows first creation, where the
// reference follows hash-map iteration order; nothing downstream depends on it.
#include "dd_build.hpp"

#include <algorithm>
#include <cctype>
#include <climits>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <map>
#include <memory>
#include <mutex>
#include <unordered_map>

namespace pmdd {

pmdd_dd FlatDD::view() const {
    pmdd_dd v;
    std::memset(&v, 0, sizeof(v));
    v.nobjs = nobjs;
    v.num_layers = num_layers();
    v.num_nodes = num_nodes();
    v.num_arcs = num_arcs();
    v.num_weights = nobjs > 0 ? static_cast<int32_t>(weights.size() / nobjs) : 0;
    v.layer_offsets = layer_offsets.data();
    v.in_arc_offsets = in_arc_offsets.data();
    v.arc_src = arc_src.data();
    v.arc_weight = arc_weight.data();
    v.weights = weights.data();
    v.min_weight = min_weight.empty() ? nullptr : min_weight.data();
    v.node_state = node_state.empty() ? nullptr : node_state.data();
    v.state_words = node_state.empty() ? 0 : state_words;
    return v;
}

// ----------------------------------------------------------------------------- text
bool IntReader::next(long long *v) {
    while (pos_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[pos_]))) ++pos_;
    if (pos_ >= s_.size()) return false;
    const char *begin = s_.c_str() + pos_;
    char *end = nullptr;
    long long x = std::strtoll(begin, &end, 10);
    if (end == begin) return false;
    pos_ += static_cast<size_t>(end - begin);
    *v = x;
    return true;
}

long long IntReader::need(const char *what) {
    long long v = 0;
    if (!next(&v)) throw std::runtime_error(std::string("instance text ended or is malformed while reading ") + what);
    return v;
}

// Knapsack format (src/pmdd/instances/knapsack_instance.cpp:17-47):
//   n_vars n_cons num_objs / num_objs rows of n_vars profits / per constraint: n_vars
//   coefficients then the right-hand side.
KnapsackData parse_knapsack(const std::string &text) {
    IntReader r(text);
    KnapsackData k;
    k.n_vars = static_cast<int>(r.need("n_vars"));
    k.n_cons = static_cast<int>(r.need("n_cons"));
    k.num_objs = static_cast<int>(r.need("num_objs"));
    if (k.n_vars <= 0 || k.n_cons < 0 || k.num_objs <= 0) throw std::runtime_error("knapsack header out of range");
    k.obj.assign(k.n_vars, std::vector<int>(k.num_objs, 0));
    k.coeffs.assign(k.n_cons, std::vector<int>(k.n_vars, 0));
    k.rhs.assign(k.n_cons, 0);
    for (int o = 0; o < k.num_objs; ++o)
        for (int i = 0; i < k.n_vars; ++i) k.obj[i][o] = static_cast<int>(r.need("objective coefficient"));
    for (int c = 0; c < k.n_cons; ++c) {
        for (int i = 0; i < k.n_vars; ++i) k.coeffs[c][i] = static_cast<int>(r.need("constraint coefficient"));
        k.rhs[c] = static_cast<int>(r.need("right-hand side"));
    }
    return k;
}

// Set packing format (src/pmdd/instances/setpacking_instance.hpp:49-80):
//   n_vars n_cons n_objs / n_objs rows of n_vars values / per constraint: k then k
//   one-based variable indices.
SetPackingData parse_setpacking(const std::string &text) {
    IntReader r(text);
    SetPackingData s;
    s.n_vars = static_cast<int>(r.need("n_vars"));
    s.n_cons = static_cast<int>(r.need("n_cons"));
    s.n_objs = static_cast<int>(r.need("n_objs"));
    if (s.n_vars <= 0 || s.n_cons < 0 || s.n_objs <= 0) throw std::runtime_error("set packing header out of range");
    s.objs.assign(s.n_objs, std::vector<int>(s.n_vars, 0));
    for (int o = 0; o < s.n_objs; ++o)
        for (int i = 0; i < s.n_vars; ++i) s.objs[o][i] = static_cast<int>(r.need("objective coefficient"));
    s.vars_cons.resize(s.n_cons);
    for (int c = 0; c < s.n_cons; ++c) {
        const int k = static_cast<int>(r.need("constraint size"));
        if (k < 0) throw std::runtime_error("negative constraint size");
        s.vars_cons[c].resize(k);
        for (int i = 0; i < k; ++i) {
            const int v = static_cast<int>(r.need("constraint variable")) - 1;
            if (v < 0 || v >= s.n_vars) throw std::runtime_error("constraint variable index out of range");
            s.vars_cons[c][i] = v;
        }
    }
    return s;
}

// TSP format (src/pmdd/instances/tsp_instance.cpp:11-32): n_objs n_cities then one
// n_cities x n_cities matrix per objective.
TSPData parse_tsp(const std::string &text) {
    IntReader r(text);
    TSPData t;
    t.n_objs = static_cast<int>(r.need("n_objs"));
    t.n_cities = static_cast<int>(r.need("n_cities"));
    if (t.n_objs <= 0 || t.n_cities < 2 || t.n_cities > 32) throw std::runtime_error("TSP header out of range (2..32 cities)");
    const size_t nn = static_cast<size_t>(t.n_cities) * t.n_cities;
    t.cost.assign(static_cast<size_t>(t.n_objs) * nn, 0);
    for (size_t i = 0; i < t.cost.size(); ++i) t.cost[i] = static_cast<int>(r.need("cost"));
    return t;
}

// ------------------------------------------------------------ binary DD scaffolding
namespace {

struct BNode {
    int32_t arc[2] = {-1, -1};  // targets (local index in the next layer) of the 0/1 arcs
};
typedef std::vector<std::vector<BNode>> BLayers;

struct VecHash {
    size_t operator()(const std::vector<int> &v) const {
        uint64_t h = 1469598103934665603ULL;
        for (int x : v) h = (h ^ static_cast<uint32_t>(x)) * 1099511628211ULL;
        return static_cast<size_t>(h ^ (h >> 29));
    }
};
struct WordsHash {
    size_t operator()(const std::vector<uint64_t> &v) const {
        uint64_t h = 0x9e3779b97f4a7c15ULL;
        for (uint64_t x : v) {
            h ^= x + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2);
            h *= 0xff51afd7ed558ccdULL;
        }
        return static_cast<size_t>(h ^ (h >> 32));
    }
};

void layer_shape(const BLayers &L, int64_t *width, int64_t *nodes) {
    int64_t w = 0, n = 0;
    for (const auto &layer : L) {
        w = std::max<int64_t>(w, static_cast<int64_t>(layer.size()));
        n += static_cast<int64_t>(layer.size());
    }
    *width = w;
    *nodes = n;
}

// Bottom-up reduction: merge nodes of a layer whose (0-target, 1-target) pairs agree and
// drop nodes left without outgoing arcs; the terminal layer is kept as is.  Same
// equivalence rule as BDDAlg::reduce (src/pmdd/bdd/bdd_alg.hpp:24-93).
void reduce_bdd(BLayers &L) {
    const int nl = static_cast<int>(L.size());
    std::vector<int32_t> remap_next;  // remap of layer l+1 old index -> new index (-1: removed)
    remap_next.resize(L[nl - 1].size());
    for (size_t i = 0; i < remap_next.size(); ++i) remap_next[i] = static_cast<int32_t>(i);
    for (int l = nl - 2; l >= 0; --l) {
        std::vector<BNode> &layer = L[l];
        std::unordered_map<uint64_t, int32_t> seen;
        seen.reserve(layer.size() * 2 + 1);
        std::vector<int32_t> remap(layer.size(), -1);
        std::vector<BNode> kept;
        kept.reserve(layer.size());
        for (size_t i = 0; i < layer.size(); ++i) {
            BNode nd = layer[i];
            for (int t = 0; t < 2; ++t) nd.arc[t] = nd.arc[t] >= 0 ? remap_next[nd.arc[t]] : -1;
            if (nd.arc[0] < 0 && nd.arc[1] < 0) continue;  // no way down: removed
            const uint64_t key = (static_cast<uint64_t>(static_cast<uint32_t>(nd.arc[0])) << 32) |
                                 static_cast<uint32_t>(nd.arc[1]);
            auto it = seen.find(key);
            if (it == seen.end()) {
                const int32_t id = static_cast<int32_t>(kept.size());
                seen.emplace(key, id);
                kept.push_back(nd);
                remap[i] = id;
            } else {
                remap[i] = it->second;
            }
        }
        layer.swap(kept);
        remap_next.swap(remap);
    }
}

// Flattens a binary DD.  Incoming arcs of each node are listed 1-arcs first, then
// 0-arcs, each group in parent order -- the maximisation arc order the reference packs
// for its GPU path (src/pmdd/enum/gpu/enum.cu:444-445, :482-494).  Weight row 0 is
// the zero vector; row 1+l is the 1-arc weight of layer l.
FlatDD flatten_bdd(const BLayers &L, const std::vector<std::vector<int>> &one_w, int nobjs) {
    FlatDD f;
    f.nobjs = nobjs;
    const int nl = static_cast<int>(L.size());
    f.layer_offsets.resize(nl + 1, 0);
    for (int l = 0; l < nl; ++l) f.layer_offsets[l + 1] = f.layer_offsets[l] + static_cast<int32_t>(L[l].size());
    const int32_t N = f.layer_offsets[nl];
    std::vector<int32_t> in_deg(N, 0);
    for (int l = 0; l + 1 < nl; ++l)
        for (const BNode &nd : L[l])
            for (int t = 0; t < 2; ++t)
                if (nd.arc[t] >= 0) in_deg[f.layer_offsets[l + 1] + nd.arc[t]]++;
    f.in_arc_offsets.resize(N + 1, 0);
    for (int32_t v = 0; v < N; ++v) f.in_arc_offsets[v + 1] = f.in_arc_offsets[v] + in_deg[v];
    const int32_t A = f.in_arc_offsets[N];
    f.arc_src.resize(A);
    f.arc_weight.resize(A);
    std::vector<int32_t> fill(f.in_arc_offsets.begin(), f.in_arc_offsets.end() - 1);
    for (int t : {1, 0}) {
        for (int l = 0; l + 1 < nl; ++l) {
            for (size_t i = 0; i < L[l].size(); ++i) {
                const int32_t tgt = L[l][i].arc[t];
                if (tgt < 0) continue;
                const int32_t v = f.layer_offsets[l + 1] + tgt;
                const int32_t a = fill[v]++;
                f.arc_src[a] = f.layer_offsets[l] + static_cast<int32_t>(i);
                f.arc_weight[a] = t == 1 ? 1 + l : 0;
            }
        }
    }
    f.weights.assign(static_cast<size_t>(nl) * nobjs, 0);  // row 0 zero + rows 1..nl-1
    for (int l = 0; l + 1 < nl; ++l)
        for (int o = 0; o < nobjs; ++o) f.weights[static_cast<size_t>(1 + l) * nobjs + o] = one_w[l][o];
    int64_t max_in = 0, total_in = 0;
    for (int l = 0; l < nl; ++l) {
        const int64_t layer_in = f.in_arc_offsets[f.layer_offsets[l + 1]] - f.in_arc_offsets[f.layer_offsets[l]];
        max_in = std::max(max_in, layer_in);
        total_in += layer_in;
    }
    f.info.max_num_in_arcs = max_in;
    f.info.total_num_in_arcs = total_in;
    f.info.num_layers = nl;
    return f;
}

void check_nobjs(int nobjs, int have) {
    if (nobjs < 1 || nobjs > 8) throw std::runtime_error("nobjs must be in 1..8");
    if (have < nobjs) throw std::runtime_error("instance has fewer objectives than the requested NOBJS");
}

}  // namespace

// -------------------------------------------------------------------- knapsack BDD
// Exact construction over used-capacity states, one layer per variable
// (src/pmdd/bdd/knapsack_bdd.cpp:10-118); then reduction and the min-weight pass
// (src/pmdd/bdd/knapsack_bdd.cpp:123-150).  The reference's second reduce + weight
// pass (src/pmdd/main.cpp:143-153) finds nothing left to merge after the first one.
// One constraint, non-negative weights: the reduced layers straight from dense arrays over
// the used capacity 0..cap (the construction kpbuild.cu runs on the device).  Top-down, a
// state's id is the rank of its first sighting (parents in id order, 0-arc before 1-arc),
// as the map-based loop below numbers them; bottom-up, the feasible completions shrink as
// the used capacity grows, so states whose (0-child, 1-child) classes agree are runs of
// consecutive reachable states, and a class takes the rank of its smallest old id, as
// reduce_bdd numbers them.  Returns false (nothing written) when the instance is not of
// that form or the dense arrays would exceed 2^26 entries.
static bool knapsack_dense_layers(const KnapsackData &k, BLayers *Lout, int64_t *ow, int64_t *on) {
    const int n = k.n_vars;
    if (n < 1 || k.n_cons != 1 || k.rhs[0] < 0) return false;
    for (int l = 0; l < n; ++l)
        if (k.coeffs[0][l] < 0) return false;
    const int64_t cap = k.rhs[0], S = cap + 1;
    if (static_cast<int64_t>(n) * S > (static_cast<int64_t>(1) << 26)) return false;
    std::vector<int32_t> idx(static_cast<size_t>(n * S), -1);  // layers 0..n-1
    std::vector<int32_t> width(n + 1, 0);
    idx[0] = 0;
    width[0] = 1;
    std::vector<int64_t> key(static_cast<size_t>(S));
    std::vector<int32_t> rank;
    const int64_t kNone = INT64_MAX;
    for (int l = 0; l + 1 < n; ++l) {
        const int32_t *cur = idx.data() + l * S;
        int32_t *nxt = idx.data() + (l + 1) * S;
        const int64_t w = k.coeffs[0][l];
        rank.assign(2 * static_cast<size_t>(width[l]), 0);
        for (int64_t st = 0; st < S; ++st) {
            int64_t kk = kNone;
            if (cur[st] >= 0) kk = 2 * static_cast<int64_t>(cur[st]);
            if (st >= w && cur[st - w] >= 0) kk = std::min(kk, 2 * static_cast<int64_t>(cur[st - w]) + 1);
            key[st] = kk;
            if (kk != kNone) rank[kk] = 1;
        }
        int32_t run = 0;
        for (int32_t &r : rank) {
            const int32_t x = r;
            r = run;
            run += x;
        }
        for (int64_t st = 0; st < S; ++st) nxt[st] = key[st] == kNone ? -1 : rank[key[st]];
        width[l + 1] = run;
    }
    width[n] = 1;
    BLayers &L = *Lout;
    L.assign(n + 1, std::vector<BNode>());
    L[n].resize(1);
    std::vector<int32_t> remap_next(1, 0), remap_cur, class_of, first_of;
    struct Cls {
        int32_t c0, c1, minold;
    };
    std::vector<Cls> cls;
    for (int l = n - 1; l >= 0; --l) {
        const int32_t *cur = idx.data() + l * S;
        const int32_t *nxt = l + 1 < n ? idx.data() + (l + 1) * S : nullptr;
        const int64_t w = k.coeffs[0][l];
        cls.clear();
        class_of.assign(width[l], -1);
        for (int64_t st = 0; st < S; ++st) {
            const int32_t old = cur[st];
            if (old < 0) continue;
            const int32_t c0 = remap_next[nxt ? nxt[st] : 0];
            const int32_t c1 = st + w <= cap ? remap_next[nxt ? nxt[st + w] : 0] : -1;
            if (cls.empty() || cls.back().c0 != c0 || cls.back().c1 != c1) cls.push_back({c0, c1, old});
            else cls.back().minold = std::min(cls.back().minold, old);
            class_of[old] = static_cast<int32_t>(cls.size()) - 1;
        }
        // number the classes by their smallest old id
        first_of.assign(width[l], -1);
        for (size_t c = 0; c < cls.size(); ++c) first_of[cls[c].minold] = static_cast<int32_t>(c);
        std::vector<int32_t> newid(cls.size(), -1);
        int32_t next_id = 0;
        for (int32_t x = 0; x < width[l]; ++x)
            if (first_of[x] >= 0) newid[first_of[x]] = next_id++;
        L[l].resize(cls.size());
        for (size_t c = 0; c < cls.size(); ++c) {
            L[l][newid[c]].arc[0] = cls[c].c0;
            L[l][newid[c]].arc[1] = cls[c].c1;
        }
        remap_cur.assign(width[l], -1);
        for (int32_t x = 0; x < width[l]; ++x)
            if (class_of[x] >= 0) remap_cur[x] = newid[class_of[x]];
        remap_next.swap(remap_cur);
    }
    *ow = 0;
    *on = 0;
    for (int l = 0; l <= n; ++l) {
        *ow = std::max<int64_t>(*ow, width[l]);
        *on += width[l];
    }
    return true;
}

FlatDD build_knapsack_bdd(const KnapsackData &k, int nobjs) {
    check_nobjs(nobjs, k.num_objs);
    const int n = k.n_vars, m = k.n_cons;
    BLayers L;
    int64_t ow = 0, on = 0;
    const bool dense = knapsack_dense_layers(k, &L, &ow, &on);
    if (!dense) {
        L.assign(n + 1, std::vector<BNode>());
        L[0].resize(1);
        L[n].resize(1);  // terminal
        std::vector<std::vector<int>> states(1, std::vector<int>(m, 0));
        const bool single = (m == 1) && k.rhs[0] >= 0 && k.rhs[0] <= (1 << 26);
        for (int l = 0; l < n; ++l) {
            std::vector<std::vector<int>> next_states;
            auto feasible_add = [&](const std::vector<int> &s, std::vector<int> *out) {
                out->resize(m);
                for (int c = 0; c < m; ++c) {
                    (*out)[c] = s[c] + k.coeffs[c][l];
                    if ((*out)[c] > k.rhs[c]) return false;
                }
                return true;
            };
            if (l < n - 1) {
                std::unordered_map<std::vector<int>, int32_t, VecHash> map;
                std::vector<int32_t> dense;
                if (single) dense.assign(static_cast<size_t>(k.rhs[0]) + 1, -1);
                auto lookup = [&](const std::vector<int> &s) -> int32_t {
                    if (single && s[0] >= 0) {
                        int32_t &slot = dense[s[0]];
                        if (slot < 0) {
                            slot = static_cast<int32_t>(next_states.size());
                            next_states.push_back(s);
                        }
                        return slot;
                    }
                    auto it = map.find(s);
                    if (it != map.end()) return it->second;
                    const int32_t id = static_cast<int32_t>(next_states.size());
                    map.emplace(s, id);
                    next_states.push_back(s);
                    return id;
                };
                std::vector<int> s1;
                for (size_t i = 0; i < states.size(); ++i) {
                    L[l][i].arc[0] = lookup(states[i]);
                    if (feasible_add(states[i], &s1)) L[l][i].arc[1] = lookup(s1);
                }
                L[l + 1].resize(next_states.size());
                states.swap(next_states);
            } else {
                std::vector<int> s1;
                for (size_t i = 0; i < states.size(); ++i) {
                    L[l][i].arc[0] = 0;
                    if (feasible_add(states[i], &s1)) L[l][i].arc[1] = 0;
                }
            }
        }
        layer_shape(L, &ow, &on);
        reduce_bdd(L);
    }
    int64_t rw, rn;
    layer_shape(L, &rw, &rn);

    std::vector<std::vector<int>> one_w(n, std::vector<int>(nobjs, 0));
    for (int l = 0; l < n; ++l)
        for (int o = 0; o < nobjs; ++o) one_w[l][o] = k.obj[l][o];
    FlatDD f = flatten_bdd(L, one_w, nobjs);
    f.problem_type = 1;
    f.info.problem_type = 1;
    f.info.original_width = ow;
    f.info.original_num_nodes = on;
    f.info.reduced_width = rw;
    f.info.reduced_num_nodes = rn;

    // Minimum used capacity over root paths, first constraint only (the reference's
    // update_node_weights reads coeffs[0]).
    if (m >= 1) {
        const int32_t N = f.num_nodes();
        f.min_weight.assign(N, 0);
        for (int l = 1; l <= n; ++l) {
            for (int32_t v = f.layer_offsets[l]; v < f.layer_offsets[l + 1]; ++v) {
                long long best = 2147483647LL;
                for (int32_t a = f.in_arc_offsets[v]; a < f.in_arc_offsets[v + 1]; ++a) {
                    long long w = f.min_weight[f.arc_src[a]];
                    if (f.arc_weight[a] != 0) w += k.coeffs[0][l - 1];
                    best = std::min(best, w);
                }
                f.min_weight[v] = static_cast<int32_t>(best);
            }
        }
    }
    return f;
}

// ------------------------------------------------------- independent-set BDD (SP)
// Set packing -> conflict graph -> independent-set BDD with the min-in-state vertex
// ordering (src/pmdd/instances/setpacking_instance.hpp:92-126,
// src/pmdd/bdd/indepset_bdd.cpp:50-165, src/pmdd/bdd/indepset_bdd.hpp:89-114).
FlatDD build_indepset_bdd(const SetPackingData &sp, int nobjs) {
    check_nobjs(nobjs, sp.n_objs);
    const int n = sp.n_vars;
    const int W = (n + 63) / 64;
    // complement of the closed neighbourhood of each vertex, W words each
    std::vector<uint64_t> keep(static_cast<size_t>(n) * W, 0);
    {
        std::vector<char> adj(static_cast<size_t>(n) * n, 0);
        for (const auto &cons : sp.vars_cons)
            for (size_t i = 0; i < cons.size(); ++i)
                for (size_t j = i + 1; j < cons.size(); ++j) {
                    adj[static_cast<size_t>(cons[i]) * n + cons[j]] = 1;
                    adj[static_cast<size_t>(cons[j]) * n + cons[i]] = 1;
                }
        for (int v = 0; v < n; ++v)
            for (int w = 0; w < n; ++w)
                if (w != v && !adj[static_cast<size_t>(v) * n + w])
                    keep[static_cast<size_t>(v) * W + w / 64] |= (1ULL << (w % 64));
    }
    BLayers L(n + 1);
    L[0].resize(1);
    // the states of a layer, flat (W words each), in node order
    std::vector<uint64_t> states(W, 0), next;
    for (int v = 0; v < n; ++v) states[v / 64] |= (1ULL << (v % 64));
    size_t count = 1;
    std::vector<int> active(n);
    for (int v = 0; v < n; ++v) active[v] = v;
    std::vector<int> counter(n, 0);
    std::vector<int> var_layer(n, -1);
    std::vector<uint64_t> node_state;  // the states of every layer, in node order
    std::vector<int32_t> table;        // open addressing: index of a next-layer state, -1 empty
    std::vector<uint64_t> s0(W), s1(W);
    auto hash_words = [W](const uint64_t *k) {
        uint64_t h = 0x9e3779b97f4a7c15ULL;
        for (int w = 0; w < W; ++w) {
            h ^= k[w] + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2);
            h *= 0xff51afd7ed558ccdULL;
        }
        return h ^ (h >> 32);
    };
    for (int l = 1; l <= n; ++l) {
        node_state.insert(node_state.end(), states.begin(), states.end());
        // min-in-state: vertex appearing in the fewest current states; ties go to the
        // first such entry of the active list, which shrinks by swap-with-last.
        for (int v : active) counter[v] = 0;
        for (size_t i = 0; i < count; ++i)
            for (int w = 0; w < W; ++w) {
                uint64_t x = states[i * W + w];
                while (x) {
                    counter[w * 64 + __builtin_ctzll(x)]++;
                    x &= x - 1;
                }
            }
        size_t sel = 0;
        for (size_t i = 1; i < active.size(); ++i)
            if (counter[active[i]] < counter[active[sel]]) sel = i;
        const int vertex = active[sel];
        active[sel] = active.back();
        active.pop_back();
        var_layer[l - 1] = vertex;

        size_t cap = 16;
        while (cap < 4 * count + 4) cap <<= 1;
        table.assign(cap, -1);
        next.clear();
        int32_t next_count = 0;
        // first sighting numbering: state i's 0-child, then its 1-child
        auto lookup = [&](const uint64_t *k) -> int32_t {
            size_t h = static_cast<size_t>(hash_words(k)) & (cap - 1);
            for (;;) {
                const int32_t id = table[h];
                if (id < 0) {
                    table[h] = next_count;
                    next.insert(next.end(), k, k + W);
                    return next_count++;
                }
                if (std::memcmp(next.data() + static_cast<size_t>(id) * W, k, sizeof(uint64_t) * W) == 0) return id;
                h = (h + 1) & (cap - 1);
            }
        };
        const uint64_t vbit = 1ULL << (vertex % 64);
        const int vw = vertex / 64;
        const uint64_t *kv = keep.data() + static_cast<size_t>(vertex) * W;
        for (size_t i = 0; i < count; ++i) {
            const uint64_t *s = states.data() + i * W;
            const bool was_set = (s[vw] & vbit) != 0;
            std::memcpy(s0.data(), s, sizeof(uint64_t) * W);
            s0[vw] &= ~vbit;
            L[l - 1][i].arc[0] = lookup(s0.data());
            if (was_set) {
                for (int w = 0; w < W; ++w) s1[w] = s0[w] & kv[w];
                L[l - 1][i].arc[1] = lookup(s1.data());
            }
        }
        L[l].resize(next_count);
        states.swap(next);
        count = static_cast<size_t>(next_count);
    }
    if (L[n].size() != 1) throw std::runtime_error("independent-set BDD did not close to a single terminal");
    node_state.insert(node_state.end(), states.begin(), states.begin() + W);
    std::vector<std::vector<int>> one_w(n, std::vector<int>(nobjs, 0));
    for (int l = 0; l < n; ++l)
        for (int o = 0; o < nobjs; ++o) one_w[l][o] = sp.objs[o][var_layer[l]];
    FlatDD f = flatten_bdd(L, one_w, nobjs);
    f.problem_type = 2;
    f.info.problem_type = 2;
    f.node_state.swap(node_state);
    f.state_words = W;
    int64_t w, nn;
    layer_shape(L, &w, &nn);
    f.info.original_width = f.info.reduced_width = w;
    f.info.original_num_nodes = f.info.reduced_num_nodes = nn;
    return f;
}

// ---------------------------------------------------------------------- TSP MDD
// Layers 0..n+1: root, the fixed first city 0 (zero-weight arc), one layer per further
// city over states (visited set, last city), then the terminal reached by returning to
// city 0.  Arc weights are negated costs (src/pmdd/mdd/tsp_mdd.cpp:21-196).
// Weight row 0 is zero; row 1 + i*n + j holds -cost[.][i][j].
// The layers, nodes and arcs (with their weight-row indices) of the n-city MDD: they
// depend on n alone, never on the costs.
static FlatDD tsp_structure(int n, int nobjs) {
    const int nl = n + 2;
    struct St {
        uint64_t S;
        int last;
    };
    std::vector<std::vector<St>> layers(nl);
    // incoming arcs per layer node, built while expanding: (src local, weight row)
    std::vector<std::vector<std::vector<std::pair<int32_t, int32_t>>>> in(nl);
    layers[0].push_back({0ULL, -1});
    layers[1].push_back({1ULL, 0});
    in[1].resize(1);
    in[1][0].push_back({0, 0});
    for (int l = 1; l < n; ++l) {
        std::unordered_map<uint64_t, int32_t> map;
        for (size_t i = 0; i < layers[l].size(); ++i) {
            const St s = layers[l][i];
            for (int v = 0; v < n; ++v) {
                if (s.S & (1ULL << v)) continue;
                const uint64_t key = ((s.S | (1ULL << v)) << 6) | static_cast<uint64_t>(v);
                int32_t id;
                auto it = map.find(key);
                if (it == map.end()) {
                    id = static_cast<int32_t>(layers[l + 1].size());
                    map.emplace(key, id);
                    layers[l + 1].push_back({s.S | (1ULL << v), v});
                    in[l + 1].emplace_back();
                } else {
                    id = it->second;
                }
                in[l + 1][id].push_back({static_cast<int32_t>(i), 1 + s.last * n + v});
            }
        }
    }
    layers[n + 1].push_back({0ULL, -1});
    in[n + 1].resize(1);
    for (size_t i = 0; i < layers[n].size(); ++i)
        in[n + 1][0].push_back({static_cast<int32_t>(i), 1 + layers[n][i].last * n + 0});

    FlatDD f;
    f.nobjs = nobjs;
    f.problem_type = 3;
    f.layer_offsets.resize(nl + 1, 0);
    for (int l = 0; l < nl; ++l) f.layer_offsets[l + 1] = f.layer_offsets[l] + static_cast<int32_t>(layers[l].size());
    const int32_t N = f.layer_offsets[nl];
    f.in_arc_offsets.assign(N + 1, 0);
    int64_t max_in = 0, total_in = 0;
    for (int l = 0; l < nl; ++l) {
        int64_t layer_in = 0;
        for (size_t i = 0; i < layers[l].size(); ++i) {
            const int32_t v = f.layer_offsets[l] + static_cast<int32_t>(i);
            const int32_t d = l == 0 ? 0 : static_cast<int32_t>(in[l][i].size());
            f.in_arc_offsets[v + 1] = f.in_arc_offsets[v] + d;
            layer_in += d;
        }
        max_in = std::max(max_in, layer_in);
        total_in += layer_in;
    }
    f.arc_src.resize(f.in_arc_offsets[N]);
    f.arc_weight.resize(f.in_arc_offsets[N]);
    for (int l = 1; l < nl; ++l)
        for (size_t i = 0; i < layers[l].size(); ++i) {
            const int32_t v = f.layer_offsets[l] + static_cast<int32_t>(i);
            int32_t a = f.in_arc_offsets[v];
            for (const auto &p : in[l][i]) {
                f.arc_src[a] = f.layer_offsets[l - 1] + p.first;
                f.arc_weight[a] = p.second;
                ++a;
            }
        }
    f.info.original_width = f.info.reduced_width = -1;
    f.info.original_num_nodes = f.info.reduced_num_nodes = -1;
    f.info.max_num_in_arcs = max_in;
    f.info.total_num_in_arcs = total_in;
    f.info.num_layers = nl;
    f.info.problem_type = 3;
    return f;
}

// Structures of up to 16 cities are kept for the life of the process (all threads share
// them); larger ones are built per call.
FlatDD build_tsp_mdd(const TSPData &t, int nobjs) {
    check_nobjs(nobjs, t.n_objs);
    const int n = t.n_cities;
    FlatDD f;
    if (n >= 1 && n <= 16) {
        static std::mutex mu;
        static std::map<int, std::unique_ptr<FlatDD>> cache;
        std::lock_guard<std::mutex> lk(mu);
        std::unique_ptr<FlatDD> &c = cache[n];
        if (!c) c.reset(new FlatDD(tsp_structure(n, 1)));
        f = *c;
    } else {
        f = tsp_structure(n, nobjs);
    }
    f.nobjs = nobjs;
    const size_t nn = static_cast<size_t>(n) * n;
    f.weights.assign((1 + nn) * nobjs, 0);
    for (size_t ij = 0; ij < nn; ++ij)
        for (int o = 0; o < nobjs; ++o) f.weights[(1 + ij) * nobjs + o] = -t.cost[o * nn + ij];
    return f;
}

FlatDD build_from_text(const std::string &text, int problem_type, int nobjs) {
    switch (problem_type) {
    case 1: return build_knapsack_bdd(parse_knapsack(text), nobjs);
    case 2: return build_indepset_bdd(parse_setpacking(text), nobjs);
    case 3: return build_tsp_mdd(parse_tsp(text), nobjs);
    default: throw std::runtime_error("problem type must be 1 (knapsack), 2 (set packing) or 3 (TSP)");
    }
}

}  // namespace pmdd

// ========================================================================= C ABI
struct pmdd_host_dd {
    pmdd::FlatDD dd;
};

namespace {
void write_err(char *err, size_t errlen, const std::string &msg) {
    if (err == nullptr || errlen == 0) return;
    const size_t n = std::min(errlen - 1, msg.size());
    std::memcpy(err, msg.data(), n);
    err[n] = '\0';
}
}  // namespace

extern "C" {

pmdd_host_dd *pmdd_build_from_text(const char *text, int32_t problem_type, int32_t nobjs, char *err,
                                   size_t errlen) {
    if (text == nullptr) {
        write_err(err, errlen, "instance text is NULL");
        return nullptr;
    }
    try {
        pmdd_host_dd *h = new pmdd_host_dd;
        h->dd = pmdd::build_from_text(std::string(text), problem_type, nobjs);
        return h;
    } catch (const std::exception &e) {
        write_err(err, errlen, e.what());
        return nullptr;
    }
}

pmdd_host_dd *pmdd_build_from_file(const char *path, int32_t problem_type, int32_t nobjs, char *err,
                                   size_t errlen) {
    std::ifstream in(path ? path : "");
    if (!in.is_open()) {
        write_err(err, errlen, std::string("Error - file ") + (path ? path : "(null)") + " could not be found");
        return nullptr;
    }
    std::stringstream ss;
    ss << in.rdbuf();
    const std::string text = ss.str();
    return pmdd_build_from_text(text.c_str(), problem_type, nobjs, err, errlen);
}

int pmdd_host_dd_view(const pmdd_host_dd *h, pmdd_dd *view) {
    if (h == nullptr || view == nullptr) return PMDD_ERR_INVALID;
    *view = h->dd.view();
    return PMDD_OK;
}

int pmdd_host_dd_info(const pmdd_host_dd *h, pmdd_dd_info *info) {
    if (h == nullptr || info == nullptr) return PMDD_ERR_INVALID;
    *info = h->dd.info;
    return PMDD_OK;
}

int pmdd_host_dd_layer_sizes(const pmdd_host_dd *h, int64_t *out, int32_t cap) {
    if (h == nullptr || out == nullptr) return PMDD_ERR_INVALID;
    const int32_t nl = h->dd.num_layers();
    if (cap < nl) return PMDD_ERR_INVALID;
    for (int32_t l = 0; l < nl; ++l) out[l] = h->dd.layer_offsets[l + 1] - h->dd.layer_offsets[l];
    return PMDD_OK;
}

void pmdd_host_dd_free(pmdd_host_dd *h) { delete h; }

void pmdd_sort_points_lex_ascending(int32_t *points, int64_t num_points, int32_t nobjs) {
    if (points == nullptr || num_points <= 1 || nobjs <= 0) return;
    std::vector<int64_t> idx(num_points);
    for (int64_t i = 0; i < num_points; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) {
        const int32_t *pa = points + a * nobjs, *pb = points + b * nobjs;
        for (int o = 0; o < nobjs; ++o)
            if (pa[o] != pb[o]) return pa[o] < pb[o];
        return false;
    });
    std::vector<int32_t> tmp(static_cast<size_t>(num_points) * nobjs);
    for (int64_t i = 0; i < num_points; ++i)
        std::memcpy(&tmp[static_cast<size_t>(i) * nobjs], points + idx[i] * nobjs, sizeof(int32_t) * nobjs);
    std::memcpy(points, tmp.data(), tmp.size() * sizeof(int32_t));
}

}  // extern "C"
