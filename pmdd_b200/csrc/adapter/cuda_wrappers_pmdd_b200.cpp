// The reference's GPU seam on top of libpmdd_gpu.so.
//
// rahulptel/PMDD calls its GPU backend through four C++ functions declared in
// src/pmdd/enum/gpu/cuda_wrappers.hpp:11-21 and implemented by its enum/gpu/*.cu files
// (or by enum/gpu/cuda_stubs.cpp when CUDA is off; the choice is made at link time,
// src/pmdd/makefile:93-104).  This file implements the same four functions: it
// flattens the reference's pointer-graph BDD / MDD into a pmdd_dd (include/pmdd.h) and
// calls pmdd_enumerate.  Linked in place of those objects, the reference's own main.cpp
// and DD constructors run unchanged on this engine.
//
// It compiles only against a reference checkout (its headers and -DNOBJS=N):
//   make -C oracle adapter REF=<reference checkout>
// which builds oracle/_ref/multiobj_nobjs<N>_pmdd from the reference's sources with
// this file linked instead of cuda_stubs.cpp.
//
// Flattening: nodes are numbered layer by layer in the order of the reference's layer
// vectors; a BDD node's incoming arcs are listed 1-arcs first, then 0-arcs (the order of
// the reference's GPU packing, src/pmdd/enum/gpu/enum.cu:444-445,482-494), each with the
// weights of its tail (Node::weights[type], a missing vector read as zeros); an MDD
// node's incoming arcs in in_arcs_list order with the arc's own weights.  Every arc gets
// its own weight row (row 0 is the zero vector).  Knapsack BDDs also carry min_weight and
// set-packing BDDs their setpack_state bitsets, for state dominance.
#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

#include "enum/gpu/cuda_wrappers.hpp"
#include "pmdd.h"

namespace {

struct Flat {
    std::vector<int32_t> layer_off, in_off, src, wrow, weights, min_weight;
    std::vector<uint64_t> state;
    int32_t state_words = 0;
};

int32_t add_row(Flat &f, const ObjType *w) {
    const int32_t row = static_cast<int32_t>(f.weights.size() / NOBJS);
    for (int o = 0; o < NOBJS; ++o) f.weights.push_back(w != nullptr ? static_cast<int32_t>(w[o]) : 0);
    return row;
}

Flat flatten(BDD *bdd, bool maximization) {
    Flat f;
    const int L = bdd->num_layers;
    std::unordered_map<const Node *, int32_t> id;
    f.layer_off.push_back(0);
    for (int l = 0; l < L; ++l) {
        for (Node *v : bdd->layers[l]) id.emplace(v, static_cast<int32_t>(id.size()));
        f.layer_off.push_back(static_cast<int32_t>(id.size()));
    }
    f.weights.assign(NOBJS, 0);
    f.in_off.push_back(0);
    const int first = maximization ? 1 : 0;
    for (int l = 0; l < L; ++l)
        for (Node *v : bdd->layers[l]) {
            for (int t : {first, 1 - first})
                for (Node *u : v->prev[t]) {
                    f.src.push_back(id.at(u));
                    f.wrow.push_back(add_row(f, u->weights[t]));
                }
            f.in_off.push_back(static_cast<int32_t>(f.src.size()));
            f.min_weight.push_back(v->min_weight);
        }
    const size_t nbits = bdd->get_root()->setpack_state.size();
    f.state_words = static_cast<int32_t>((nbits + 63) / 64);
    for (int l = 0; l < L && nbits > 0; ++l)
        for (Node *v : bdd->layers[l]) {
            const size_t at = f.state.size();
            f.state.resize(at + f.state_words, 0);
            for (size_t b = v->setpack_state.find_first(); b != boost::dynamic_bitset<>::npos;
                 b = v->setpack_state.find_next(b))
                f.state[at + b / 64] |= 1ULL << (b % 64);
        }
    return f;
}

Flat flatten(MDD *mdd) {
    Flat f;
    const int L = mdd->num_layers;
    std::unordered_map<const MDDNode *, int32_t> id;
    f.layer_off.push_back(0);
    for (int l = 0; l < L; ++l) {
        for (MDDNode *v : mdd->layers[l]) id.emplace(v, static_cast<int32_t>(id.size()));
        f.layer_off.push_back(static_cast<int32_t>(id.size()));
    }
    f.weights.assign(NOBJS, 0);
    f.in_off.push_back(0);
    for (int l = 0; l < L; ++l)
        for (MDDNode *v : mdd->layers[l]) {
            for (MDDArc *a : v->in_arcs_list) {
                f.src.push_back(id.at(a->tail));
                f.wrow.push_back(add_row(f, a->weights));
            }
            f.in_off.push_back(static_cast<int32_t>(f.src.size()));
        }
    return f;
}

pmdd_dd view(const Flat &f, int problem_type) {
    pmdd_dd d{};
    d.nobjs = NOBJS;
    d.num_layers = static_cast<int32_t>(f.layer_off.size()) - 1;
    d.num_nodes = f.layer_off.back();
    d.num_arcs = static_cast<int32_t>(f.src.size());
    d.num_weights = static_cast<int32_t>(f.weights.size() / NOBJS);
    d.layer_offsets = f.layer_off.data();
    d.in_arc_offsets = f.in_off.data();
    d.arc_src = f.src.data();
    d.arc_weight = f.wrow.data();
    d.weights = f.weights.data();
    d.min_weight = problem_type == 1 && !f.min_weight.empty() ? f.min_weight.data() : nullptr;
    if (problem_type == 2 && !f.state.empty()) {
        d.node_state = f.state.data();
        d.state_words = f.state_words;
    }
    return d;
}

ParetoFrontier *run(const pmdd_dd &dd, int method, int problem_type, int state_dominance, EnumerationStats *stats,
                    std::string *reason, long long max_cand, long long max_prod) {
    pmdd_options o;
    pmdd_options_default(&o);
    o.method = method;
    o.problem_type = problem_type;
    o.state_dominance = state_dominance;
    if (max_cand > 0) o.max_cand = max_cand;
    if (max_prod > 0) o.max_prod = max_prod;
    pmdd_frontier fr{};
    pmdd_stats st{};
    char err[512] = {0};
    if (pmdd_enumerate(&dd, &o, &fr, &st, err, sizeof(err)) != PMDD_OK) {
        if (reason) *reason = err;
        return nullptr;
    }
    if (fr.elem_bytes != static_cast<int32_t>(sizeof(ObjType))) {
        pmdd_frontier_free(&fr);
        if (reason) *reason = "objective sums exceed the range of the reference's ObjType";
        return nullptr;
    }
    ParetoFrontier *pf = new ParetoFrontier;
    const ObjType *p = static_cast<const ObjType *>(fr.points);
    pf->sols.assign(p, p + fr.num_points * NOBJS);
    pmdd_frontier_free(&fr);
    if (stats) {
        stats->wall_pack_transfer_s = st.wall_pack_transfer_s;
        stats->wall_join_s = st.wall_join_s;
        stats->kernel_expand_td_s = st.kernel_expand_td_s;
        stats->kernel_dominance_s = st.kernel_dominance_s;
        stats->kernel_total_s = st.kernel_total_s;
        stats->gpu_mem_peak_used_bytes = st.gpu_mem_peak_used_bytes;
        stats->gpu_mem_peak_reserved_bytes = st.gpu_mem_peak_reserved_bytes;
        stats->work_candidates_total = st.work_candidates_total;
        stats->work_candidates_peak = st.work_candidates_peak;
        stats->work_frontier_survivors_total = st.work_frontier_survivors_total;
        stats->work_frontier_peak_points = st.work_frontier_peak_points;
        stats->work_join_products_total = st.work_join_products_total;
        stats->dominance_filtered_total = static_cast<int>(st.dominance_filtered_total);
        stats->layer_coupling = st.layer_coupling;
    }
    return pf;
}

}  // namespace

ParetoFrontier *topdown_cuda_enumerate(BDD *bdd, bool maximization, const int problem_type,
                                       const int state_dominance, EnumerationStats *stats, std::string *reason,
                                       long long gpu_batch_size) {
    const Flat f = flatten(bdd, maximization);
    return run(view(f, problem_type), 1, problem_type, state_dominance, stats, reason, gpu_batch_size, 0);
}

ParetoFrontier *topdown_mdd_cuda_enumerate(MDD *mdd, EnumerationStats *stats, std::string *reason,
                                           long long gpu_batch_size) {
    const Flat f = flatten(mdd);
    return run(view(f, 3), 1, 3, 0, stats, reason, gpu_batch_size, 0);
}

ParetoFrontier *coupled_cuda_enumerate(MDD *mdd, EnumerationStats *stats, std::string *reason,
                                       long long gpu_batch_size, long long gpu_max_prod) {
    const Flat f = flatten(mdd);
    return run(view(f, 3), 3, 3, 0, stats, reason, gpu_batch_size, gpu_max_prod);
}

// The reference's GPU coupled driver ignores state_dominance (enum.cu:595-756); this
// engine applies it to the top-down layers as the reference's CPU coupled method does
// (enum/cpu/enum.cpp:275-285).  The frontier is the same either way.
ParetoFrontier *coupled_bdd_cuda_enumerate(BDD *bdd, bool maximization, const int problem_type,
                                           const int state_dominance, EnumerationStats *stats, std::string *reason,
                                           long long gpu_batch_size, long long gpu_max_prod) {
    const Flat f = flatten(bdd, maximization);
    return run(view(f, problem_type), 3, problem_type, state_dominance, stats, reason, gpu_batch_size, gpu_max_prod);
}
