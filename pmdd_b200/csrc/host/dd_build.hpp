// Host front end: instance parsing and exact DD compilation into the flat layout of
// pmdd_dd (include/pmdd.h).  Reference counterparts are listed in include/pmdd_host.h.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "pmdd.h"
#include "pmdd_host.h"

namespace pmdd {

// Owner of a compiled flat DD.  Node ids are global and layer-major.
struct FlatDD {
    int32_t nobjs = 0;
    int32_t problem_type = 0;
    std::vector<int32_t> layer_offsets;   // L+1
    std::vector<int32_t> in_arc_offsets;  // N+1
    std::vector<int32_t> arc_src;         // A
    std::vector<int32_t> arc_weight;      // A
    std::vector<int32_t> weights;         // K*d
    std::vector<int32_t> min_weight;      // N (knapsack only)
    std::vector<uint64_t> node_state;     // N*state_words (set packing only)
    int32_t state_words = 0;
    pmdd_dd_info info{};

    int32_t num_layers() const { return static_cast<int32_t>(layer_offsets.size()) - 1; }
    int32_t num_nodes() const { return layer_offsets.empty() ? 0 : layer_offsets.back(); }
    int32_t num_arcs() const { return static_cast<int32_t>(arc_src.size()); }
    pmdd_dd view() const;
};

// Whitespace-separated integer reader over an in-memory instance text.
class IntReader {
  public:
    explicit IntReader(const std::string &text) : s_(text), pos_(0) {}
    bool next(long long *v);
    long long need(const char *what);  // throws std::runtime_error on EOF / garbage

  private:
    const std::string &s_;
    size_t pos_;
};

// Instance data, as read by the reference's parsers.
struct KnapsackData {
    int n_vars = 0, n_cons = 0, num_objs = 0;
    std::vector<std::vector<int>> obj;     // [n_vars][num_objs]
    std::vector<std::vector<int>> coeffs;  // [n_cons][n_vars]
    std::vector<int> rhs;                  // [n_cons]
};
struct SetPackingData {
    int n_vars = 0, n_cons = 0, n_objs = 0;
    std::vector<std::vector<int>> objs;       // [n_objs][n_vars]
    std::vector<std::vector<int>> vars_cons;  // 0-based variable lists
};
struct TSPData {
    int n_cities = 0, n_objs = 0;
    std::vector<int> cost;  // [n_objs][n][n] row-major
};

KnapsackData parse_knapsack(const std::string &text);
SetPackingData parse_setpacking(const std::string &text);
TSPData parse_tsp(const std::string &text);

FlatDD build_knapsack_bdd(const KnapsackData &inst, int nobjs);
FlatDD build_indepset_bdd(const SetPackingData &inst, int nobjs);
FlatDD build_tsp_mdd(const TSPData &inst, int nobjs);

FlatDD build_from_text(const std::string &text, int problem_type, int nobjs);

}  // namespace pmdd
