// Test infrastructure (oracle): runs the reference's own CPU enumeration
// (topdown_cpu_enumerate / coupled_cpu_enumerate, src/pmdd/enum/cpu/enum.cpp, with its
// state-dominance passes, src/pmdd/enum/cpu/dominance.cpp) on a decision diagram given in
// the flat layout of include/pmdd.h, so that the reference sees the DD with exactly this
// project's node numbering.  The reference binary builds its own DDs, whose node order
// within a layer comes from hash-map iteration; the set-packing state-dominance pass picks
// partners in layer order, so its label counts are only comparable on one numbering.
//
// Self-written driver; it links the reference's CPU objects that oracle/Makefile compiles
// from the reference sources (everything but main.cpp) and is built into oracle/_ref/.
//
//   ref_harness_nobjs<N> <dd file> <problem type> <method 1|3> <state dominance>
//
// DD file (little-endian, written by oracle.write_flat_dd): int32 magic 0x46444450,
// nobjs, num_layers, num_nodes, num_arcs, num_weights, has_min_weight, state_words; then
// int32 layer_offsets[L+1], in_arc_offsets[N+1], arc_src[A], arc_weight[A],
// weights[K*nobjs], min_weight[N] (if present); uint64 node_state[N*state_words].
// Output: one JSON line of counters, then the frontier, one comma-separated point a line.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "bdd/bdd.hpp"
#include "enum/cpu/cpu_wrappers.hpp"
#include "enum/pareto_frontier.hpp"
#include "util/stats.hpp"

namespace {

template <class T>
bool read_vec(FILE *f, std::vector<T> &v, size_t n) {
    v.resize(n);
    return n == 0 || std::fread(v.data(), sizeof(T), n, f) == n;
}

int fail(const char *msg) {
    std::fprintf(stderr, "ref_harness: %s\n", msg);
    return 2;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 5) return fail("usage: ref_harness <dd file> <problem type> <method> <state dominance>");
    const int problem_type = std::atoi(argv[2]), method = std::atoi(argv[3]), sd = std::atoi(argv[4]);
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return fail("cannot open the DD file");
    int32_t hdr[8];
    if (std::fread(hdr, sizeof(int32_t), 8, f) != 8 || hdr[0] != 0x46444450) return fail("bad DD header");
    const int d = hdr[1], L = hdr[2], N = hdr[3], A = hdr[4], K = hdr[5], has_minw = hdr[6], W = hdr[7];
    if (d != NOBJS) return fail("objective count differs from this build's NOBJS");
    std::vector<int32_t> lo, io, src, aw, wts, minw;
    std::vector<uint64_t> st;
    bool ok = read_vec(f, lo, L + 1) && read_vec(f, io, static_cast<size_t>(N) + 1) && read_vec(f, src, A) &&
              read_vec(f, aw, A) && read_vec(f, wts, static_cast<size_t>(K) * d);
    if (ok && has_minw) ok = read_vec(f, minw, N);
    if (ok && W > 0) ok = read_vec(f, st, static_cast<size_t>(N) * W);
    std::fclose(f);
    if (!ok) return fail("truncated DD file");

    // the reference's BDD, nodes added layer by layer in this numbering
    BDD *bdd = new BDD(L);
    std::vector<Node *> node(N);
    for (int l = 0; l < L; ++l)
        for (int32_t v = lo[l]; v < lo[l + 1]; ++v) node[v] = bdd->add_node(l);
    std::vector<std::vector<ObjType>> rows(K, std::vector<ObjType>(d));
    for (int r = 0; r < K; ++r)
        for (int o = 0; o < d; ++o) rows[r][o] = wts[static_cast<size_t>(r) * d + o];
    for (int32_t v = 0; v < N; ++v)
        for (int32_t a = io[v]; a < io[v + 1]; ++a) {
            const int type = aw[a] != 0 ? 1 : 0;
            node[src[a]]->add_out_arc(node[v], type);
            node[src[a]]->set_arc_weights(type, rows[aw[a]].data());
        }
    const int nvars = L - 1;
    for (int32_t v = 0; v < N; ++v) {
        node[v]->min_weight = has_minw ? minw[v] : 0;
        if (W > 0) {
            node[v]->setpack_state.resize(nvars, false);
            for (int b = 0; b < nvars; ++b)
                if ((st[static_cast<size_t>(v) * W + b / 64] >> (b % 64)) & 1ULL) node[v]->setpack_state.set(b);
        }
    }

    EnumerationStats stats;
    ParetoFrontier *pf = method == 3 ? coupled_cpu_enumerate(bdd, true, problem_type, sd, &stats, 1)
                                     : topdown_cpu_enumerate(bdd, true, problem_type, sd, &stats, 1);
    if (!pf) return fail("enumeration returned no frontier");
    std::printf("{\"num_solutions\": %d, \"dominance_filtered_total\": %d, \"work_candidates_total\": %lld, "
                "\"work_frontier_survivors_total\": %lld, \"work_join_products_total\": %lld, "
                "\"layer_coupling\": %d}\n",
                pf->get_num_sols(), stats.dominance_filtered_total, stats.work_candidates_total,
                stats.work_frontier_survivors_total, stats.work_join_products_total, stats.layer_coupling);
    for (size_t i = 0; i + d <= pf->sols.size(); i += d) {
        for (int o = 0; o < d; ++o) std::printf(o ? ",%d" : "%d", pf->sols[i + o]);
        std::printf("\n");
    }
    return 0;
}
