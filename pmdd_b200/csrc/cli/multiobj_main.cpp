// multiobj_nobjs<N> -- drop-in command line for the GPU backend of rahulptel/PMDD.
//
// Same positional arguments, options, defaults and messages as the reference CLI
// (src/pmdd/util/cli_parser.cpp:181-488), the same three stdout lines
// (src/pmdd/util/output_utils.cpp:302-374), the same gzip'd frontier CSV
// (output_utils.cpp:87-152; ascending lexicographic order, "%d" values joined by ',',
// written by pmdd_write_frontier_csv_gz of the host library)
// and the same stats JSONL record (output_utils.cpp:154-300, schema_version 1).
// The number of objectives comes from the program name (multiobj_nobjs3 -> 3), as the
// reference's compile-time NOBJS does; PMDD_NOBJS overrides it.
//
// This binary drives the B200 engine; it has no CPU enumeration.  `--backend cpu`
// (the reference's default) is rejected with a message naming --backend gpu.
#include <cctype>
#include <cerrno>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <sys/resource.h>
#include <vector>

#include "host/dd_build.hpp"
#include "pmdd.h"
#include "pmdd_host.h"

namespace {

const long long kDefaultMaxCand = 20000000LL;
const long long kDefaultMaxProd = 625000LL;

struct Options {
    std::string input_path;
    int problem_type = 0, method = 0, state_dominance = 0;
    bool gpu = false;
    int cpu_threads = 1;
    long long max_cand = kDefaultMaxCand, max_prod = kDefaultMaxProd;
    bool save_frontier = false, save_stats = false;
    std::string frontier_out_path, stats_out_path;
};

std::string stem_of(const std::string &path, const char *fallback) {
    std::string base = path;
    const size_t slash = base.find_last_of("/\\");
    if (slash != std::string::npos) base = base.substr(slash + 1);
    const size_t dot = base.find_last_of('.');
    if (dot != std::string::npos) base = base.substr(0, dot);
    return base.empty() ? std::string(fallback) : base;
}

bool parse_positive_int(const std::string &v, int *out) {
    if (v.empty()) return false;
    errno = 0;
    char *end = nullptr;
    const long x = std::strtol(v.c_str(), &end, 10);
    if (errno != 0 || end == v.c_str() || *end != '\0' || x <= 0 || x > INT_MAX) return false;
    if (out) *out = static_cast<int>(x);
    return true;
}

// Positive integer with an optional K/M/B suffix (1e3/1e6/1e9).
bool parse_count(const std::string &v, long long *out) {
    if (v.empty()) return false;
    long long mult = 1;
    std::string digits = v;
    const char last = v.back();
    if (std::isalpha(static_cast<unsigned char>(last))) {
        digits = v.substr(0, v.size() - 1);
        switch (std::toupper(static_cast<unsigned char>(last))) {
        case 'K': mult = 1000LL; break;
        case 'M': mult = 1000000LL; break;
        case 'B': mult = 1000000000LL; break;
        default: return false;
        }
    }
    if (digits.empty()) return false;
    for (char c : digits)
        if (!std::isdigit(static_cast<unsigned char>(c))) return false;
    errno = 0;
    char *end = nullptr;
    const long long x = std::strtoll(digits.c_str(), &end, 10);
    if (errno != 0 || *end != '\0' || x <= 0 || x > LLONG_MAX / mult) return false;
    *out = x * mult;
    return true;
}

void print_usage() {
    std::cout << "\nUsage: multiobj_nobjs<NUM_OBJS> [input file] [problem type] [method] [state_dominance] [options]\n"
              << "\n\twhere:\n"
              << "\t\tproblem_type = 1: knapsack\n\t\tproblem_type = 2: set packing\n\t\tproblem_type = 3: TSP\n\n"
              << "\t\tmethod = 1: top-down BFS\n\t\tmethod = 3: dynamic layer cutset\n\n"
              << "\t\tstate_dominance = 0:  disable state dominance\n\t\tstate_dominance = 1:  state dominance strategy 1\n\n"
              << "\t\t--backend gpu (this build drives the B200 engine only)\n"
              << "\t\t--save-frontier: save Pareto frontier to <input_stem>.frontier.csv.gz\n"
              << "\t\t--frontier-out <path>: save Pareto frontier to explicit gzip CSV path\n"
              << "\t\t--save-stats: save one JSONL record with run statistics\n"
              << "\t\t--stats-out <path>: save JSONL statistics to explicit path\n"
              << "\t\t--max-cand <N>: GPU candidate batch cap; supports K, M, B suffixes (default 20M)\n"
              << "\t\t--max-prod <N>: GPU coupled batch product cap; supports K, M, B suffixes (default 625K)\n"
              << "\t\toptional arguments can be provided in any order\n"
              << std::endl;
}

// Mirrors parse_cli_args (src/pmdd/util/cli_parser.cpp:181-488).
bool parse_args(int argc, char **argv, Options *o, std::string *error) {
    if (argc < 5) return false;
    o->input_path = argv[1];
    o->problem_type = std::atoi(argv[2]);
    o->method = std::atoi(argv[3]);
    o->state_dominance = std::atoi(argv[4]);
    if (o->problem_type < 1 || o->problem_type > 3) {
        *error = "Error - invalid problem type '" + std::string(argv[2]) +
                 "'. Valid problem types are 1 (knapsack), 2 (set packing), 3 (TSP).";
        return false;
    }
    bool backend_set = false, named = false, shorthand = false, threads_set = false, cand_set = false,
         prod_set = false;
    for (int i = 5; i < argc; ++i) {
        const std::string t(argv[i]);
        if (t == "--backend") {
            if (shorthand) { *error = "Error - cannot mix --backend with shorthand backend token."; return false; }
            if (backend_set) { *error = "Error - backend provided multiple times."; return false; }
            if (i + 1 >= argc) { *error = "Error - --backend requires a value (cpu or gpu)."; return false; }
            const std::string v(argv[++i]);
            if (v == "cpu") o->gpu = false;
            else if (v == "gpu") o->gpu = true;
            else if (v == "cuda") { *error = "Error - backend token 'cuda' is unsupported; use 'gpu'."; return false; }
            else { *error = "Error - invalid backend '" + v + "'. Use cpu or gpu."; return false; }
            backend_set = named = true;
        } else if (t == "--cpu-threads") {
            if (threads_set) { *error = "Error - cpu thread count provided multiple times."; return false; }
            if (i + 1 >= argc) { *error = "Error - --cpu-threads requires a positive integer."; return false; }
            const std::string v(argv[++i]);
            if (!parse_positive_int(v, &o->cpu_threads)) {
                *error = "Error - invalid --cpu-threads value '" + v + "' (expected positive integer).";
                return false;
            }
            threads_set = true;
        } else if (t == "--max-cand") {
            if (cand_set) { *error = "Error - GPU candidate batch cap provided multiple times."; return false; }
            if (i + 1 >= argc) {
                *error = "Error - --max-cand requires a positive integer, optionally using K, M, or B suffix.";
                return false;
            }
            const std::string v(argv[++i]);
            if (!parse_count(v, &o->max_cand)) {
                *error = "Error - invalid --max-cand value '" + v +
                         "' (expected positive integer with optional K, M, or B suffix).";
                return false;
            }
            cand_set = true;
        } else if (t == "--max-prod") {
            if (prod_set) { *error = "Error - GPU coupled batch product cap provided multiple times."; return false; }
            if (i + 1 >= argc) {
                *error = "Error - --max-prod requires a positive integer, optionally using K, M, or B suffix.";
                return false;
            }
            const std::string v(argv[++i]);
            if (!parse_count(v, &o->max_prod)) {
                *error = "Error - invalid --max-prod value '" + v +
                         "' (expected positive integer with optional K, M, or B suffix).";
                return false;
            }
            prod_set = true;
        } else if (t == "cpu" || t == "gpu") {
            if (named) { *error = "Error - cannot mix shorthand backend token with --backend."; return false; }
            if (backend_set) { *error = "Error - backend provided multiple times."; return false; }
            o->gpu = (t == "gpu");
            backend_set = shorthand = true;
            if (i + 1 < argc) {
                const std::string nx(argv[i + 1]);
                errno = 0;
                char *end = nullptr;
                const long raw = std::strtol(nx.c_str(), &end, 10);
                const bool is_int = errno == 0 && end != nx.c_str() && *end == '\0';
                if (is_int && t == "gpu") {
                    *error = "Error - gpu shorthand does not accept a kernel value; use 'gpu'.";
                    return false;
                }
                if (is_int && t == "cpu") {
                    if (threads_set) { *error = "Error - cpu threads provided multiple times."; return false; }
                    if (raw <= 0 || raw > INT_MAX) {
                        *error = "Error - invalid cpu shorthand thread count '" + nx + "' (expected positive integer).";
                        return false;
                    }
                    o->cpu_threads = static_cast<int>(raw);
                    threads_set = true;
                    ++i;
                }
            }
        } else if (t == "cuda") {
            *error = "Error - backend token 'cuda' is unsupported; use 'gpu'.";
            return false;
        } else if (t == "--save-frontier") {
            o->save_frontier = true;
        } else if (t == "--frontier-out") {
            if (i + 1 >= argc) { *error = "Error - --frontier-out requires a file path."; return false; }
            o->frontier_out_path = argv[++i];
            if (o->frontier_out_path.empty()) { *error = "Error - --frontier-out path cannot be empty."; return false; }
            o->save_frontier = true;
        } else if (t == "--save-stats") {
            o->save_stats = true;
        } else if (t == "--stats-out") {
            if (i + 1 >= argc) { *error = "Error - --stats-out requires a file path."; return false; }
            o->stats_out_path = argv[++i];
            if (o->stats_out_path.empty()) { *error = "Error - --stats-out path cannot be empty."; return false; }
            o->save_stats = true;
        } else {
            int n = 0;
            if (parse_positive_int(t, &n))
                *error = "Error - positional numeric argument '" + t +
                         "' must immediately follow shorthand backend token cpu|gpu.";
            else
                *error = "Error - unrecognized optional argument '" + t + "'.";
            return false;
        }
    }
    if (o->save_frontier && o->frontier_out_path.empty())
        o->frontier_out_path = stem_of(o->input_path, "frontier") + ".frontier.csv.gz";
    if (o->save_stats && o->stats_out_path.empty()) o->stats_out_path = stem_of(o->input_path, "stats") + ".stats.jsonl";
    if (o->gpu && threads_set) { *error = "Error - cpu thread options are not valid with backend=gpu."; return false; }
    if (!o->gpu && cand_set) { *error = "Error - --max-cand is only valid with backend=gpu."; return false; }
    if (!o->gpu && prod_set) { *error = "Error - --max-prod is only valid with backend=gpu."; return false; }
    if (o->gpu && o->method != 1 && o->method != 3) {
        *error = "Error - GPU backend is unsupported for method " + std::to_string(o->method) + ".";
        return false;
    }
    return true;
}

std::string json_escape(const std::string &v) {
    std::string s;
    for (unsigned char c : v) {
        switch (c) {
        case '"': s += "\\\""; break;
        case '\\': s += "\\\\"; break;
        case '\b': s += "\\b"; break;
        case '\f': s += "\\f"; break;
        case '\n': s += "\\n"; break;
        case '\r': s += "\\r"; break;
        case '\t': s += "\\t"; break;
        default:
            if (c < 0x20) {
                static const char hex[] = "0123456789abcdef";
                s += "\\u00";
                s += hex[(c >> 4) & 15];
                s += hex[c & 15];
            } else {
                s += static_cast<char>(c);
            }
        }
    }
    return s;
}

struct RunTimes {
    double cpu_compile_s = 0, cpu_enumeration_s = 0, wall_compile_s = 0, wall_enumeration_s = 0;
};

template <class V>
void json_array(std::ostream &out, const std::vector<V> &v) {
    out << "[";
    for (size_t i = 0; i < v.size(); ++i) out << (i ? "," : "") << v[i];
    out << "]";
}

bool write_stats(const Options &o, const pmdd_stats &st, const pmdd_dd_info &info, const std::vector<long> &layers,
                 int64_t num_solutions, const RunTimes &rt, std::string *error) {
    std::ofstream out(o.stats_out_path.c_str(), std::ios::out | std::ios::app);
    if (!out.is_open()) {
        *error = "could not open output path";
        return false;
    }
    struct rusage ru;
    getrusage(RUSAGE_SELF, &ru);
    const long long cpu_mem_peak = static_cast<long long>(ru.ru_maxrss) * 1024LL;
    const double cpu_total = rt.cpu_compile_s + rt.cpu_enumeration_s;
    out << std::fixed << std::setprecision(6);
    out << "{\"schema_version\":1,\"identity\":{\"input_path\":\"" << json_escape(o.input_path)
        << "\",\"problem_type\":" << o.problem_type << ",\"method\":" << o.method
        << ",\"state_dominance\":" << o.state_dominance << ",\"backend\":\"gpu\",\"cpu_threads\":" << o.cpu_threads
        << "},";
    out << "\"outputs\":{\"num_solutions\":" << num_solutions << ",\"save_frontier\":"
        << (o.save_frontier ? "true" : "false") << ",\"frontier_out_path\":\"" << json_escape(o.frontier_out_path)
        << "\"},";
    out << "\"timing\":{\"cpu\":{\"cpu_compile_s\":" << rt.cpu_compile_s << ",\"cpu_enumeration_s\":"
        << rt.cpu_enumeration_s << ",\"cpu_total_s\":" << cpu_total << ",\"cpu_state_dominance_s\":" << 0.0
        << "},\"wall\":{\"wall_compile_s\":" << rt.wall_compile_s << ",\"wall_enumeration_s\":" << rt.wall_enumeration_s
        << "},\"kernel\":{\"kernel_expand_td_s\":" << st.kernel_expand_td_s << ",\"kernel_dominance_s\":"
        << st.kernel_dominance_s << ",\"kernel_total_s\":" << st.kernel_total_s << "}},";
    out << "\"memory\":{\"cpu\":{\"cpu_mem_peak_bytes\":" << cpu_mem_peak << "},\"gpu\":{\"gpu_mem_peak_used_bytes\":"
        << st.gpu_mem_peak_used_bytes << ",\"gpu_mem_peak_reserved_bytes\":" << st.gpu_mem_peak_reserved_bytes << "}},";
    out << "\"work\":{\"work_candidates_total\":" << st.work_candidates_total << ",\"work_candidates_peak\":"
        << st.work_candidates_peak << ",\"work_frontier_survivors_total\":" << st.work_frontier_survivors_total
        << ",\"work_frontier_peak_points\":" << st.work_frontier_peak_points << ",\"work_join_products_total\":"
        << st.work_join_products_total << "},";
    out << "\"dominance\":{\"dominance_filtered_total\":" << st.dominance_filtered_total << "},";
    out << "\"structure\":{\"is_tsp_branch\":" << (o.problem_type == 3 ? "true" : "false")
        << ",\"postprocess_sort_applied\":true,\"original_width\":" << info.original_width
        << ",\"reduced_width\":" << info.reduced_width << ",\"original_num_nodes\":" << info.original_num_nodes
        << ",\"reduced_num_nodes\":" << info.reduced_num_nodes << ",\"max_num_nodes_per_layer\":";
    json_array(out, layers);
    out << ",\"max_num_in_arcs\":" << info.max_num_in_arcs << ",\"total_num_in_arcs\":" << info.total_num_in_arcs
        << ",\"layer_coupling\":" << st.layer_coupling << "},";
    out << "\"metrics\":{\"wall_state_dominance_s\":" << 0.0 << ",\"wall_cutset_sort_s\":" << 0.0
        << ",\"wall_cutset_convolution_s\":" << 0.0 << ",\"wall_cutset_partial_merge_s\":" << 0.0
        << ",\"wall_pack_transfer_s\":" << st.wall_pack_transfer_s << ",\"wall_join_s\":" << st.wall_join_s
        << ",\"cpu_layers_td\":" << st.layers_td << ",\"cpu_layers_bu\":" << st.layers_bu
        << ",\"cpu_nodes_expanded\":0,\"cpu_cutset_size\":" << st.cutset_size
        << ",\"std_candidates_per_layer\":[],\"std_frontier_survivors_per_layer\":[]},";
    out << "\"status\":{\"status_state\":\"ok\",\"status_error_message\":\"\"}}\n";
    if (!out.good()) {
        *error = "failed while writing JSONL output";
        return false;
    }
    return true;
}

int nobjs_from_name(const char *argv0) {
    const char *env = std::getenv("PMDD_NOBJS");
    if (env && *env) return std::atoi(env);
    std::string s(argv0 ? argv0 : "");
    size_t i = s.size();
    while (i > 0 && std::isdigit(static_cast<unsigned char>(s[i - 1]))) --i;
    if (i < s.size()) return std::atoi(s.c_str() + i);
    return 3;
}

}  // namespace

int main(int argc, char **argv) {
    Options o;
    std::string perr;
    if (!parse_args(argc, argv, &o, &perr)) {
        if (!perr.empty()) std::cout << perr << std::endl;
        print_usage();
        return 1;
    }
    if (!o.gpu) {
        std::cout << "Error - this build runs the B200 GPU engine only; use --backend gpu." << std::endl;
        return 1;
    }
    const int nobjs = nobjs_from_name(argv[0]);
    // one instance per process: let the engine use most of the free device memory
    setenv("PMDD_ARENA_FRACTION", "0.85", 0);
    typedef std::chrono::steady_clock Clock;
    RunTimes rt;
    // compile: read + DD construction (for TSP the reference times construction only)
    std::ifstream in(o.input_path.c_str());
    if (!in.is_open()) {
        std::cout << "Error - file " << o.input_path << " could not be found" << std::endl;
        return 1;
    }
    std::stringstream ss;
    ss << in.rdbuf();
    const Clock::time_point w0 = Clock::now();
    const clock_t c0 = std::clock();
    pmdd::FlatDD dd;
    try {
        dd = pmdd::build_from_text(ss.str(), o.problem_type, nobjs);
    } catch (const std::exception &e) {
        std::cout << "Error - " << e.what() << std::endl;
        return 1;
    }
    rt.cpu_compile_s = static_cast<double>(std::clock() - c0) / CLOCKS_PER_SEC;
    rt.wall_compile_s = std::chrono::duration<double>(Clock::now() - w0).count();

    pmdd_options opts;
    pmdd_options_default(&opts);
    opts.method = o.method;
    opts.problem_type = o.problem_type;
    opts.state_dominance = o.state_dominance;
    opts.max_cand = o.max_cand;
    opts.max_prod = o.max_prod;
    const pmdd_dd view = dd.view();
    pmdd_frontier fr;
    pmdd_stats st;
    char err[512] = {0};
    const Clock::time_point w1 = Clock::now();
    const clock_t c1 = std::clock();
    const int rc = pmdd_enumerate(&view, &opts, &fr, &st, err, sizeof(err));
    rt.cpu_enumeration_s = static_cast<double>(std::clock() - c1) / CLOCKS_PER_SEC;
    rt.wall_enumeration_s = std::chrono::duration<double>(Clock::now() - w1).count();
    if (rc != PMDD_OK) {
        std::cout << "Error - GPU backend requested but " << (o.method == 3 ? "coupled" : "top-down")
                  << " enumeration failed";
        if (err[0]) std::cout << ": " << err;
        std::cout << std::endl;
        return 1;
    }
    if (fr.elem_bytes != 4) {
        std::cout << "Error - objective sums exceed 32-bit integers; use the library API for 64-bit frontiers"
                  << std::endl;
        pmdd_frontier_free(&fr);
        return 1;
    }
    std::vector<int32_t> pts(static_cast<const int32_t *>(fr.points),
                             static_cast<const int32_t *>(fr.points) + fr.num_points * nobjs);
    const int64_t num_solutions = fr.num_points;
    pmdd_frontier_free(&fr);
    pmdd_sort_points_lex_ascending(pts.data(), num_solutions, nobjs);
    if (o.save_frontier) {
        char e[256] = {0};
        if (pmdd_write_frontier_csv_gz(pts.data(), num_solutions, nobjs, 4, 0, o.frontier_out_path.c_str(), e,
                                       sizeof(e)) != PMDD_OK) {
            std::cout << "Error - failed to save frontier to '" << o.frontier_out_path << "': " << e << std::endl;
            return 1;
        }
    }
    const double cpu_total = rt.cpu_compile_s + rt.cpu_enumeration_s;
    std::cout << num_solutions << std::endl << cpu_total << std::endl;
    const pmdd_dd_info &info = dd.info;
    if (o.problem_type == 3) {
        std::cout << rt.cpu_compile_s << "\t" << rt.cpu_enumeration_s << "\t" << rt.wall_compile_s << "\t"
                  << rt.wall_enumeration_s << std::endl;
    } else {
        std::cout << o.method << "\t" << o.state_dominance << "\t" << info.original_width << "\t" << info.reduced_width
                  << "\t" << info.original_num_nodes << "\t" << info.reduced_num_nodes << "\t" << rt.cpu_compile_s
                  << "\t" << rt.cpu_enumeration_s << "\t" << st.layer_coupling << "\t" << st.dominance_filtered_total
                  << "\t" << 0 << "\t" << rt.wall_compile_s << "\t" << rt.wall_enumeration_s << std::endl;
    }
    if (o.save_stats) {
        std::vector<long> layers;
        for (int l = 0; l < dd.num_layers(); ++l) layers.push_back(dd.layer_offsets[l + 1] - dd.layer_offsets[l]);
        std::string e;
        if (!write_stats(o, st, info, layers, num_solutions, rt, &e)) {
            std::cerr << "Error - failed to save stats to '" << o.stats_out_path << "': " << e << '\n';
            return 1;
        }
    }
    return 0;
}
