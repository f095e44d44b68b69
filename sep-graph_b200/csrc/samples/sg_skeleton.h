// Shared command-line surface of the hybrid_* samples: the flags of the
// reference's include/utils/app_skeleton.h:42-87 with the same names and
// defaults, the Skeleton<App> single / interactive / command-file driver
// (app_skeleton.h:92-158, interactors of include/utils/interactor.h), graph
// loading with a per-process cache (GetCachedGraph, src/utils/utils.cpp:37-65),
// and the small checkers behind --check.  Everything here calls the library
// through include/sepgraph.h only.
#pragma once
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <deque>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../../include/sepgraph.h"
#include "sg_flags.h"

// App (app_skeleton.h:41-46)
DEFINE_bool(interactive, false, "Run an interactive session");
DEFINE_string(cmdfile, "", "A file with commands to execute");
DEFINE_int32(max_iteration, 200, "Maximum iterated rounds");
DEFINE_bool(priority, false, "Enable priority scheduling (may not available for all algorithms)");
DEFINE_int32(prio_delta, 0, "The soft priority delta");
// DO algorithms (48-51)
DEFINE_double(edge_factor, 1.0, "Unvisited edges = edge_factor * nedges");
DEFINE_double(alpha, 15, "DO BFS/SSSP/BC heuristic parameter");
DEFINE_double(beta, 18, "DO BFS/SSSP/BC heuristic parameter");
// General (53-59)
DEFINE_string(output, "", "File to store output to");
DEFINE_bool(check, false, "Check results");
DEFINE_bool(verbose, true, "Verbose prints");
DEFINE_bool(trace, false, "Trace prints (effects performance)");
DEFINE_string(lb_push, "", "load-balancing policy for push (none/coarse/fine/hybrid)");
DEFINE_string(lb_pull, "", "load-balancing policy for pull (none/coarse/fine/hybrid)");
// Input (61-66)
DEFINE_string(graphfile, "", "A file with a graph in Galois .gr or MatrixMarket format");
DEFINE_string(format, "gr", "graph format (gr/market)");
DEFINE_bool(undirected, false, "treat input graph as undirected graph");
DEFINE_string(json, "", "output running data as json format");
DEFINE_bool(stats, false, "Print graph statistics");
// Generation (68-76); gen_seed and gen_rmat_scale are additions (seeded generators)
DEFINE_bool(gen_graph, false, "Generate a random graph");
DEFINE_int32(gen_nnodes, 100000, "Number of nodes for random graph generation");
DEFINE_int32(gen_factor, 10, "A factor number for graph generation");
DEFINE_int32(gen_method, 0, "0: random graph, 1/2: two-way chain, 3: cliques, 4: RMAT (--gen_rmat_scale)");
DEFINE_bool(gen_weights, false, "Generate edge weights if missing in graph input");
DEFINE_int32(gen_weight_range, 100, "The range to generate edge weights from");
DEFINE_int32(gen_seed, 1, "Seed of the graph and weight generators");
DEFINE_int32(gen_rmat_scale, 16, "RMAT scale for --gen_method 4 (edge factor = --gen_factor)");
// System (79-81)
DEFINE_int32(block_size, 256, "Block size for traversal kernels");
DEFINE_int32(grid_size, 20, "Grid size for traversal kernels (resident blocks per SM here; 0 = auto)");
// Worklist (84-87)
DEFINE_double(wl_alloc_factor, 0.2, "Worklist allocation factor (worklists are bounded by |V| here)");
DEFINE_bool(wl_sort, false, "Sort worklist by node id");
DEFINE_bool(wl_unique, false, "Unique duplicated nodes (worklists never hold duplicates here)");
DEFINE_int32(device, 0, "CUDA device");

#define SG_CHECK(call)                                                                                       \
    do {                                                                                                     \
        sg_status _s = (call);                                                                               \
        if (_s != SG_OK) {                                                                                   \
            std::fprintf(stderr, "%s failed: %s (%s)\n", #call, sg_status_string(_s), sg_last_error(g_ctx)); \
            return false;                                                                                    \
        }                                                                                                    \
    } while (0)

static sg_ctx *g_ctx = nullptr;

// The run record written when --json is set (JsonWriter, src/utils/to_json.cpp:8-61):
// one object with the keys of Engine::SaveToJson (framework.cuh:205-257) and the
// sample's own, numbers, strings and string lists, keys sorted and indented by
// four spaces as the reference's writer prints them.
struct JsonRecord {
    std::map<std::string, std::string> kv;  // key -> serialised value
    static std::string quote(const std::string &s) {
        std::string r = "\"";
        for (unsigned char ch : s) {
            if (ch == '"' || ch == '\\') {
                r += '\\';
                r += (char)ch;
            } else if (ch < 0x20) {
                char b[8];
                std::snprintf(b, sizeof b, "\\u%04x", ch);
                r += b;
            } else {
                r += (char)ch;
            }
        }
        return r + "\"";
    }
    void put(const std::string &k, double v) {
        char b[64];
        if (std::isfinite(v)) std::snprintf(b, sizeof b, "%.9g", v);
        else std::snprintf(b, sizeof b, "null");
        kv[k] = b;
    }
    void put_int(const std::string &k, long long v) { kv[k] = std::to_string(v); }
    void put(const std::string &k, const std::string &v) { kv[k] = quote(v); }
    void put(const std::string &k, const char *v) { kv[k] = quote(v); }
    void put(const std::string &k, const std::vector<std::string> &v) {
        if (v.empty()) {
            kv[k] = "[]";
            return;
        }
        std::string r = "[\n";
        for (size_t i = 0; i < v.size(); ++i) r += "        " + quote(v[i]) + (i + 1 < v.size() ? ",\n" : "\n");
        kv[k] = r + "    ]";
    }
    double get(const std::string &k) const {
        auto it = kv.find(k);
        return it == kv.end() ? 0.0 : std::atof(it->second.c_str());
    }
    ~JsonRecord() {
        if (FLAGS_json.empty()) return;
        std::ofstream f(FLAGS_json);
        f << "{\n";
        size_t i = 0;
        for (const auto &e : kv) f << "    " << quote(e.first) << ": " << e.second << (++i < kv.size() ? ",\n" : "\n");
        f << "}\n";
    }
};

struct LoadedGraph {
    sg_hgraph *host = nullptr;
    sg_graph *dev = nullptr;
    uint32_t nv = 0;
    uint64_t ne = 0;
    const uint32_t *off = nullptr, *idx = nullptr, *w = nullptr;
};

// Host graph cache across interactive commands (GetCachedGraph).
static std::map<std::string, sg_hgraph *> &graph_cache() {
    static std::map<std::string, sg_hgraph *> m;
    return m;
}

inline void CleanupGraphs() {
    for (auto &kv : graph_cache()) sg_hgraph_destroy(kv.second);
    graph_cache().clear();
}

inline sg_status gen_host_graph(sg_hgraph **out) {
    const uint64_t seed = (uint64_t)FLAGS_gen_seed;
    switch (FLAGS_gen_method) {
        case 4:
            return sg_hgraph_gen_rmat(FLAGS_gen_rmat_scale, FLAGS_gen_factor, 0.57, 0.19, 0.19, seed, 0, out);
        case 1:
        case 2: {  // two-way chain
            const uint32_t n = (uint32_t)FLAGS_gen_nnodes;
            std::vector<uint32_t> off(n + 1, 0), idx;
            for (uint32_t v = 0; v < n; ++v) {
                if (v > 0) idx.push_back(v - 1);
                if (v + 1 < n) idx.push_back(v + 1);
                off[v + 1] = (uint32_t)idx.size();
            }
            return sg_hgraph_from_csr(n, idx.size(), off.data(), idx.data(), nullptr, out);
        }
        case 3: {  // disjoint cliques of gen_factor vertices
            const uint32_t n = (uint32_t)FLAGS_gen_nnodes, k = std::max(1, FLAGS_gen_factor);
            std::vector<uint32_t> off(n + 1, 0), idx;
            for (uint32_t v = 0; v < n; ++v) {
                const uint32_t b = v / k * k, e = std::min(n, b + k);
                for (uint32_t u = b; u < e; ++u)
                    if (u != v) idx.push_back(u);
                off[v + 1] = (uint32_t)idx.size();
            }
            return sg_hgraph_from_csr(n, idx.size(), off.data(), idx.data(), nullptr, out);
        }
        default:
            return sg_hgraph_gen_random(FLAGS_gen_nnodes, FLAGS_gen_factor, seed, out);
    }
}

inline bool LoadGraph(LoadedGraph &lg) {
    sg_hgraph *h = nullptr;
    std::string key;
    if (FLAGS_gen_graph) {
        key = "gen:" + std::to_string(FLAGS_gen_method) + ":" + std::to_string(FLAGS_gen_nnodes) + ":" +
              std::to_string(FLAGS_gen_factor) + ":" + std::to_string(FLAGS_gen_seed) + ":" +
              std::to_string(FLAGS_gen_rmat_scale);
    } else {
        if (FLAGS_graphfile.empty()) {
            std::printf("A Graph File must be provided\n");
            return false;
        }
        key = FLAGS_format + ":" + FLAGS_graphfile;
    }
    auto it = graph_cache().find(key);
    if (it != graph_cache().end()) {
        h = it->second;
    } else {
        sg_status st;
        if (FLAGS_gen_graph)
            st = gen_host_graph(&h);
        else if (FLAGS_format == "gr")
            st = sg_hgraph_read_gr(FLAGS_graphfile.c_str(), &h);
        else if (FLAGS_format == "market")
            st = sg_hgraph_read_market(FLAGS_graphfile.c_str(), 0, &h);
        else {
            std::fprintf(stderr, "unsupported graph format '%s' (gr/market)\n", FLAGS_format.c_str());
            return false;
        }
        if (st != SG_OK) {
            std::fprintf(stderr, "loading graph failed: %s\n", sg_status_string(st));
            return false;
        }
        graph_cache()[key] = h;
    }
    sg_hgraph_info(h, &lg.nv, &lg.ne, &lg.off, &lg.idx, &lg.w);
    if (!lg.w && FLAGS_gen_weights) {
        if (FLAGS_verbose)
            std::printf("\nNo edge data in the input graph, generating edge weights from the range [1, %d]\n",
                        FLAGS_gen_weight_range);
        sg_hgraph_gen_weights(h, 1, (uint32_t)FLAGS_gen_weight_range + 1, (uint64_t)FLAGS_gen_seed + 1);
        sg_hgraph_info(h, &lg.nv, &lg.ne, &lg.off, &lg.idx, &lg.w);
    }
    if (lg.nv == 0) {
        std::printf("Empty graph!\n");
        return false;
    }
    if (FLAGS_stats) {
        uint32_t v = 0, d = 0;
        sg_hgraph_max_degree_vertex(h, &v, &d);
        std::printf("The graph has %u vertices, and %llu edges (avg. degree: %f, max. degree: %u)\n", lg.nv,
                    (unsigned long long)lg.ne, (double)lg.ne / lg.nv, d);
        return false;
    }
    if (!g_ctx && sg_init(FLAGS_device, &g_ctx) != SG_OK) {
        std::fprintf(stderr, "no usable CUDA device\n");
        return false;
    }
    lg.host = h;
    const sg_status st = sg_graph_create_from_host(g_ctx, h, FLAGS_undirected ? SG_GRAPH_SYMMETRIC : 0, &lg.dev);
    if (st != SG_OK) {
        std::fprintf(stderr, "sg_graph_create: %s (%s)\n", sg_status_string(st), sg_last_error(g_ctx));
        return false;
    }
    if (FLAGS_verbose)
        std::printf("The graph has %u vertices, and %llu edges (average degree: %f)\n", lg.nv,
                    (unsigned long long)lg.ne, (double)lg.ne / lg.nv);
    return true;
}

inline int parse_lb(const std::string &s) {
    if (s.empty()) return SG_LB_AUTO;
    if (s == "none") return SG_LB_NONE;
    if (s == "coarse") return SG_LB_COARSE_GRAINED;
    if (s == "fine") return SG_LB_FINE_GRAINED;
    if (s == "hybrid") return SG_LB_HYBRID;
    std::fprintf(stderr, "unknown load-balancing policy '%s'\n", s.c_str());
    std::exit(1);
}

inline int parse_variant(const std::string &s) {
    static const char *names[] = {"sync_push_td", "sync_push_dd", "sync_pull_td", "sync_pull_dd",
                                  "async_push_td", "async_push_dd", "async_pull_td", "async_pull_dd"};
    for (int i = 0; i < 8; ++i)
        if (s == names[i]) return i;
    return -2;
}

inline const char *variant_name(int v) {
    static const char *names[] = {"SYNC_PUSH_TD", "SYNC_PUSH_DD", "SYNC_PULL_TD", "SYNC_PULL_DD",
                                  "ASYNC_PUSH_TD", "ASYNC_PUSH_DD", "ASYNC_PULL_TD", "ASYNC_PULL_DD"};
    return v >= 0 && v < 8 ? names[v] : "AUTO";
}

// Options common to every sample, from the shared flags.
inline sg_options CommonOptions() {
    sg_options o;
    sg_options_default(&o);
    o.max_iteration = FLAGS_max_iteration;
    o.alpha = FLAGS_alpha;
    o.beta = FLAGS_beta;
    o.edge_factor = FLAGS_edge_factor;
    o.lb_push = parse_lb(FLAGS_lb_push);
    o.lb_pull = parse_lb(FLAGS_lb_pull);
    o.trace = FLAGS_trace;
    o.wl_sort = FLAGS_wl_sort;
    o.blocks_per_sm = FLAGS_grid_size > 0 && FLAGS_grid_size <= 32 ? FLAGS_grid_size : 0;
    return o;
}

inline const char *lb_name(int lb) {  // LBToString (common.h:179-200)
    switch (lb) {
        case SG_LB_NONE: return "NONE";
        case SG_LB_COARSE_GRAINED: return "COARSED_GRAINED";
        case SG_LB_FINE_GRAINED: return "FINE_GRAINED";
        case SG_LB_HYBRID: return "HYBRID";
        default: return "UNKNOWN";
    }
}

// PrintInfo / --trace lines (framework.cuh:259-313, 334-348) and the run
// record's SaveToJson keys (framework.cuh:205-257).  `iterative` is the
// engine's AlgoType (ITERATIVE_SCHEME for PageRank).
inline void PrintRun(const sg_stats &st, const sg_options &o, const LoadedGraph &g, bool iterative, JsonRecord &js) {
    std::vector<std::string> rounds;
    if (FLAGS_trace)
        for (uint32_t i = 0; i < st.n_trace; ++i) {
            const sg_round_trace &t = st.trace[i];
            char line[512];
            std::snprintf(line, sizeof line,
                          "Round: %u Policy to execute: %s Time: %f In-nodes: %u Out-nodes: %u Input-edges: %llu "
                          "Output-edges: %llu Total-workload: %lld",
                          t.round, variant_name(t.variant), t.time_ms, t.in_nodes, t.out_nodes,
                          (unsigned long long)t.in_workload, (unsigned long long)t.out_workload,
                          (long long)t.total_workload);
            std::printf("%s\n", line);
            rounds.emplace_back(line);
        }
    std::printf("--------------Time statistics---------\n");
    std::printf("Kernel time: %f\n", st.time_kernel_ms);
    std::printf("Total time: %f\n", st.time_total_ms);
    std::printf("Total rounds: %u\n", st.rounds);
    std::printf("Time/round: %f\n", st.rounds ? st.time_total_ms / st.rounds : 0.0);
    std::printf("--------------Engine info-------------\n");
    if (o.variant >= 0) std::printf("Force variant: %s\n", variant_name(o.variant));
    for (int v = 0; v < 8; ++v)
        if (st.rounds_by_variant[v]) std::printf("%s rounds: %u\n", variant_name(v), st.rounds_by_variant[v]);
    std::printf("Max iteration reached: %s\n", st.max_iteration_reached ? "YES" : "NO");
    std::printf("Edges reached: %llu  GTEPS: %f\n", (unsigned long long)st.edges_reached,
                st.time_total_ms > 0 ? st.edges_reached / st.time_total_ms / 1e6 : 0.0);
    // The reference times these host-side stages around separate kernels; here
    // they run inside the one device-resident launch and are part of time_kernel.
    for (const char *k : {"time_input_active_node", "time_output_active_node", "time_input_workload",
                          "time_output_workload", "time_queue2bitmap", "time_bitmap2queue", "time_rebuild_worklist",
                          "time_priority_sample", "time_sort_worklist", "time_unique_worklist"})
        js.put(k, 0.0);
    js.put("time_kernel", st.time_kernel_ms);
    js.put("time_total", st.time_total_ms);
    js.put("time_per_round", st.rounds ? st.time_total_ms / st.rounds : 0.0);
    js.put_int("num_iteration", st.rounds);
    if (o.variant >= 0) js.put("force_variant", variant_name(o.variant));
    if (o.lb_push != SG_LB_AUTO) js.put("force_push_load_balancing", lb_name(o.lb_push));
    if (o.lb_pull != SG_LB_AUTO) js.put("force_pull_load_balancing", lb_name(o.lb_pull));
    if (o.priority == SG_PRIORITY_LOW_HIGH) {
        js.put("priority_type", "low_high");
        js.put("priority_delta", o.priority_delta);
    } else if (o.priority == SG_PRIORITY_SAMPLING) {
        js.put("priority_type", "sampling");
        js.put("cut_threshold", o.cut_threshold);
    } else {
        js.put("priority_type", "none");
    }
    js.put("fused_kernel", o.fused ? "YES" : "NO");
    js.put("max_iteration_reached", st.max_iteration_reached ? "YES" : "NO");
    char dev[256] = "";
    if (g_ctx && sg_device_info(g_ctx, nullptr, nullptr, nullptr, dev, sizeof dev) == SG_OK) js.put("device", dev);
    js.put("dataset", FLAGS_graphfile);
    js.put_int("nnodes", g.nv);
    js.put_int("nedges", (long long)g.ne);
    js.put("algo_type", iterative ? "ITERATIVE_SCHEME" : "TRAVERSAL_SCHEME");
    if (FLAGS_trace) js.put("round", rounds);
}

// ---- host checkers behind --check (FIFO BFS / label-correcting SSSP /
// residual-push PageRank / Brandes BC, as the samples' *_host.cpp compute them)
inline std::vector<uint32_t> HostBFS(const LoadedGraph &g, uint32_t s) {
    std::vector<uint32_t> lv(g.nv, 0xffffffffu);
    std::deque<uint32_t> q{s};
    lv[s] = 0;
    while (!q.empty()) {
        uint32_t u = q.front();
        q.pop_front();
        for (uint32_t e = g.off[u]; e < g.off[u + 1]; ++e)
            if (lv[g.idx[e]] == 0xffffffffu) {
                lv[g.idx[e]] = lv[u] + 1;
                q.push_back(g.idx[e]);
            }
    }
    return lv;
}

inline std::vector<uint32_t> HostSSSP(const LoadedGraph &g, uint32_t s) {
    std::vector<uint32_t> d(g.nv, 0xffffffffu);
    std::deque<uint32_t> q{s};
    d[s] = 0;
    while (!q.empty()) {
        uint32_t u = q.front();
        q.pop_front();
        for (uint32_t e = g.off[u]; e < g.off[u + 1]; ++e) {
            uint32_t c = d[u] + (g.w ? g.w[e] : 1u);
            if (c < d[g.idx[e]]) {
                d[g.idx[e]] = c;
                q.push_back(g.idx[e]);
            }
        }
    }
    return d;
}

template <class App>
struct Skeleton {
    int operator()(int argc, char **argv) {
        if (!sgflags::ParseCommandLineFlags(&argc, &argv, true)) return 1;
        int rc = 0;
        if (!FLAGS_cmdfile.empty()) {
            std::ifstream f(FLAGS_cmdfile);
            if (!f) {
                std::fprintf(stderr, "cannot open command file %s\n", FLAGS_cmdfile.c_str());
                return 1;
            }
            std::cout << "\nStarting a command file " << App::Name() << " session" << std::endl;
            std::string line;
            while (std::getline(f, line)) rc |= RunCommand(line);
        } else if (FLAGS_interactive) {
            std::cout << "\nStarting an interactive " << App::Name() << " session" << std::endl;
            rc = Run();
            std::string line;
            while (true) {
                std::cout << "\n<< " << std::flush;
                if (!std::getline(std::cin, line) || line == "exit" || line == "x") break;
                rc |= RunCommand(line);
            }
        } else {
            rc = Run();
        }
        CleanupGraphs();
        if (g_ctx) sg_destroy(g_ctx);
        return rc;
    }

    int RunCommand(const std::string &line) {
        sgflags::FlagSaver fs;
        std::vector<std::string> toks{App::Name()};
        std::istringstream is(line);
        for (std::string t; is >> t;) toks.push_back(t);
        std::vector<char *> av;
        for (auto &t : toks) av.push_back(&t[0]);
        int ac = (int)av.size();
        char **avp = av.data();
        if (!sgflags::ParseCommandLineFlags(&ac, &avp, false)) return 1;
        return Run();
    }

    // Returns 0 when the run (and --check) passed; the reference prints the
    // check's outcome but always returns 0 (app_skeleton.h:155-156).
    int Run() {
        std::printf("\nTesting single GPU %s\n--------------------\n\n", App::NameUpper());
        const bool ok = App::Single();
        std::printf("Overall: Test %s\n", ok ? "passed" : "FAILED");
        return ok ? 0 : 1;
    }
};
