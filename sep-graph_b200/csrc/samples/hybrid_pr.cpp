// hybrid_pr: flags and flow of samples/hybrid_pr (main.cpp, hybrid_pr.cu:128-210,
// hybrid_pr_host.cpp:36-38).  --check compares against a residual-push
// PageRank in double with the sample's 5% relative rule (hybrid_pr_host.cpp:126-161).
#include <algorithm>
#include <cmath>
#include <numeric>

#include "sg_skeleton.h"

DEFINE_double(cut_threshold, 0, "Cut threshold for index calculation");
DEFINE_bool(sparse, false, "disable load-balancing for sparse graph");
DEFINE_string(variant, "", "force variant as async/sync push/pull dd/td");
DEFINE_double(error, 0.01, "PR error tolerance");
DEFINE_int32(top_ranks, 10, "The number of top ranks to compare for PR regression");
DEFINE_bool(print_ranks, false, "Write out ranks to output");
DEFINE_bool(norm, false, "Normalize PR output ranks (L1)");

static std::vector<double> HostPR(const LoadedGraph &g, double error) {
    std::vector<double> res(g.nv, 0.0), rank(g.nv, 0.15);
    for (uint32_t u = 0; u < g.nv; ++u) {
        uint32_t d = g.off[u + 1] - g.off[u];
        if (!d) continue;
        for (uint32_t e = g.off[u]; e < g.off[u + 1]; ++e) res[g.idx[e]] += 0.15 * 0.85 / d;
    }
    std::deque<uint32_t> q;
    for (uint32_t u = 0; u < g.nv; ++u) q.push_back(u);
    while (!q.empty()) {
        uint32_t u = q.front();
        q.pop_front();
        double r = res[u];
        rank[u] += r;
        res[u] = 0;
        uint32_t d = g.off[u + 1] - g.off[u];
        if (!d) continue;
        for (uint32_t e = g.off[u]; e < g.off[u + 1]; ++e) {
            double p = res[g.idx[e]];
            res[g.idx[e]] += r * 0.85 / d;
            if (p < error && p + r * 0.85 / d > error) q.push_back(g.idx[e]);
        }
    }
    return rank;
}

static bool HybridPageRank() {
    LoadedGraph g;
    if (!LoadGraph(g)) return false;
    sg_options o = CommonOptions();
    o.pr_error = FLAGS_error;
    if (FLAGS_cut_threshold > 0) {  // engine_opt.SetSampleBasedPriority (hybrid_pr.cu:135-137)
        o.priority = SG_PRIORITY_SAMPLING;
        o.cut_threshold = FLAGS_cut_threshold;
    }
    if (FLAGS_sparse) {
        o.lb_push = SG_LB_NONE;
        o.lb_pull = SG_LB_NONE;
    }
    if (!FLAGS_variant.empty()) {
        if (FLAGS_variant != "async_push_dd" && FLAGS_variant != "async_push_td" && FLAGS_variant != "sync_pull_td") {
            std::fprintf(stderr, "unsupported variant\n");
            return false;
        }
        o.variant = parse_variant(FLAGS_variant);
    }
    std::vector<float> ranks(g.nv), residual(g.nv);
    std::vector<sg_round_trace> trace(FLAGS_trace ? std::max(1, FLAGS_max_iteration) : 0);
    sg_stats st{};
    st.trace = trace.empty() ? nullptr : trace.data();
    st.trace_capacity = (uint32_t)trace.size();
    JsonRecord js;
    SG_CHECK(sg_pagerank(g.dev, &o, ranks.data(), residual.data(), &st));
    PrintRun(st, o, g, true, js);
    js.put("error_tolerance", FLAGS_error);
    double sum = 0;
    for (float r : ranks) sum += r;
    std::printf("Total rank : %f\nmax residual: %f\n", sum, *std::max_element(residual.begin(), residual.end()));
    bool ok = true;
    if (FLAGS_check) {
        auto ref = HostPR(g, FLAGS_error);
        std::vector<double> a(ranks.begin(), ranks.end());
        if (FLAGS_norm) {
            double sa = std::accumulate(a.begin(), a.end(), 0.0), sr = std::accumulate(ref.begin(), ref.end(), 0.0);
            for (auto &x : a) x /= sa;
            for (auto &x : ref) x /= sr;
        }
        int diffs = 0;
        for (uint32_t v = 0; v < g.nv; ++v) {
            if (std::fabs(a[v]) < 0.01 && std::fabs(ref[v] - 1) < 0.01) continue;
            const double err = std::fabs(a[v]) < 0.01 ? std::fabs(a[v] - ref[v]) : std::fabs((a[v] - ref[v]) / ref[v]);
            diffs += err > 0.05;
        }
        std::printf("total errors: %d\n", diffs);
        ok = diffs == 0;
    } else {
        std::printf("Warning: Result not checked\n");
    }
    if (!FLAGS_output.empty()) {
        std::vector<uint32_t> order(g.nv);
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return ranks[x] > ranks[y]; });
        FILE *f = std::fopen(FLAGS_output.c_str(), "w");
        if (f) {
            std::fprintf(f, "ALPHA %e EPSILON %e\nRANKS 1--%u of %u\n", 0.85, FLAGS_error, g.nv, g.nv);
            for (uint32_t i = 0; i < g.nv; ++i) {
                if (!FLAGS_print_ranks)
                    std::fprintf(f, "%u %u\n", i + 1, order[i]);
                else
                    std::fprintf(f, "%u %e\n", order[i], FLAGS_norm ? ranks[order[i]] / sum : ranks[order[i]]);
            }
            std::fclose(f);
        }
    }
    sg_graph_destroy(g.dev);
    return ok;
}

struct App {
    static const char *Name() { return "page rank"; }
    static const char *NameUpper() { return "Page Rank"; }
    static bool Single() { return HybridPageRank(); }
};

int main(int argc, char **argv) { return Skeleton<App>()(argc, argv); }
