// hybrid_bfs: same flags and flow as the reference sample
// (samples/hybrid_bfs/main.cpp, hybrid_bfs.cu:173-243), driving the engine
// through the C ABI.
#include <algorithm>

#include "sg_skeleton.h"

DEFINE_int32(source_node, 0, "The source node for the BFS traversal (clamped to [0, nnodes-1])");
DEFINE_bool(sparse, false, "use async/push/dd + fusion for high-diameter");
DEFINE_string(variant, "", "force variant as async/sync push/pull dd/td");
DEFINE_bool(non_atomic, true, "using non-atomic operation for accumulate");

static bool HybridBFS() {
    LoadedGraph g;
    if (!LoadGraph(g)) return false;
    const uint32_t src = (uint32_t)std::min<int64_t>(std::max<int64_t>(0, FLAGS_source_node), g.nv - 1);
    sg_options o = CommonOptions();
    o.non_atomic = FLAGS_non_atomic;
    if (!FLAGS_variant.empty()) {
        if (FLAGS_variant != "async_push_dd" && FLAGS_variant != "async_pull_dd") {
            std::fprintf(stderr, "unsupported variant\n");
            return false;
        }
        o.variant = parse_variant(FLAGS_variant);
    }
    if (FLAGS_sparse) {
        o.fused = 1;
        o.variant = SG_ASYNC_PUSH_DD;
        o.lb_push = SG_LB_NONE;
    } else if (o.lb_pull == SG_LB_AUTO) {
        o.lb_pull = SG_LB_NONE;  // hybrid_bfs.cu:210
    }
    std::vector<uint32_t> levels(g.nv);
    std::vector<sg_round_trace> trace(FLAGS_trace ? std::max(1, FLAGS_max_iteration) : 0);
    sg_stats st{};
    st.trace = trace.empty() ? nullptr : trace.data();
    st.trace_capacity = (uint32_t)trace.size();
    JsonRecord js;
    SG_CHECK(sg_bfs(g.dev, src, &o, levels.data(), &st));
    PrintRun(st, o, g, false, js);
    js.put("non_atomic", FLAGS_non_atomic ? "YES" : "NO");
    bool ok = true;
    if (FLAGS_check) {
        const auto ref = HostBFS(g, src);
        int errors = 0;
        for (uint32_t v = 0; v < g.nv; ++v) errors += levels[v] != ref[v];
        std::printf("total errors: %d\n", errors);
        ok = errors == 0;
    } else {
        std::printf("Warning: Result not checked\n");
    }
    if (!FLAGS_output.empty()) {
        FILE *f = std::fopen(FLAGS_output.c_str(), "w");
        for (uint32_t v = 0; f && v < g.nv; ++v)
            levels[v] == 0xffffffffu ? std::fprintf(f, "%u INF\n", v) : std::fprintf(f, "%u %u\n", v, levels[v]);
        if (f) std::fclose(f);
    }
    sg_graph_destroy(g.dev);
    return ok;
}

struct App {
    static const char *Name() { return "bfs"; }
    static const char *NameUpper() { return "BFS"; }
    static bool Single() { return HybridBFS(); }
};

int main(int argc, char **argv) { return Skeleton<App>()(argc, argv); }
