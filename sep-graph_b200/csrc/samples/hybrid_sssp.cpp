// hybrid_sssp: flags and flow of samples/hybrid_sssp (hybrid_sssp.cu:151-243).
#include <algorithm>

#include "sg_skeleton.h"

DEFINE_int32(source_node, 0, "The source node for the SSSP traversal (clamped to [0, nnodes-1])");
DEFINE_bool(sparse, false, "use async/push/dd + fusion for high-diameter");
DEFINE_string(variant, "", "force variant as async/sync push/pull dd/td");

static bool HybridSSSP() {
    LoadedGraph g;
    if (!LoadGraph(g)) return false;
    const uint32_t src = (uint32_t)std::min<int64_t>(std::max<int64_t>(0, FLAGS_source_node), g.nv - 1);
    sg_options o = CommonOptions();
    if (!FLAGS_variant.empty()) {
        if (FLAGS_variant != "async_push_dd" && FLAGS_variant != "async_pull_dd" && FLAGS_variant != "async_push_td") {
            std::fprintf(stderr, "unsupported variant\n");
            return false;
        }
        o.variant = parse_variant(FLAGS_variant);
    }
    if (FLAGS_sparse) {  // fused two-level priority, delta = 32 * avg weight / avg degree
        o.fused = 1;
        o.priority = SG_PRIORITY_LOW_HIGH;
        o.variant = SG_ASYNC_PUSH_DD;
        o.lb_push = SG_LB_NONE;
    }
    if (FLAGS_prio_delta > 0) {
        std::printf("Enable priority for scale-free dataset\n");
        o.priority = SG_PRIORITY_LOW_HIGH;
        o.priority_delta = FLAGS_prio_delta;
    }
    std::vector<uint32_t> dist(g.nv);
    std::vector<sg_round_trace> trace(FLAGS_trace ? std::max(1, FLAGS_max_iteration) : 0);
    sg_stats st{};
    st.trace = trace.empty() ? nullptr : trace.data();
    st.trace_capacity = (uint32_t)trace.size();
    JsonRecord js;
    SG_CHECK(sg_sssp(g.dev, src, &o, dist.data(), &st));
    PrintRun(st, o, g, false, js);
    bool ok = true;
    if (FLAGS_check) {
        const auto ref = HostSSSP(g, src);
        int errors = 0;
        for (uint32_t v = 0; v < g.nv; ++v) errors += dist[v] != ref[v];
        std::printf("total errors: %d\n", errors);
        ok = errors == 0;
    } else {
        std::printf("Warning: Result not checked\n");
    }
    if (!FLAGS_output.empty()) {
        FILE *f = std::fopen(FLAGS_output.c_str(), "w");
        for (uint32_t v = 0; f && v < g.nv; ++v)
            dist[v] == 0xffffffffu ? std::fprintf(f, "%u INF\n", v) : std::fprintf(f, "%u %u\n", v, dist[v]);
        if (f) std::fclose(f);
    }
    sg_graph_destroy(g.dev);
    return ok;
}

struct App {
    static const char *Name() { return "sssp"; }
    static const char *NameUpper() { return "SSSP"; }
    static bool Single() { return HybridSSSP(); }
};

int main(int argc, char **argv) { return Skeleton<App>()(argc, argv); }
