// gtools: the reference's graph converter (samples/tools/gtools.cpp) with the
// same flags and output files, its preprocessing (--deself_cycle,
// --deduplicate, --d2ud) run on the GPU by sg_graph_build.  The graph is read
// on the host (Galois .gr, MatrixMarket or METIS), its CSR handed to the
// device as an edge list in CSR order, and the processed CSR copied back for
// the text outputs: "src<splitter>out_degree" per vertex (--out_degree) and
// "src<splitter>dst[<splitter>weight]" per edge (--output).
#include <cstdio>
#include <string>
#include <vector>

#include "../../../include/sepgraph.h"
#include "sg_flags.h"

DEFINE_string(graphfile, "", "A file with a graph in Dimacs 10 format");
DEFINE_bool(ggr, true, "Graph file is a Galois binary GR file");
DEFINE_string(output, "", "edge list output");
DEFINE_string(out_degree, "", "Save out degree to file");
DEFINE_string(splitter, "\t", "the splitter between nodes pair");
DEFINE_bool(deself_cycle, false, "remove self-cycle, e.g. 0-0, 1-1 ...");
DEFINE_bool(deduplicate, true, "remove duplicated edges");
DEFINE_string(format, "gr", "graph format (gr/market/metis formats are supported)");
DEFINE_bool(d2ud, false, "convert directed graph to undirected graph");
DEFINE_int32(device, 0, "CUDA device");

static int fail(const char *what, sg_status st, sg_ctx *ctx) {
    std::fprintf(stderr, "%s: %s %s\n", what, sg_status_string(st), ctx ? sg_last_error(ctx) : "");
    return 1;
}

int main(int argc, char **argv) {
    if (!sgflags::ParseCommandLineFlags(&argc, &argv, true)) return 1;
    if (FLAGS_graphfile.empty()) {
        std::printf("A Graph File must be provided\n");
        return 0;
    }
    std::printf("\nLoading graph %s\n", FLAGS_graphfile.c_str());
    sg_hgraph *h = nullptr;
    sg_status st;
    if (FLAGS_format == "gr") st = sg_hgraph_read_gr(FLAGS_graphfile.c_str(), &h);
    else if (FLAGS_format == "market") st = sg_hgraph_read_market(FLAGS_graphfile.c_str(), 0, &h);
    else if (FLAGS_format == "metis") st = sg_hgraph_read_metis(FLAGS_graphfile.c_str(), &h);
    else {
        std::fprintf(stderr, "unsupported graph format\n");
        return 1;
    }
    if (st != SG_OK) return fail("read graph", st, nullptr);
    uint32_t nv = 0;
    uint64_t ne = 0;
    const uint32_t *off = nullptr, *idx = nullptr, *w = nullptr;
    sg_hgraph_info(h, &nv, &ne, &off, &idx, &w);
    if (nv == 0) std::printf("Empty graph!\n");
    std::printf(w ? "Weighted graph\n" : "Unweighted graph\n");

    std::vector<uint32_t> src(ne);
    for (uint32_t v = 0; v < nv; ++v)
        for (uint32_t e = off[v]; e < off[v + 1]; ++e) src[e] = v;
    sg_ctx *ctx = nullptr;
    if ((st = sg_init(FLAGS_device, &ctx)) != SG_OK) return fail("sg_init", st, nullptr);
    const uint32_t flags = (FLAGS_deself_cycle ? SG_BUILD_DESELF_CYCLE : 0u) |
                           (FLAGS_deduplicate ? SG_BUILD_DEDUPLICATE : 0u) | (FLAGS_d2ud ? SG_BUILD_D2UD : 0u);
    sg_graph *g = nullptr;
    st = sg_graph_build(ctx, nv ? nv : 1, ne, src.data(), idx, w, flags, SG_GRAPH_NO_CSC, &g);
    if (st != SG_OK) return fail("sg_graph_build", st, ctx);
    uint64_t ne2 = 0;
    sg_graph_info(g, nullptr, &ne2, nullptr, nullptr);
    std::vector<uint32_t> row((size_t)(nv ? nv : 1) + 1), col(ne2), wt(w ? ne2 : 0);
    if ((st = sg_graph_copy_out(g, 0, row.data(), col.data(), w ? wt.data() : nullptr)) != SG_OK)
        return fail("sg_graph_copy_out", st, ctx);
    if (FLAGS_deself_cycle) std::printf("Self-cycle removed\n");
    if (FLAGS_deduplicate) std::printf("Duplicated edges removed\n");
    if (FLAGS_d2ud) std::printf("Converted to undirected graph\n");
    std::printf("nodes: %u edges: %llu\n", nv, (unsigned long long)ne2);
    const char *sp = FLAGS_splitter.c_str();
    if (!FLAGS_out_degree.empty()) {
        FILE *f = std::fopen(FLAGS_out_degree.c_str(), "w");
        if (!f) {
            std::fprintf(stderr, "can not open file %s", FLAGS_out_degree.c_str());
            return 1;
        }
        for (uint32_t v = 0; v < nv; ++v) std::fprintf(f, "%u%s%u\n", v, sp, row[v + 1] - row[v]);
        std::fclose(f);
        std::printf("Out-degree written!\n");
    }
    if (!FLAGS_output.empty()) {
        FILE *f = std::fopen(FLAGS_output.c_str(), "w");
        if (!f) {
            std::fprintf(stderr, "can not open file %s", FLAGS_output.c_str());
            return 1;
        }
        std::printf("Writing to edgelist...\n");
        for (uint32_t v = 0; v < nv; ++v)
            for (uint32_t e = row[v]; e < row[v + 1]; ++e) {
                if (w) std::fprintf(f, "%u%s%u%s%u\n", v, sp, col[e], sp, wt[e]);
                else std::fprintf(f, "%u%s%u\n", v, sp, col[e]);
            }
        std::fclose(f);
        std::printf("Edgelist written!\n");
    }
    sg_graph_destroy(g);
    sg_destroy(ctx);
    sg_hgraph_destroy(h);
    return 0;
}
