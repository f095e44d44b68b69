// Oracle support (test infrastructure, never linked into the product).
//
// C-ABI wrapper around the reference's own single-threaded host checkers,
// compiled from the reference sources where they lie by oracle/Makefile
// (target `ref`) into oracle/_ref/libsgref.so:
//   BFSHost                    samples/hybrid_bfs/hybrid_bfs_host.cpp:33-60
//   SSSPHostNaive              samples/hybrid_sssp/hybrid_sssp_host.cpp:34-60
//   PageRankHost               samples/hybrid_pr/hybrid_pr_host.cpp:43-124
//   PageRankCheckErrors        samples/hybrid_pr/hybrid_pr_host.cpp:126-161
//   BetweennessCentralityHost  samples/hybrid_bc/hybrid_bc_host.cpp:16-92
//   BCCheckErrors              samples/hybrid_bc/hybrid_bc_host.cpp:94-127
//   CSCGraph(csr, false)       include/groute/graphs/csr_graph.h:400-441 (csr_tocsc)
// The graph is bound (not copied) into the reference's host CSRGraph via
// CSRGraph::Bind (include/groute/graphs/csr_graph.h), exactly as the
// reference's traversal::Context does for a loaded .gr file.
#include <cstdint>
#include <cstring>
#include <vector>
#include <utility>
#include <gflags/gflags.h>
#include <groute/graphs/csr_graph.h>

// Flags the host checkers DECLARE but whose DEFINE lives in the reference's
// sample main.cpp / app_skeleton.h (not compiled here).
DEFINE_double(error, 0.01, "PR error tolerance");
DEFINE_bool(verbose, false, "Verbose prints");
DECLARE_bool(norm);

typedef uint32_t level_t;
typedef uint32_t distance_t;
typedef float rank_t;

std::vector<level_t> BFSHost(const groute::graphs::host::CSRGraph &graph, index_t source_node);
int BFSCheckErrors(const std::vector<level_t> &levels, const std::vector<level_t> &regression);
std::vector<distance_t> SSSPHostNaive(const groute::graphs::host::CSRGraph &graph,
                                      const distance_t *edge_weights, index_t source_node);
int SSSPCheckErrors(const std::vector<distance_t> &distances, const std::vector<distance_t> &regression);
std::vector<rank_t> PageRankHost(const groute::graphs::host::CSRGraph &graph);
int PageRankCheckErrors(std::vector<rank_t> &ranks, std::vector<rank_t> &regression);
std::pair<std::vector<float>, std::vector<float>>
BetweennessCentralityHost(const groute::graphs::host::CSRGraph &graph, index_t src);
int BCCheckErrors(std::vector<float> &regression_bc_values, std::vector<float> &bc_values);

namespace {
void bind(groute::graphs::host::CSRGraph &g, uint32_t nv, uint32_t ne, const uint32_t *offsets,
          const uint32_t *indices, const uint32_t *weights) {
    g.Bind(nv, ne, const_cast<index_t *>(offsets), const_cast<index_t *>(indices),
           const_cast<index_t *>(weights), nullptr);
}
}  // namespace

extern "C" {

int sgref_bfs(uint32_t nv, uint32_t ne, const uint32_t *offsets, const uint32_t *indices, uint32_t src,
              uint32_t *levels_out) {
    groute::graphs::host::CSRGraph g;
    bind(g, nv, ne, offsets, indices, nullptr);
    std::vector<level_t> lv = BFSHost(g, src);
    std::memcpy(levels_out, lv.data(), sizeof(level_t) * nv);
    return 0;
}

int sgref_bfs_check(uint32_t n, const uint32_t *levels, const uint32_t *regression) {
    std::vector<level_t> a(levels, levels + n), b(regression, regression + n);
    return BFSCheckErrors(a, b);
}

int sgref_sssp(uint32_t nv, uint32_t ne, const uint32_t *offsets, const uint32_t *indices,
               const uint32_t *weights, uint32_t src, uint32_t *dist_out) {
    groute::graphs::host::CSRGraph g;
    bind(g, nv, ne, offsets, indices, weights);
    std::vector<distance_t> d = SSSPHostNaive(g, weights, src);
    std::memcpy(dist_out, d.data(), sizeof(distance_t) * nv);
    return 0;
}

int sgref_sssp_check(uint32_t n, const uint32_t *dist, const uint32_t *regression) {
    std::vector<distance_t> a(dist, dist + n), b(regression, regression + n);
    return SSSPCheckErrors(a, b);
}

int sgref_pagerank(uint32_t nv, uint32_t ne, const uint32_t *offsets, const uint32_t *indices, double error,
                   float *ranks_out) {
    groute::graphs::host::CSRGraph g;
    bind(g, nv, ne, offsets, indices, nullptr);
    FLAGS_error = error;
    std::vector<rank_t> r = PageRankHost(g);
    std::memcpy(ranks_out, r.data(), sizeof(rank_t) * nv);
    return 0;
}

// Returns the number of vertices the reference's 5% checker flags.
int sgref_pagerank_check(uint32_t n, const float *ranks, const float *regression, int norm) {
    std::vector<rank_t> a(ranks, ranks + n), b(regression, regression + n);
    FLAGS_norm = norm != 0;
    int e = PageRankCheckErrors(a, b);
    FLAGS_norm = false;
    return e;
}

int sgref_bc(uint32_t nv, uint32_t ne, const uint32_t *offsets, const uint32_t *indices, uint32_t src,
             float *bc_out, float *sigma_out) {
    groute::graphs::host::CSRGraph g;
    bind(g, nv, ne, offsets, indices, nullptr);
    auto r = BetweennessCentralityHost(g, src);
    std::memcpy(bc_out, r.first.data(), sizeof(float) * nv);
    std::memcpy(sigma_out, r.second.data(), sizeof(float) * nv);
    return 0;
}

int sgref_bc_check(uint32_t n, const float *regression, const float *values) {
    std::vector<float> a(regression, regression + n), b(values, values + n);
    return BCCheckErrors(a, b);
}

int sgref_csr_tocsc(uint32_t nv, uint32_t ne, const uint32_t *offsets, const uint32_t *indices,
                    const uint32_t *weights, uint32_t *coff, uint32_t *cidx, uint32_t *cw) {
    groute::graphs::host::CSRGraph g;
    bind(g, nv, ne, offsets, indices, weights);
    groute::graphs::host::CSCGraph c(g, false);
    std::memcpy(coff, c.col_start, sizeof(uint32_t) * (nv + 1));
    std::memcpy(cidx, c.edge_source, sizeof(uint32_t) * ne);
    if (weights && cw) std::memcpy(cw, c.edge_weights, sizeof(uint32_t) * ne);
    return 0;
}

}  // extern "C"
