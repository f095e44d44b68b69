// Host CSR graph container and ingest helpers (internal to libsepgraph_b200).
#pragma once
#include <cstdint>
#include <vector>

#include "../../../include/sepgraph.h"

struct sg_hgraph {
    uint32_t nv = 0;
    uint64_t ne = 0;
    std::vector<uint32_t> offsets;  // nv + 1
    std::vector<uint32_t> indices;  // ne
    std::vector<uint32_t> weights;  // ne or empty
};

namespace sgb {
using HostGraph = sg_hgraph;

uint64_t splitmix64(uint64_t x);
unsigned host_threads();
sg_status gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed, uint32_t flags,
                   HostGraph &g);
sg_status gen_grid(uint32_t rows, uint32_t cols, uint32_t flags, HostGraph &g);
sg_status gen_random(uint32_t nv, uint32_t gen_factor, uint64_t seed, HostGraph &g);
sg_status gen_weights(HostGraph &g, uint32_t lo, uint32_t hi, uint64_t seed);
sg_status from_csr(uint32_t nv, uint64_t ne, const uint32_t *offsets, const uint32_t *indices, const uint32_t *weights,
                   HostGraph &g);
sg_status read_gr(const char *path, HostGraph &g);
sg_status write_gr(const HostGraph &g, const char *path);
sg_status read_market(const char *path, bool symmetrize, HostGraph &g);
sg_status read_metis(const char *path, HostGraph &g);
sg_status max_degree_vertex(const HostGraph &g, uint32_t *vertex, uint32_t *degree);
sg_status pick_sources(const HostGraph &g, uint32_t n, uint64_t seed, uint32_t *out);
}  // namespace sgb
