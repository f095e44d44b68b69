// Host-side graph ingest for the B200 engine: seeded generators, CSR build,
// and on-disk formats.  Everything here is cold-path host code (the GPU path
// starts at sg_graph_create); it is multi-threaded with std::thread because
// RMAT scale 22-23 produces 67-268 M edges.
//
// Reference counterparts:
//  - graph generation: include/utils/graphs/traversal.h:102-134 (random/chain/
//    clique generators, unseeded std::default_random_engine at 173-189).  The
//    reference has no RMAT generator; this one is seeded and counter-based so
//    the same (scale, seed) gives the same graph on any thread count.
//  - symmetrise / drop self-loops / deduplicate: samples/tools/gtools.cpp:56-328
//    (the converter the reference uses to prepare undirected inputs).
//  - Galois .gr binary format: src/utils/parser.cpp:409-506 (ReadGraphGR).
//  - MatrixMarket: src/utils/parser.cpp:508-665 (ReadGraphMarket).  Same
//    semantics (1-based ids, per-source sorted set dedup, integer weights),
//    except that nedges is the deduplicated count (the reference keeps the
//    pre-dedup header count).
#include "sg_hgraph.h"

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <set>
#include <string>
#include <thread>
#include <vector>

namespace sgb {

uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

unsigned host_threads() {
    unsigned n = std::thread::hardware_concurrency();
    if (n == 0) n = 1;
    if (n > 64) n = 64;
    return n;
}

// Runs f(begin, end) over [0, n) split in contiguous chunks across threads.
template <typename F>
static void parallel_for(uint64_t n, F f) {
    unsigned nt = host_threads();
    if (n < (1u << 16) || nt == 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> ts;
    uint64_t chunk = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; ++t) {
        uint64_t b = t * chunk, e = std::min<uint64_t>(n, b + chunk);
        if (b >= e) break;
        ts.emplace_back([=] { f(b, e); });
    }
    for (auto &t : ts) t.join();
}

// Dynamic scheduling over [0, n) in blocks of `grain` (for skewed per-row work).
template <typename F>
static void parallel_for_dynamic(uint64_t n, uint64_t grain, F f) {
    unsigned nt = host_threads();
    if (n <= grain || nt == 1) {
        f(0, n);
        return;
    }
    std::atomic<uint64_t> next(0);
    std::vector<std::thread> ts;
    for (unsigned t = 0; t < nt; ++t) {
        ts.emplace_back([&] {
            for (;;) {
                uint64_t b = next.fetch_add(grain);
                if (b >= n) break;
                f(b, std::min<uint64_t>(n, b + grain));
            }
        });
    }
    for (auto &t : ts) t.join();
}

// Builds a CSR from an edge list: counting sort by source, then per-row sort
// and (optionally) unique.  Rows come out sorted by destination, which makes
// the result independent of thread count and insertion order.
static sg_status build_csr(uint32_t nv, const std::vector<uint32_t> &src, const std::vector<uint32_t> &dst,
                           bool keep_self_loops, bool keep_dups, HostGraph &g) {
    const uint64_t m = src.size();
    std::vector<std::atomic<uint32_t>> deg(nv);
    for (uint32_t v = 0; v < nv; ++v) deg[v].store(0, std::memory_order_relaxed);
    parallel_for(m, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; ++i) {
            if (!keep_self_loops && src[i] == dst[i]) continue;
            deg[src[i]].fetch_add(1, std::memory_order_relaxed);
        }
    });
    std::vector<uint64_t> off(nv + 1, 0);
    for (uint32_t v = 0; v < nv; ++v) off[v + 1] = off[v] + deg[v].load(std::memory_order_relaxed);
    const uint64_t total = off[nv];
    std::vector<uint32_t> col;
    try {
        col.resize(total);
    } catch (...) {
        return SG_ERR_OUT_OF_MEMORY;
    }
    std::vector<std::atomic<uint64_t>> cur(nv);
    for (uint32_t v = 0; v < nv; ++v) cur[v].store(off[v], std::memory_order_relaxed);
    parallel_for(m, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; ++i) {
            if (!keep_self_loops && src[i] == dst[i]) continue;
            uint64_t p = cur[src[i]].fetch_add(1, std::memory_order_relaxed);
            col[p] = dst[i];
        }
    });
    // sort + unique each row; record new degree
    std::vector<uint32_t> ndeg(nv, 0);
    parallel_for_dynamic(nv, 4096, [&](uint64_t b, uint64_t e) {
        for (uint64_t v = b; v < e; ++v) {
            auto first = col.begin() + off[v], last = col.begin() + off[v + 1];
            std::sort(first, last);
            if (!keep_dups) last = std::unique(first, last);
            ndeg[v] = (uint32_t)(last - first);
        }
    });
    std::vector<uint64_t> noff(nv + 1, 0);
    for (uint32_t v = 0; v < nv; ++v) noff[v + 1] = noff[v] + ndeg[v];
    if (noff[nv] >= (1ull << 32)) return SG_ERR_INVALID_ARG;  // index_t edges must fit uint32
    g.nv = nv;
    g.ne = noff[nv];
    g.offsets.assign(nv + 1, 0);
    g.indices.resize(g.ne);
    for (uint32_t v = 0; v <= nv; ++v) g.offsets[v] = (uint32_t)noff[v];
    parallel_for(nv, [&](uint64_t b, uint64_t e) {
        for (uint64_t v = b; v < e; ++v)
            std::copy(col.begin() + off[v], col.begin() + off[v] + ndeg[v], g.indices.begin() + noff[v]);
    });
    g.weights.clear();
    return SG_OK;
}

sg_status gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed, uint32_t flags,
                   HostGraph &g) {
    if (scale == 0 || scale > 30 || edge_factor == 0) return SG_ERR_INVALID_ARG;
    if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return SG_ERR_INVALID_ARG;
    const uint32_t nv = 1u << scale;
    const uint64_t m = (uint64_t)edge_factor << scale;
    const bool sym = flags & SG_GEN_SYMMETRIC;
    const uint64_t total = sym ? 2 * m : m;
    std::vector<uint32_t> src, dst;
    try {
        src.resize(total);
        dst.resize(total);
    } catch (...) {
        return SG_ERR_OUT_OF_MEMORY;
    }
    const double ab = a + b, abc = a + b + c;
    const uint64_t stream = splitmix64(seed ^ 0x5245A7ULL);
    parallel_for(m, [&](uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; ++i) {
            uint64_t st = splitmix64(stream + i * 0xD1B54A32D192ED03ULL);
            uint32_t u = 0, v = 0;
            for (uint32_t l = 0; l < scale; ++l) {
                st = splitmix64(st);
                const double r = (double)(st >> 11) * (1.0 / 9007199254740992.0);
                uint32_t bu = 0, bv = 0;
                if (r < a) {
                } else if (r < ab) {
                    bv = 1;
                } else if (r < abc) {
                    bu = 1;
                } else {
                    bu = 1;
                    bv = 1;
                }
                u = (u << 1) | bu;
                v = (v << 1) | bv;
            }
            src[i] = u;
            dst[i] = v;
            if (sym) {
                src[m + i] = v;
                dst[m + i] = u;
            }
        }
    });
    return build_csr(nv, src, dst, flags & SG_GEN_KEEP_SELF_LOOPS, flags & SG_GEN_KEEP_DUPLICATES, g);
}

sg_status gen_grid(uint32_t rows, uint32_t cols, uint32_t flags, HostGraph &g) {
    (void)flags;
    if (rows == 0 || cols == 0) return SG_ERR_INVALID_ARG;
    const uint64_t nv64 = (uint64_t)rows * cols;
    if (nv64 >= (1ull << 32)) return SG_ERR_INVALID_ARG;
    const uint32_t nv = (uint32_t)nv64;
    g.nv = nv;
    g.offsets.assign(nv + 1, 0);
    // 4-neighbour, both directions; neighbours listed in increasing id order
    // (up, left, right, down), so rows are sorted like every other CSR here.
    for (uint32_t v = 0; v < nv; ++v) {
        uint32_t r = v / cols, cc = v % cols;
        uint32_t d = (r > 0) + (cc > 0) + (cc + 1 < cols) + (r + 1 < rows);
        g.offsets[v + 1] = g.offsets[v] + d;
    }
    g.ne = g.offsets[nv];
    g.indices.resize(g.ne);
    parallel_for(nv, [&](uint64_t b, uint64_t e) {
        for (uint64_t v = b; v < e; ++v) {
            uint32_t r = (uint32_t)(v / cols), cc = (uint32_t)(v % cols);
            uint32_t p = g.offsets[v];
            if (r > 0) g.indices[p++] = (uint32_t)(v - cols);
            if (cc > 0) g.indices[p++] = (uint32_t)(v - 1);
            if (cc + 1 < cols) g.indices[p++] = (uint32_t)(v + 1);
            if (r + 1 < rows) g.indices[p++] = (uint32_t)(v + cols);
        }
    });
    g.weights.clear();
    return SG_OK;
}

sg_status gen_random(uint32_t nv, uint32_t gen_factor, uint64_t seed, HostGraph &g) {
    if (nv < 2 || gen_factor < 1 || gen_factor >= nv) return SG_ERR_INVALID_ARG;
    g.nv = nv;
    g.offsets.assign(nv + 1, 0);
    std::vector<uint32_t> deg(nv);
    const uint64_t stream = splitmix64(seed ^ 0x6E6E6E6EULL);
    for (uint32_t v = 0; v < nv; ++v) deg[v] = 1 + (uint32_t)(splitmix64(stream + 2ull * v) % gen_factor);
    for (uint32_t v = 0; v < nv; ++v) g.offsets[v + 1] = g.offsets[v] + deg[v];
    g.ne = g.offsets[nv];
    g.indices.resize(g.ne);
    parallel_for(nv, [&](uint64_t b, uint64_t e) {
        for (uint64_t v = b; v < e; ++v) {
            uint64_t st = splitmix64(stream + 2ull * v + 1);
            uint32_t *row = g.indices.data() + g.offsets[v];
            uint32_t n = 0;
            while (n < deg[v]) {
                st = splitmix64(st);
                const uint32_t u = (uint32_t)(st % nv);
                if (u == v || std::find(row, row + n, u) != row + n) continue;
                row[n++] = u;
            }
            std::sort(row, row + n);
        }
    });
    g.weights.clear();
    return SG_OK;
}

sg_status gen_weights(HostGraph &g, uint32_t lo, uint32_t hi, uint64_t seed) {
    if (hi <= lo) return SG_ERR_INVALID_ARG;
    const uint64_t span = hi - lo;
    g.weights.resize(g.ne);
    const uint64_t stream = splitmix64(seed ^ 0x57E16ULL);
    parallel_for(g.ne, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; ++i) g.weights[i] = lo + (uint32_t)(splitmix64(stream + i) % span);
    });
    return SG_OK;
}

sg_status from_csr(uint32_t nv, uint64_t ne, const uint32_t *offsets, const uint32_t *indices, const uint32_t *weights,
                   HostGraph &g) {
    if (!offsets || (ne && !indices)) return SG_ERR_INVALID_ARG;
    if (ne >= (1ull << 32) || offsets[0] != 0 || offsets[nv] != ne) return SG_ERR_INVALID_ARG;
    for (uint32_t v = 0; v < nv; ++v)
        if (offsets[v + 1] < offsets[v]) return SG_ERR_INVALID_ARG;
    for (uint64_t e = 0; e < ne; ++e)
        if (indices[e] >= nv) return SG_ERR_INVALID_ARG;
    g.nv = nv;
    g.ne = ne;
    g.offsets.assign(offsets, offsets + nv + 1);
    g.indices.assign(indices, indices + ne);
    if (weights)
        g.weights.assign(weights, weights + ne);
    else
        g.weights.clear();
    return SG_OK;
}

// Galois .gr (version 1): u64 header {version=1, edge-data size, nnodes, nedges},
// nnodes u64 row END offsets, nedges u32 destinations, 4 bytes of padding when
// nedges is odd and edge data follows, then nedges u32 edge data.
sg_status read_gr(const char *path, HostGraph &g) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return SG_ERR_IO;
    uint64_t h[4];
    sg_status st = SG_OK;
    if (std::fread(h, sizeof(uint64_t), 4, f) != 4) {
        st = SG_ERR_FORMAT;
    } else if (h[0] != 1 || h[2] >= (1ull << 32) || h[3] >= (1ull << 32) || (h[1] != 0 && h[1] != 4)) {
        st = SG_ERR_FORMAT;
    } else {
        const uint32_t nv = (uint32_t)h[2];
        const uint64_t ne = h[3];
        std::vector<uint64_t> ends(nv);
        g.nv = nv;
        g.ne = ne;
        g.offsets.assign(nv + 1, 0);
        g.indices.resize(ne);
        if (nv && std::fread(ends.data(), sizeof(uint64_t), nv, f) != nv) st = SG_ERR_FORMAT;
        for (uint32_t v = 0; st == SG_OK && v < nv; ++v) {
            if (ends[v] > ne || (v && ends[v] < ends[v - 1])) st = SG_ERR_FORMAT;
            g.offsets[v + 1] = (uint32_t)ends[v];
        }
        if (st == SG_OK && nv && g.offsets[nv] != ne) st = SG_ERR_FORMAT;
        if (st == SG_OK && ne && std::fread(g.indices.data(), sizeof(uint32_t), ne, f) != ne) st = SG_ERR_FORMAT;
        for (uint64_t e = 0; st == SG_OK && e < ne; ++e)
            if (g.indices[e] >= nv) st = SG_ERR_FORMAT;
        if (st == SG_OK && h[1] == 4) {
            if (ne % 2) std::fseek(f, 4, SEEK_CUR);
            g.weights.resize(ne);
            if (ne && std::fread(g.weights.data(), sizeof(uint32_t), ne, f) != ne) st = SG_ERR_FORMAT;
        } else {
            g.weights.clear();
        }
    }
    std::fclose(f);
    return st;
}

sg_status write_gr(const HostGraph &g, const char *path) {
    FILE *f = std::fopen(path, "wb");
    if (!f) return SG_ERR_IO;
    const bool w = !g.weights.empty();
    uint64_t h[4] = {1, w ? 4ull : 0ull, g.nv, g.ne};
    bool ok = std::fwrite(h, sizeof(uint64_t), 4, f) == 4;
    for (uint32_t v = 0; ok && v < g.nv; ++v) {
        uint64_t e = g.offsets[v + 1];
        ok = std::fwrite(&e, sizeof(uint64_t), 1, f) == 1;
    }
    if (ok && g.ne) ok = std::fwrite(g.indices.data(), sizeof(uint32_t), g.ne, f) == g.ne;
    if (ok && w) {
        if (g.ne % 2) {
            uint32_t pad = 0;
            ok = std::fwrite(&pad, sizeof(uint32_t), 1, f) == 1;
        }
        if (ok && g.ne) ok = std::fwrite(g.weights.data(), sizeof(uint32_t), g.ne, f) == g.ne;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? SG_OK : SG_ERR_IO;
}

// METIS graph file (ReadGraph, src/utils/parser.cpp:230-396): '%' comment
// lines are skipped; the header is "n m [fmt [ncon]]" with m counting every
// undirected edge once; fmt's digits select vertex sizes, vertex weights
// (ncon per vertex, ncon > 0 only with vertex weights) and edge weights;
// vertex i's line lists 1-based neighbours, each followed by its positive
// weight when edge weights are present, in file order (no sorting or
// deduplication); exactly 2m entries must be listed.  Vertex sizes and
// weights are read and dropped (the engine has no use for them).  The
// reference scans the header with a 64-bit conversion into 32-bit fields
// (parser.h SCIDX); the header is read here as the format defines it.
sg_status read_metis(const char *path, HostGraph &g) {
    FILE *f = std::fopen(path, "r");
    if (!f) return SG_ERR_IO;
    std::string line;
    auto next_line = [&]() -> bool {
        do {
            line.clear();
            int c;
            bool any = false;
            while ((c = std::fgetc(f)) != EOF) {
                any = true;
                if (c == '\n') break;
                line.push_back((char)c);
            }
            if (!any) return false;
        } while (!line.empty() && line[0] == '%');
        return true;
    };
    auto fail = [&](sg_status st) {
        std::fclose(f);
        return st;
    };
    unsigned long long n = 0, m = 0, fmt = 0, ncon = 0;
    if (!next_line()) return fail(SG_ERR_FORMAT);
    const int fields = std::sscanf(line.c_str(), "%llu %llu %llu %llu", &n, &m, &fmt, &ncon);
    if (fields < 2 || n == 0 || m == 0 || n >= (1ull << 32) || 2 * m >= (1ull << 32) || fmt > 111)
        return fail(SG_ERR_FORMAT);
    const bool readvs = (fmt / 100) % 10 == 1, readvw = (fmt / 10) % 10 == 1, readew = fmt % 10 == 1;
    if (ncon > 0 && !readvw) return fail(SG_ERR_FORMAT);
    if (ncon == 0) ncon = 1;
    const uint64_t ne = 2 * m;
    g.nv = (uint32_t)n;
    g.offsets.assign(n + 1, 0);
    g.indices.clear();
    g.weights.clear();
    try {
        g.indices.reserve(ne);
        if (readew) g.weights.reserve(ne);
    } catch (...) {
        return fail(SG_ERR_OUT_OF_MEMORY);
    }
    for (uint64_t i = 0; i < n; ++i) {
        if (!next_line()) return fail(SG_ERR_FORMAT);
        const char *cur = line.c_str();
        char *end = nullptr;
        if (readvs) {
            const long long vs = std::strtoll(cur, &end, 10);
            if (end == cur || vs < 0) return fail(SG_ERR_FORMAT);
            cur = end;
        }
        if (readvw) {
            for (uint64_t l = 0; l < ncon; ++l) {
                const long long vw = std::strtoll(cur, &end, 10);
                if (end == cur || vw < 0) return fail(SG_ERR_FORMAT);
                cur = end;
            }
        }
        for (;;) {
            const long long e = std::strtoll(cur, &end, 10);
            if (end == cur) break;
            cur = end;
            if (e < 1 || (unsigned long long)e > n) return fail(SG_ERR_FORMAT);
            long long w = 1;
            if (readew) {
                w = std::strtoll(cur, &end, 10);
                if (end == cur || w <= 0 || w >= (1ll << 32)) return fail(SG_ERR_FORMAT);
                cur = end;
            }
            if (g.indices.size() == ne) return fail(SG_ERR_FORMAT);  // more entries than 2m
            g.indices.push_back((uint32_t)(e - 1));
            if (readew) g.weights.push_back((uint32_t)w);
        }
        g.offsets[i + 1] = (uint32_t)g.indices.size();
    }
    std::fclose(f);
    if (g.indices.size() != ne) return SG_ERR_FORMAT;
    g.ne = ne;
    return SG_OK;
}

sg_status read_market(const char *path, bool symmetrize, HostGraph &g) {
    FILE *f = std::fopen(path, "r");
    if (!f) return SG_ERR_IO;
    std::vector<char> line(1 << 16);
    auto next_line = [&]() -> bool {
        do {
            if (!std::fgets(line.data(), (int)line.size(), f)) return false;
        } while (line[0] == '%');
        return true;
    };
    unsigned long long rows = 0, cols = 0, nnz = 0;
    if (!next_line() || std::sscanf(line.data(), "%llu %llu %llu", &rows, &cols, &nnz) != 3 || rows >= (1ull << 32)) {
        std::fclose(f);
        return SG_ERR_FORMAT;
    }
    const uint32_t nv = (uint32_t)std::max(rows, cols);
    int weighted = -1;  // decided on the first entry, like parser.cpp:560-588
    std::vector<std::pair<uint32_t, uint32_t>> el;
    std::vector<uint32_t> wl;
    for (unsigned long long i = 0; i < nnz; ++i) {
        if (!next_line()) {
            std::fclose(f);
            return SG_ERR_FORMAT;
        }
        char *p = line.data(), *end = nullptr;
        long long s = std::strtoll(p, &end, 10) - 1;
        long long d = std::strtoll(end, &end, 10) - 1;
        if (s < 0 || d < 0 || (unsigned long long)s >= nv || (unsigned long long)d >= nv) {
            std::fclose(f);
            return SG_ERR_FORMAT;
        }
        if (weighted < 0) {
            weighted = 0;
            for (char *q = end; *q; ++q) {
                if (*q == '.') {
                    std::fclose(f);
                    return SG_ERR_FORMAT;  // float weights unsupported, as in the reference
                }
                if (*q >= '0' && *q <= '9') weighted = 1;
            }
        }
        uint32_t w = weighted ? (uint32_t)std::strtoul(end, &end, 10) : 0;
        el.emplace_back((uint32_t)s, (uint32_t)d);
        if (weighted) wl.push_back(w);
        if (symmetrize && s != d) {
            el.emplace_back((uint32_t)d, (uint32_t)s);
            if (weighted) wl.push_back(w);
        }
    }
    std::fclose(f);
    // per-source ordered set of dst (or (dst, w)) -> sorted, deduplicated rows
    std::vector<uint64_t> order(el.size());
    for (uint64_t i = 0; i < order.size(); ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](uint64_t x, uint64_t y) {
        if (el[x] != el[y]) return el[x] < el[y];
        return weighted ? wl[x] < wl[y] : x < y;
    });
    g.nv = nv;
    g.offsets.assign(nv + 1, 0);
    g.indices.clear();
    g.weights.clear();
    for (uint64_t k = 0; k < order.size(); ++k) {
        uint64_t i = order[k];
        if (k) {
            uint64_t j = order[k - 1];
            bool same = el[i] == el[j] && (!weighted || wl[i] == wl[j]);
            if (same) continue;
        }
        g.indices.push_back(el[i].second);
        if (weighted) g.weights.push_back(wl[i]);
        g.offsets[el[i].first + 1]++;
    }
    for (uint32_t v = 0; v < nv; ++v) g.offsets[v + 1] += g.offsets[v];
    g.ne = g.indices.size();
    return SG_OK;
}

sg_status max_degree_vertex(const HostGraph &g, uint32_t *vertex, uint32_t *degree) {
    uint32_t best = 0, bd = 0;
    for (uint32_t v = 0; v < g.nv; ++v) {
        uint32_t d = g.offsets[v + 1] - g.offsets[v];
        if (d > bd) {
            bd = d;
            best = v;
        }
    }
    if (vertex) *vertex = best;
    if (degree) *degree = bd;
    return SG_OK;
}

sg_status pick_sources(const HostGraph &g, uint32_t n, uint64_t seed, uint32_t *out) {
    if (!out || g.nv == 0) return SG_ERR_INVALID_ARG;
    const uint64_t stream = splitmix64(seed ^ 0x5EEDULL);
    uint32_t got = 0;
    for (uint64_t k = 0; got < n; ++k) {
        if (k > 64ull * g.nv + 1024) return SG_ERR_INVALID_ARG;  // not enough vertices with out-degree > 0
        uint32_t v = (uint32_t)(splitmix64(stream + k) % g.nv);
        if (g.offsets[v + 1] == g.offsets[v]) continue;
        bool dup = false;
        for (uint32_t i = 0; i < got; ++i) dup |= out[i] == v;
        if (dup && n <= g.nv) continue;
        out[got++] = v;
    }
    return SG_OK;
}

}  // namespace sgb
