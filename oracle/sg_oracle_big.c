/*
 * ORACLE — test infrastructure only.  Never linked into or called by the
 * product library; only tests/, __graft_entry__.smoke() and bench.py's
 * parity checks, cpu_baseline and reference arm load it.
 *
 * Inputs and checkers for the full-size workloads, where the one-thread
 * restatements in sg_oracle.c take too long or the product's own generators
 * must not be used (the reference arm of the benchmark runs without the
 * product library):
 *
 *   sgo_rmat_edges / sgo_build_csr
 *       the seeded RMAT generator and CSR construction the benchmark's graphs
 *       come from (counter-based splitmix64 stream per edge, recursive
 *       quadrant choice with probabilities a/b/c/d per level; rows sorted by
 *       destination, self-loops and duplicates dropped unless kept).  A CPU
 *       test proves the CSR equal, word for word, to the product library's
 *       generator, so both arms of the benchmark run on one graph.
 *   sgo_gen_weights, sgo_pick_sources
 *       the seeded weight and source streams of the same generator.
 *   sgo_dijkstra
 *       single-source shortest paths with a binary heap: with uint32 weights
 *       the distances are unique, so it returns exactly what SSSPHostNaive
 *       (samples/hybrid_sssp/hybrid_sssp_host.cpp:34-60) returns, in
 *       O(E log V) instead of the label-correcting FIFO's worst case (minutes
 *       on a 4096x4096 grid).  Pinned to sgo_sssp by a CPU test.
 *   sgo_pagerank_jacobi_f64
 *       the fixed point PageRankHost (samples/hybrid_pr/hybrid_pr_host.cpp:
 *       43-124) converges to, rank(v) = (1 - 0.85) + 0.85 * sum over in-edges
 *       u->v of rank(u) / outdeg(u) (vertices without out-edges keep their
 *       rank), solved in double by Jacobi sweeps over the in-edges on all host
 *       threads until the L1 change falls below tol * L1 norm.  Pinned to
 *       sgo_pagerank_f64 by a CPU test.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define SGO_INF 0xffffffffu
#define SGO_ALPHA 0.85 /* hybrid_pr_common.h:39 */

static uint64_t sgo_splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

/* Raw RMAT edges: m = edge_factor << scale of them, followed (sym) by their
 * reverses.  src/dst hold m (or 2m) entries. */
int sgo_rmat_edges(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed, int sym,
                   uint32_t *src, uint32_t *dst) {
    if (scale == 0 || scale > 30 || edge_factor == 0) return -1;
    const uint64_t m = (uint64_t)edge_factor << scale;
    const double ab = a + b, abc = a + b + c;
    const uint64_t stream = sgo_splitmix64(seed ^ 0x5245A7ULL);
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)m; ++ii) {
        const uint64_t i = (uint64_t)ii;
        uint64_t st = sgo_splitmix64(stream + i * 0xD1B54A32D192ED03ULL);
        uint32_t u = 0, v = 0;
        for (uint32_t l = 0; l < scale; ++l) {
            st = sgo_splitmix64(st);
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
    return 0;
}

static int cmp_u32(const void *x, const void *y) {
    const uint32_t a = *(const uint32_t *)x, b = *(const uint32_t *)y;
    return (a > b) - (a < b);
}

/* Edge list -> CSR with rows sorted by destination; self-loops and duplicate
 * (src, dst) pairs dropped unless kept.  idx must hold m entries; *ne gets the
 * edge count.  Returns -2 when the edge count does not fit 32-bit offsets. */
int sgo_build_csr(uint32_t nv, uint64_t m, const uint32_t *src, const uint32_t *dst, int keep_self_loops,
                  int keep_dups, uint32_t *off_out, uint32_t *idx, uint64_t *ne) {
    uint64_t *off = (uint64_t *)calloc((size_t)nv + 1, sizeof(uint64_t));
    uint64_t *cur = (uint64_t *)malloc(((size_t)nv + 1) * sizeof(uint64_t));
    uint32_t *ndeg = (uint32_t *)calloc((size_t)nv + 1, sizeof(uint32_t));
    if (!off || !cur || !ndeg) return -1;
    for (uint64_t i = 0; i < m; ++i)
        if (keep_self_loops || src[i] != dst[i]) off[src[i] + 1]++;
    for (uint32_t v = 0; v < nv; ++v) off[v + 1] += off[v];
    memcpy(cur, off, ((size_t)nv + 1) * sizeof(uint64_t));
    for (uint64_t i = 0; i < m; ++i)
        if (keep_self_loops || src[i] != dst[i]) idx[cur[src[i]]++] = dst[i];
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t vv = 0; vv < (int64_t)nv; ++vv) {
        uint32_t *row = idx + off[vv];
        const uint64_t n = off[vv + 1] - off[vv];
        qsort(row, (size_t)n, sizeof(uint32_t), cmp_u32);
        uint64_t k = n;
        if (!keep_dups && n > 1) {
            k = 1;
            for (uint64_t j = 1; j < n; ++j)
                if (row[j] != row[k - 1]) row[k++] = row[j];
        }
        ndeg[vv] = (uint32_t)k;
    }
    /* compact the rows in place (each row moves left or stays) */
    uint64_t w = 0;
    off_out[0] = 0;
    for (uint32_t v = 0; v < nv; ++v) {
        if (w != off[v]) memmove(idx + w, idx + off[v], (size_t)ndeg[v] * sizeof(uint32_t));
        w += ndeg[v];
        if (w >= (1ull << 32)) {
            free(off);
            free(cur);
            free(ndeg);
            return -2;
        }
        off_out[v + 1] = (uint32_t)w;
    }
    *ne = w;
    free(off);
    free(cur);
    free(ndeg);
    return 0;
}

/* Weights in [lo, hi) from the stream (seed, edge index). */
int sgo_gen_weights(uint64_t ne, uint32_t lo, uint32_t hi, uint64_t seed, uint32_t *w) {
    if (hi <= lo) return -1;
    const uint64_t span = hi - lo;
    const uint64_t stream = sgo_splitmix64(seed ^ 0x57E16ULL);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)ne; ++i) w[i] = lo + (uint32_t)(sgo_splitmix64(stream + (uint64_t)i) % span);
    return 0;
}

/* n distinct (while n <= nv) seeded vertices with out-degree > 0. */
int sgo_pick_sources(uint32_t nv, const uint32_t *off, uint32_t n, uint64_t seed, uint32_t *out) {
    if (nv == 0) return -1;
    const uint64_t stream = sgo_splitmix64(seed ^ 0x5EEDULL);
    uint32_t got = 0;
    for (uint64_t k = 0; got < n; ++k) {
        if (k > 64ull * nv + 1024) return -1;
        const uint32_t v = (uint32_t)(sgo_splitmix64(stream + k) % nv);
        if (off[v + 1] == off[v]) continue;
        int dup = 0;
        for (uint32_t i = 0; i < got; ++i) dup |= out[i] == v;
        if (dup && n <= nv) continue;
        out[got++] = v;
    }
    return 0;
}

/* ---------------------------------------------------------------- Dijkstra
 * Lazy binary min-heap of (distance << 32 | vertex) keys. */
typedef struct {
    uint64_t *a;
    size_t n, cap;
} heap_t;

static int heap_push(heap_t *h, uint64_t key) {
    if (h->n == h->cap) {
        size_t nc = h->cap ? 2 * h->cap : 1024;
        uint64_t *na = (uint64_t *)realloc(h->a, nc * sizeof(uint64_t));
        if (!na) return 0;
        h->a = na;
        h->cap = nc;
    }
    size_t i = h->n++;
    while (i > 0) {
        size_t p = (i - 1) / 2;
        if (h->a[p] <= key) break;
        h->a[i] = h->a[p];
        i = p;
    }
    h->a[i] = key;
    return 1;
}

static uint64_t heap_pop(heap_t *h) {
    uint64_t top = h->a[0], last = h->a[--h->n];
    size_t i = 0;
    for (;;) {
        size_t l = 2 * i + 1;
        if (l >= h->n) break;
        size_t r = l + 1, s = (r < h->n && h->a[r] < h->a[l]) ? r : l;
        if (h->a[s] >= last) break;
        h->a[i] = h->a[s];
        i = s;
    }
    if (h->n) h->a[i] = last;
    return top;
}

int sgo_dijkstra(uint32_t nv, const uint32_t *off, const uint32_t *idx, const uint32_t *w, uint32_t src,
                 uint32_t *dist) {
    if (src >= nv) return -1;
    heap_t h = {NULL, 0, 0};
    for (uint32_t v = 0; v < nv; ++v) dist[v] = SGO_INF;
    dist[src] = 0;
    if (!heap_push(&h, (uint64_t)src)) return -2;
    while (h.n) {
        const uint64_t k = heap_pop(&h);
        const uint32_t v = (uint32_t)k, d = (uint32_t)(k >> 32);
        if (d != dist[v]) continue; /* stale entry */
        for (uint32_t e = off[v]; e < off[v + 1]; ++e) {
            const uint32_t u = idx[e];
            const uint64_t cand = (uint64_t)d + (w ? w[e] : 1u);
            if (cand < dist[u]) { /* 64-bit sum: no wrap-around */
                dist[u] = (uint32_t)cand;
                if (!heap_push(&h, (cand << 32) | u)) {
                    free(h.a);
                    return -2;
                }
            }
        }
    }
    free(h.a);
    return 0;
}

/* ---------------------------------------------------------------- PageRank fixed point, FP64 */
int sgo_pagerank_jacobi_f64(uint32_t nv, const uint32_t *off, const uint32_t *idx, double tol, uint32_t max_iter,
                            double *ranks, uint32_t *iterations) {
    const uint64_t ne = off[nv];
    uint64_t *coff = (uint64_t *)calloc((size_t)nv + 1, sizeof(uint64_t));
    uint64_t *cur = (uint64_t *)malloc(((size_t)nv + 1) * sizeof(uint64_t));
    uint32_t *csrc = (uint32_t *)malloc((ne ? ne : 1) * sizeof(uint32_t));
    double *contrib = (double *)malloc(((size_t)nv + 1) * sizeof(double));
    double *next = (double *)malloc(((size_t)nv + 1) * sizeof(double));
    if (!coff || !cur || !csrc || !contrib || !next) return -1;
    for (uint64_t e = 0; e < ne; ++e) coff[idx[e] + 1]++;
    for (uint32_t v = 0; v < nv; ++v) coff[v + 1] += coff[v];
    memcpy(cur, coff, ((size_t)nv + 1) * sizeof(uint64_t));
    for (uint32_t u = 0; u < nv; ++u)
        for (uint32_t e = off[u]; e < off[u + 1]; ++e) csrc[cur[idx[e]]++] = u;
    for (uint32_t v = 0; v < nv; ++v) ranks[v] = 1.0 - SGO_ALPHA;
    uint32_t it = 0;
    for (; it < max_iter; ++it) {
#pragma omp parallel for schedule(static)
        for (int64_t u = 0; u < (int64_t)nv; ++u) {
            const uint32_t deg = off[u + 1] - off[u];
            contrib[u] = deg ? SGO_ALPHA * ranks[u] / deg : 0.0;
        }
        double diff = 0.0, norm = 0.0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(+ : diff, norm)
        for (int64_t v = 0; v < (int64_t)nv; ++v) {
            double s = 0.0;
            for (uint64_t e = coff[v]; e < coff[v + 1]; ++e) s += contrib[csrc[e]];
            const double x = (1.0 - SGO_ALPHA) + s;
            diff += x > ranks[v] ? x - ranks[v] : ranks[v] - x;
            norm += x;
            next[v] = x;
        }
        memcpy(ranks, next, (size_t)nv * sizeof(double));
        if (diff <= tol * norm) {
            ++it;
            break;
        }
    }
    if (iterations) *iterations = it;
    free(coff);
    free(cur);
    free(csrc);
    free(contrib);
    free(next);
    return 0;
}

/* Number of host threads the parallel loops above use. */
int sgo_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
