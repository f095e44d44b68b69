/*
 * ORACLE — test infrastructure only.  Never linked into or called by the
 * product library; only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference arm load it (as the checker or the CPU baseline).
 *
 * Plain-C restatement of the reference's single-threaded host algorithms:
 *   sgo_bfs            BFSHost                    samples/hybrid_bfs/hybrid_bfs_host.cpp:33-60
 *   sgo_sssp           SSSPHostNaive              samples/hybrid_sssp/hybrid_sssp_host.cpp:34-60
 *   sgo_pagerank_f32   PageRankHost               samples/hybrid_pr/hybrid_pr_host.cpp:43-124
 *   sgo_pagerank_f64   same algorithm in double (precision oracle)
 *   sgo_bc_f32         BetweennessCentralityHost  samples/hybrid_bc/hybrid_bc_host.cpp:16-92
 *   sgo_bc_f64         same algorithm with double path counts and dependencies
 * The f32 forms repeat the reference's float arithmetic step for step (same
 * operation order, float storage, double constants) so that they reproduce its
 * output bit for bit; tests pin them against the reference compiled from its
 * own sources (oracle/_ref) and against committed golden vectors.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SGO_INF 0xffffffffu
#define SGO_ALPHA 0.85 /* hybrid_pr_common.h:39 */

typedef struct {
    uint32_t *a;
    size_t head, tail, cap;
} fifo_t;

static int fifo_init(fifo_t *q, size_t cap) {
    q->cap = cap < 16 ? 16 : cap;
    q->head = q->tail = 0;
    q->a = (uint32_t *)malloc(q->cap * sizeof(uint32_t));
    return q->a != NULL;
}
static int fifo_push(fifo_t *q, uint32_t v) {
    if (q->tail == q->cap) {
        if (q->head > 0) { /* compact */
            memmove(q->a, q->a + q->head, (q->tail - q->head) * sizeof(uint32_t));
            q->tail -= q->head;
            q->head = 0;
        }
        if (q->tail == q->cap) {
            size_t nc = q->cap * 2;
            uint32_t *na = (uint32_t *)realloc(q->a, nc * sizeof(uint32_t));
            if (!na) return 0;
            q->a = na;
            q->cap = nc;
        }
    }
    q->a[q->tail++] = v;
    return 1;
}
static int fifo_empty(const fifo_t *q) { return q->head == q->tail; }
static uint32_t fifo_pop(fifo_t *q) { return q->a[q->head++]; }
static void fifo_free(fifo_t *q) { free(q->a); }

/* BFSHost: FIFO traversal, level[dst] = level[node] + 1 on first visit. */
int sgo_bfs(uint32_t nv, const uint32_t *off, const uint32_t *idx, uint32_t src, uint32_t *levels) {
    fifo_t q;
    if (src >= nv || !fifo_init(&q, nv)) return -1;
    for (uint32_t v = 0; v < nv; ++v) levels[v] = SGO_INF;
    levels[src] = 0;
    fifo_push(&q, src);
    while (!fifo_empty(&q)) {
        uint32_t node = fifo_pop(&q);
        uint32_t lv = levels[node];
        for (uint32_t e = off[node]; e < off[node + 1]; ++e) {
            uint32_t d = idx[e];
            if (levels[d] == SGO_INF) {
                levels[d] = lv + 1;
                if (!fifo_push(&q, d)) return -2;
            }
        }
    }
    fifo_free(&q);
    return 0;
}

/* SSSPHostNaive: FIFO label-correcting; a vertex is re-queued on every improvement. */
int sgo_sssp(uint32_t nv, const uint32_t *off, const uint32_t *idx, const uint32_t *w, uint32_t src, uint32_t *dist) {
    fifo_t q;
    if (src >= nv || !fifo_init(&q, nv)) return -1;
    for (uint32_t v = 0; v < nv; ++v) dist[v] = SGO_INF;
    dist[src] = 0;
    fifo_push(&q, src);
    while (!fifo_empty(&q)) {
        uint32_t node = fifo_pop(&q);
        uint32_t dn = dist[node];
        for (uint32_t e = off[node]; e < off[node + 1]; ++e) {
            uint32_t d = idx[e];
            uint32_t cand = dn + (w ? w[e] : 1u);
            if (dist[d] > cand) {
                dist[d] = cand;
                if (!fifo_push(&q, d)) return -2;
            }
        }
    }
    fifo_free(&q);
    return 0;
}

/* PageRankHost in float, operation for operation. */
int sgo_pagerank_f32(uint32_t nv, const uint32_t *off, const uint32_t *idx, double error, float *ranks,
                     uint32_t *iterations) {
    float *residual = (float *)calloc(nv ? nv : 1, sizeof(float));
    fifo_t in, out;
    if (!residual || !fifo_init(&in, nv) || !fifo_init(&out, nv)) return -1;
    for (uint32_t v = 0; v < nv; ++v) ranks[v] = (float)(1.0 - SGO_ALPHA);
    for (uint32_t v = 0; v < nv; ++v) {
        uint32_t deg = off[v + 1] - off[v];
        if (deg == 0) continue;
        float update = (float)(((1.0 - SGO_ALPHA) * SGO_ALPHA) / deg);
        for (uint32_t e = off[v]; e < off[v + 1]; ++e) residual[idx[e]] += update;
    }
    for (uint32_t v = 0; v < nv; ++v) fifo_push(&in, v);
    uint32_t it = 0;
    while (!fifo_empty(&in)) {
        while (!fifo_empty(&in)) {
            uint32_t node = fifo_pop(&in);
            float res = residual[node];
            ranks[node] += res;
            residual[node] = 0;
            uint32_t deg = off[node + 1] - off[node];
            if (deg == 0) continue;
            float update = (float)(res * SGO_ALPHA / deg);
            for (uint32_t e = off[node]; e < off[node + 1]; ++e) {
                uint32_t d = idx[e];
                float prev = residual[d];
                residual[d] += update;
                float sum = prev + update;
                if ((double)sum > error && (double)prev < error) {
                    if (!fifo_push(&out, d)) return -2;
                }
            }
        }
        ++it;
        fifo_t t = in;
        in = out;
        out = t;
        out.head = out.tail = 0;
    }
    if (iterations) *iterations = it;
    fifo_free(&in);
    fifo_free(&out);
    free(residual);
    return 0;
}

/* Same residual-push PageRank in double (the precision oracle). */
int sgo_pagerank_f64(uint32_t nv, const uint32_t *off, const uint32_t *idx, double error, double *ranks,
                     uint32_t *iterations) {
    double *residual = (double *)calloc(nv ? nv : 1, sizeof(double));
    fifo_t in, out;
    if (!residual || !fifo_init(&in, nv) || !fifo_init(&out, nv)) return -1;
    for (uint32_t v = 0; v < nv; ++v) ranks[v] = 1.0 - SGO_ALPHA;
    for (uint32_t v = 0; v < nv; ++v) {
        uint32_t deg = off[v + 1] - off[v];
        if (deg == 0) continue;
        double update = ((1.0 - SGO_ALPHA) * SGO_ALPHA) / deg;
        for (uint32_t e = off[v]; e < off[v + 1]; ++e) residual[idx[e]] += update;
    }
    for (uint32_t v = 0; v < nv; ++v) fifo_push(&in, v);
    uint32_t it = 0;
    while (!fifo_empty(&in)) {
        while (!fifo_empty(&in)) {
            uint32_t node = fifo_pop(&in);
            double res = residual[node];
            ranks[node] += res;
            residual[node] = 0;
            uint32_t deg = off[node + 1] - off[node];
            if (deg == 0) continue;
            double update = res * SGO_ALPHA / deg;
            for (uint32_t e = off[node]; e < off[node + 1]; ++e) {
                uint32_t d = idx[e];
                double prev = residual[d];
                residual[d] += update;
                if (prev + update > error && prev < error) {
                    if (!fifo_push(&out, d)) return -2;
                }
            }
        }
        ++it;
        fifo_t t = in;
        in = out;
        out = t;
        out.head = out.tail = 0;
    }
    if (iterations) *iterations = it;
    fifo_free(&in);
    fifo_free(&out);
    free(residual);
    return 0;
}

/* BetweennessCentralityHost: level-synchronous forward pass counting shortest
 * paths, backward accumulation over depths search_depth-2 .. 1, then x0.5.
 * Generated twice: float (reference arithmetic) and double. */
#define SGO_BC_BODY(REAL, SIGMA_ADD_ONE)                                                      \
    int32_t *path = (int32_t *)malloc((nv ? nv : 1) * sizeof(int32_t));                      \
    fifo_t in, out;                                                                            \
    if (src >= nv || !path || !fifo_init(&in, nv) || !fifo_init(&out, nv)) return -1;         \
    for (uint32_t v = 0; v < nv; ++v) {                                                        \
        path[v] = -1;                                                                          \
        bc[v] = 0;                                                                             \
        sigma[v] = 0;                                                                          \
    }                                                                                          \
    path[src] = 0;                                                                             \
    int32_t depth = 0;                                                                         \
    sigma[src] = 1;                                                                            \
    fifo_push(&in, src);                                                                       \
    while (!fifo_empty(&in)) {                                                                 \
        while (!fifo_empty(&in)) {                                                             \
            uint32_t node = fifo_pop(&in);                                                     \
            int32_t nd = path[node] + 1;                                                       \
            for (uint32_t e = off[node]; e < off[node + 1]; ++e) {                             \
                uint32_t d = idx[e];                                                           \
                if (path[d] == -1) {                                                           \
                    path[d] = nd;                                                              \
                    sigma[d] += sigma[node];                                                   \
                    if (depth < nd) depth = nd;                                                \
                    if (!fifo_push(&out, d)) return -2;                                        \
                } else if (path[d] == path[node] + 1) {                                        \
                    sigma[d] += sigma[node];                                                   \
                }                                                                              \
            }                                                                                  \
        }                                                                                      \
        fifo_t t = in;                                                                         \
        in = out;                                                                              \
        out = t;                                                                               \
        out.head = out.tail = 0;                                                               \
    }                                                                                          \
    depth++;                                                                                   \
    for (int32_t it = depth - 2; it > 0; --it)                                                 \
        for (uint32_t node = 0; node < nv; ++node)                                             \
            if (path[node] == it)                                                              \
                for (uint32_t e = off[node]; e < off[node + 1]; ++e) {                         \
                    uint32_t d = idx[e];                                                       \
                    if (path[d] == it + 1)                                                     \
                        bc[node] += SIGMA_ADD_ONE * sigma[node] / sigma[d] * (SIGMA_ADD_ONE + bc[d]); \
                }                                                                              \
    for (uint32_t v = 0; v < nv; ++v) bc[v] *= (REAL)0.5;                                      \
    if (levels)                                                                                \
        for (uint32_t v = 0; v < nv; ++v) levels[v] = path[v] < 0 ? SGO_INF : (uint32_t)path[v]; \
    fifo_free(&in);                                                                            \
    fifo_free(&out);                                                                           \
    free(path);                                                                                \
    return 0;

int sgo_bc_f32(uint32_t nv, const uint32_t *off, const uint32_t *idx, uint32_t src, float *bc, float *sigma,
               uint32_t *levels) {
    SGO_BC_BODY(float, 1.0f)
}

int sgo_bc_f64(uint32_t nv, const uint32_t *off, const uint32_t *idx, uint32_t src, double *bc, double *sigma,
               uint32_t *levels) {
    SGO_BC_BODY(double, 1.0)
}
