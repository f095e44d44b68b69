/*
 * sepgraph.h — C ABI of the B200-native hybrid graph engine (libsepgraph_b200.so).
 *
 * The reference (SEP-Graph) exposes its hot path as a header-only C++ template
 * API: Engine<TValue,TBuffer,TWeight,TAppImpl,...> driven by the four sample
 * functions HybridBFS/HybridSSSP/HybridPageRank/HybridBC.  Device functors
 * cannot cross a C ABI, so the functor/template layer stays C++ (see
 * sep-graph_b200/csrc/sg_api.cuh and sg_engine.cuh) and this ABI exposes the
 * four instantiated algorithms plus the graph store, options and statistics.
 * Each entry point names the reference interface it replaces.
 *
 * Conventions
 *  - Every call returns an sg_status; nothing calls exit() or assert() (the
 *    reference uses exit(1) in GROUTE_CUDA_CHECK, include/groute/internal/cuda_utils.h:41-65).
 *  - Output buffers are caller-owned.  An output pointer may be host memory
 *    (pageable or pinned) or device memory on the context's device; the
 *    library detects which with cudaPointerGetAttributes.
 *  - One sg_ctx per host thread.  All work of a context is ordered on its
 *    stream (sg_ctx_set_stream to share a caller's stream).
 *  - Indices are uint32 (index_t in include/groute/graphs/common.h:36);
 *    edge counts are uint64 at the boundary and must be < 2^32 inside.
 */
#ifndef SEPGRAPH_B200_H
#define SEPGRAPH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SG_ABI_VERSION 2

typedef enum sg_status {
    SG_OK = 0,
    SG_ERR_INVALID_ARG = 1,   /* null pointer, out-of-range vertex, bad option */
    SG_ERR_CUDA = 2,          /* a CUDA runtime call failed (message in sg_last_error) */
    SG_ERR_OUT_OF_MEMORY = 3, /* device or host allocation failed */
    SG_ERR_TIMEOUT = 4,       /* a bounded device-side wait gave up (no GPU hang) */
    SG_ERR_CAPACITY = 5,      /* a device worklist would have overflowed; nothing was written past it */
    SG_ERR_UNSUPPORTED = 6,   /* variant the reference also rejects (e.g. ASYNC_PULL_TD, framework.cuh:672-673) */
    SG_ERR_OVERFLOW = 7,      /* uint64 path count overflow in BC */
    SG_ERR_NO_DEVICE = 8,     /* no CUDA device / cooperative launch unsupported */
    SG_ERR_IO = 9,            /* graph file could not be read or written */
    SG_ERR_FORMAT = 10,       /* graph file is malformed */
    SG_ERR_BUSY = 11          /* server queue full / budget exhausted */
} sg_status;

typedef struct sg_ctx sg_ctx;             /* device + stream + scratch cache */
typedef struct sg_graph sg_graph;         /* device-resident CSR (+CSC) graph */
typedef struct sg_hgraph sg_hgraph;       /* host CSR graph (generators, file I/O) */

/* ------------------------------------------------------------------ selectors
 * Mirror of include/framework/common.h:13-41 (LoadBalancing, Priority, Model,
 * MsgPassing, Scheduling) and AlgoVariant (common.h:43-177).  A variant id is
 * (model << 2) | (msg_passing << 1) | scheduling with SYNC=0/ASYNC=1,
 * PUSH=0/PULL=1, TOPOLOGY_DRIVEN=0/DATA_DRIVEN=1. */
enum { SG_LB_NONE = 0, SG_LB_COARSE_GRAINED = 1, SG_LB_FINE_GRAINED = 2, SG_LB_HYBRID = 3, SG_LB_AUTO = -1 };
enum { SG_PRIORITY_NONE = 0, SG_PRIORITY_LOW_HIGH = 1, SG_PRIORITY_SAMPLING = 2 };
enum {
    SG_VARIANT_AUTO = -1,
    SG_SYNC_PUSH_TD = 0, SG_SYNC_PUSH_DD = 1, SG_SYNC_PULL_TD = 2, SG_SYNC_PULL_DD = 3,
    SG_ASYNC_PUSH_TD = 4, SG_ASYNC_PUSH_DD = 5, SG_ASYNC_PULL_TD = 6, SG_ASYNC_PULL_DD = 7
};

/* Graph creation flags. */
/* CSC aliases CSR (reference --undirected, csr_graph.h:405-410).  With weights,
 * per-edge weights that differ between u->v and v->u get their own CSC weight
 * array (the reference would pull the reverse edge's weight). */
#define SG_GRAPH_SYMMETRIC 0x1u
#define SG_GRAPH_NO_CSC 0x2u     /* do not build the in-edge (CSC) view; pull variants then fail */

/* Engine options: union of EngineOptions (common.h:203-321) and the flags the
 * reference reads from gflags (include/utils/app_skeleton.h:42-87). */
typedef struct sg_options {
    int32_t variant;          /* SG_VARIANT_AUTO = hybrid policy; else ForceVariant() */
    int32_t lb_push;          /* SetLoadBalancing(PUSH, ..); SG_LB_AUTO = --lb_push "" rule */
    int32_t lb_pull;          /* SetLoadBalancing(PULL, ..) */
    int32_t priority;         /* SG_PRIORITY_NONE / LOW_HIGH (SetTwoLevelBasedPriority) */
    double priority_delta;    /* two-level priority step; <=0 with LOW_HIGH = auto (32*avg_w/avg_deg) */
    double cut_threshold;     /* with SG_PRIORITY_SAMPLING: SetSampleBasedPriority; each ASYNC_PUSH_TD round
                                 takes the vertices above the buffer value at 1000*(1-cut) of 1000 sampled */
    double alpha;             /* --alpha (15) */
    double beta;              /* --beta (18) */
    double edge_factor;       /* --edge_factor (1.0) */
    int32_t max_iteration;    /* --max_iteration (200) */
    int32_t fused;            /* SetFused(); the device-resident round loop is always used */
    int32_t block_size;       /* --block_size (256); 0 = library choice */
    int32_t non_atomic;       /* BFS --non_atomic (true) */
    int32_t trace;            /* --trace: record one sg_round_trace per round */
    double pr_error;          /* PageRank residual threshold (--error, 0.01) */
    double timeout_s;         /* bound on any device-side wait; 0 = default (30 s) */
    int32_t blocking;         /* 1: wait and fill sg_stats (default); 0: enqueue only */
    int32_t blocks_per_sm;    /* resident engine blocks per SM; 0 = library choice by graph size */
    int32_t heavy_degree;     /* push/pull: vertices above this many edges are split into chunks; 0 = 32 */
    int32_t chunk_edges;      /* edges per chunk of a split vertex; 0 = 256 */
    int32_t team_blocks;      /* batched launches: blocks per team; 0 = by graph size */
    int32_t local_depth;      /* levels a block follows its own discoveries before a round ends
                                 (0 = off; with variant SG_ASYNC_PUSH_DD and functors whose
                                 ReorderSafe() holds only) */
    int32_t wl_sort;          /* --wl_sort: sort the worklist of each data-driven push round by vertex id
                                 (framework.cuh:488-496); single-query calls, batches ignore it */
    int32_t worklist;         /* worklists of a forced SG_ASYNC_PUSH_DD run with load balancing: 0 = library
                                 choice, SG_WORKLIST_QUEUE = deduplicated queues, SG_WORKLIST_BITMAP = the
                                 output slot's bitmap itself (fire-and-forget bit sets, no appends) */
    int32_t l2_persist;       /* L2 persistence window on the array a launch updates at random (the tentative
                                 values; the pulled values of a topology-driven pull) for single-query
                                 calls: 0 = library choice (on where the device supports it), 1 = on,
                                 -1 = off.  Set on the launch's stream for that launch only; the L2
                                 set-aside it needs is returned when the last context of the device is
                                 destroyed. */
    int32_t pull_scan;        /* data-driven pull into vertices of at most 32 in-edges: 0 = library choice
                                 (SG_PULL_SCAN_THREAD), SG_PULL_SCAN_THREAD = one thread per vertex with early
                                 exit, SG_PULL_SCAN_WARP = a warp walks 32 vertices' in-edge lists together */
    int32_t hub_stage;        /* 256-edge hub chunks of SSSP: 0 = library choice, 1 = each chunk's
                                 destinations and weights staged in shared memory by bulk copies (TMA engine)
                                 one chunk ahead, -1 = read from global memory by each lane */
    int32_t reserved[1];
} sg_options;
#define SG_PULL_SCAN_THREAD 1
#define SG_PULL_SCAN_WARP 2
#define SG_WORKLIST_AUTO 0
#define SG_WORKLIST_QUEUE 1
#define SG_WORKLIST_BITMAP 2

/* Per-round trace record (the reference's --trace line, framework.cuh:334-348). */
typedef struct sg_round_trace {
    uint32_t round;
    int32_t variant;
    uint32_t in_nodes, out_nodes;
    uint64_t in_workload, out_workload;
    int64_t total_workload;
    float time_ms;
    uint32_t pad;
} sg_round_trace;

/* Run statistics (RunningInfo, include/framework/hybrid_policy.h:36-120). */
typedef struct sg_stats {
    uint32_t rounds;               /* num_iteration */
    uint32_t max_iteration_reached;
    uint32_t rounds_by_variant[8]; /* indexed by variant id */
    double time_total_ms;          /* device time of the whole solve (CUDA events) */
    double time_kernel_ms;         /* device time of the round loop */
    uint64_t edges_processed;      /* edges expanded or scanned, summed over rounds */
    uint64_t vertices_processed;   /* worklist items processed, summed over rounds */
    uint64_t edges_reached;        /* sum of out-degrees of reached vertices (GTEPS numerator) */
    uint32_t vertices_reached;
    uint32_t search_depth;         /* BFS/BC: max level */
    uint32_t device_error;         /* raw device error bits (0 = none) */
    uint32_t n_trace;              /* number of records written to trace (if provided) */
    sg_round_trace *trace;         /* caller-provided array or NULL */
    uint32_t trace_capacity;
    uint32_t pad;
} sg_stats;

/* ------------------------------------------------------------------ context */
const char *sg_status_string(sg_status s);
int sg_abi_version(void);
/* Replaces Engine::Engine(AlgoType)'s device setup (framework.cuh:84-93), which is hard-wired to device 0. */
sg_status sg_init(int device, sg_ctx **out);
sg_status sg_destroy(sg_ctx *ctx);
sg_status sg_ctx_set_stream(sg_ctx *ctx, void *cuda_stream); /* NULL = context's own stream */
sg_status sg_ctx_get_stream(sg_ctx *ctx, void **cuda_stream);
/* Waits for all enqueued work; returns the first device error of non-blocking calls. */
sg_status sg_ctx_synchronize(sg_ctx *ctx);
/* Detail message of the last failure on this context (never NULL). */
const char *sg_last_error(const sg_ctx *ctx);
sg_status sg_device_info(sg_ctx *ctx, int *sm_count, uint64_t *hbm_bytes, uint64_t *l2_bytes, char *name, size_t name_len);

/* ------------------------------------------------------------------ graph store
 * Replaces Engine::LoadGraph (framework.cuh:99-133) + single::CSRGraphAllocator /
 * CSCGraphAllocator (csr_graph.h:1596-1783): uploads CSR, builds CSC (csr_tocsc,
 * csr_graph.h:329-397) unless symmetric. offsets has nv+1 entries. */
sg_status sg_graph_create(sg_ctx *ctx, uint32_t nv, uint64_t ne, const uint32_t *offsets, const uint32_t *indices,
                          const uint32_t *weights, uint32_t flags, sg_graph **out);
sg_status sg_graph_create_from_host(sg_ctx *ctx, const sg_hgraph *h, uint32_t flags, sg_graph **out);
/* The context keeps the arena of the last released graph (the larger one when
 * several are released) and the next sg_graph_create / sg_graph_build whose
 * graph needs between half of it and all of it reuses it, so reloading a graph
 * costs no device allocation.  sg_ctx_release_cached frees that arena and the
 * context's scratch of single-query and batched calls (reallocated on demand);
 * sg_destroy frees everything. */
sg_status sg_graph_destroy(sg_graph *g);
sg_status sg_ctx_release_cached(sg_ctx *ctx);
sg_status sg_graph_info(const sg_graph *g, uint32_t *nv, uint64_t *ne, uint64_t *device_bytes, int *weighted);

/* Edge list -> device graph, built on the GPU.  Replaces the preprocessing of
 * the reference's converter (samples/tools/gtools.cpp:56-328) together with the
 * CSR construction and csr_tocsc (csr_graph.h:329-397) that Engine::LoadGraph
 * runs on the host.  src/dst/weights hold m entries (host or device memory;
 * weights may be NULL).  Within a row, edges keep their input order unless a
 * flag orders them; the CSC view is built on the device as for sg_graph_create.
 * Failure: SG_ERR_INVALID_ARG for an endpoint >= nv or more than 2^32-2 entries
 * (after --d2ud doubling). */
#define SG_BUILD_DESELF_CYCLE 0x1u /* gtools --deself_cycle: drop edges u->u */
#define SG_BUILD_DEDUPLICATE 0x2u  /* gtools --deduplicate: per source keep the first edge to each destination */
#define SG_BUILD_D2UD 0x4u         /* gtools --d2ud: add every reverse edge; rows sorted by destination and
                                      deduplicated, the first inserted edge's weight kept; implies
                                      SG_GRAPH_SYMMETRIC */
#define SG_BUILD_SORT_ROWS 0x8u    /* rows ordered by destination (input order among equal destinations) */
sg_status sg_graph_build(sg_ctx *ctx, uint32_t nv, uint64_t m, const uint32_t *src, const uint32_t *dst,
                         const uint32_t *weights, uint32_t build_flags, uint32_t graph_flags, sg_graph **out);
/* Copies a device graph's CSR (csc == 0) or in-edge CSC view (csc != 0) into
 * caller buffers (host or device): offsets nv+1, indices ne, weights ne (NULL
 * skips them).  SG_ERR_UNSUPPORTED when the graph has no CSC view.  No
 * reference counterpart (the reference keeps its CSC on the host,
 * csr_graph.h:1596-1783). */
sg_status sg_graph_copy_out(const sg_graph *g, int csc, uint32_t *offsets, uint32_t *indices, uint32_t *weights);

sg_status sg_options_default(sg_options *opt);

/* ------------------------------------------------------------------ algorithms */
/* HybridBFS (samples/hybrid_bfs/hybrid_bfs.cu:173-243). levels_out: nv uint32, UINT32_MAX = unreached. */
sg_status sg_bfs(sg_graph *g, uint32_t source, const sg_options *opt, uint32_t *levels_out, sg_stats *stats);
/* HybridSSSP (samples/hybrid_sssp/hybrid_sssp.cu:151-243). Unweighted graphs use weight 1. */
sg_status sg_sssp(sg_graph *g, uint32_t source, const sg_options *opt, uint32_t *dist_out, sg_stats *stats);
/* HybridPageRank (samples/hybrid_pr/hybrid_pr.cu:128-210). Damping 0.85 as ALPHA in hybrid_pr_common.h:39.
 * ranks_out: nv float (the engine value array); residual_out optional (GatherBuffer). */
sg_status sg_pagerank(sg_graph *g, const sg_options *opt, float *ranks_out, float *residual_out, sg_stats *stats);
/* HybridBC (samples/hybrid_bc/hybrid_bc.cu:303-412): single-source Brandes, bc already halved
 * like hybrid_bc.cu:374-376. sigma_out optional (uint64 path counts). */
sg_status sg_bc(sg_graph *g, uint32_t source, const sg_options *opt, float *bc_out, uint64_t *sigma_out,
                sg_stats *stats);

/* ------------------------------------------------------------------ batching
 * No counterpart in the reference (one source per Engine).  Multi-source BFS:
 * up to 64 sources in one persistent launch with 64-bit per-vertex source
 * masks.  levels_out holds nsrc rows of nv uint32 (row i = BFS from
 * sources[i], identical to sg_bfs from that source). */
sg_status sg_msbfs(sg_graph *g, const uint32_t *sources, uint32_t nsrc, const sg_options *opt, uint32_t *levels_out,
                   sg_stats *stats);

/* sg_msbfs on a chosen context (stream and scratch of ctx; the graph may belong
 * to another context of the same device). */
sg_status sg_msbfs_on(sg_ctx *ctx, sg_graph *g, const uint32_t *sources, uint32_t nsrc, const sg_options *opt,
                      uint32_t *levels_out, sg_stats *stats);

/* One query of a batch: graph (any graph of the context), source, and the
 * output array of graph->nv uint32 (host or device memory). */
/* Multi-source BC: up to 32 sources of one graph in one launch (bit-parallel
 * forward over in-edges, level-by-level backward); bc_out holds nsrc rows of
 * nv floats (host or device), row i equal to sg_bc(g, sources[i]) within
 * float summation order.  Needs the graph's in-edge view (CSC or
 * SG_GRAPH_SYMMETRIC), else SG_ERR_UNSUPPORTED.  Device memory ~ 40 x nv x 32
 * bytes of scratch.  No reference counterpart (one source per Engine). */
sg_status sg_msbc(sg_graph *g, const uint32_t *sources, uint32_t nsrc, const sg_options *opt, float *bc_out,
                  sg_stats *stats);

typedef struct sg_batch_query {
    sg_graph *graph;
    uint32_t source;
    uint32_t pad;
    void *out;
} sg_batch_query;

/* Batched SSSP / BFS: n queries over any mix of graphs in ONE cooperative
 * launch.  The grid is split into teams of blocks (sg_options.team_blocks =
 * blocks per team, 0 = by graph size); each team runs one query's whole round
 * loop with its own frontiers and takes the next query (largest graphs first)
 * when done.  Every output equals sg_sssp / sg_bfs for that query.  stats is
 * the aggregate (time of the launch, summed reached edges);
 * per_query_ms (optional, n floats) receives each query's device time. */
sg_status sg_sssp_batch(sg_ctx *ctx, const sg_batch_query *q, uint32_t n, const sg_options *opt, sg_stats *stats,
                        float *per_query_ms);
sg_status sg_bfs_batch(sg_ctx *ctx, const sg_batch_query *q, uint32_t n, const sg_options *opt, sg_stats *stats,
                       float *per_query_ms);

/* Batched single-source BC: each team runs one query's hybrid forward pass and
 * its backward dependency pass in the same launch; out receives graph->nv
 * floats equal to sg_bc's bc_out for that source (path counts stay on the
 * device).  stats->edges_reached counts both traversals, as sg_bc does. */
sg_status sg_bc_batch(sg_ctx *ctx, const sg_batch_query *q, uint32_t n, const sg_options *opt, sg_stats *stats,
                      float *per_query_ms);

/* A batch planned once and launched many times (algo = SG_QUERY_BFS, _SSSP or
 * _BC): query descriptors, team workspaces (owned by the plan) and outputs are
 * fixed at creation, and each launch replays one CUDA graph holding the
 * per-launch memsets and the cooperative kernel on the context's stream (or
 * issues the same calls directly where the driver cannot capture them;
 * sg_batch_plan_captured tells which).  Outputs must be device memory.
 * sg_batch_plan_launch does not wait; sg_batch_plan_wait waits for the last
 * launch and fills stats / per_query_ms like sg_sssp_batch.  The graphs must
 * outlive the plan. */
typedef struct sg_batch_plan sg_batch_plan;
sg_status sg_batch_plan_create(sg_ctx *ctx, int algo, const sg_batch_query *q, uint32_t n, const sg_options *opt,
                               sg_batch_plan **out);
sg_status sg_batch_plan_launch(sg_batch_plan *plan);
sg_status sg_batch_plan_wait(sg_batch_plan *plan, sg_stats *stats, float *per_query_ms);
int sg_batch_plan_captured(const sg_batch_plan *plan);
sg_status sg_batch_plan_destroy(sg_batch_plan *plan);

/* ------------------------------------------------------------------ serving
 * No counterpart in the reference.  A query server over device-resident
 * graphs with continuous batching: `slots` worker threads, each with its own
 * context and stream, repeatedly take a group of pending queries (one
 * algorithm, across graphs by default, up to max_batch),
 * admit them against the HBM budget and run them as one batched launch
 * (multi-source BFS or BC per graph, sg_sssp_batch / sg_bfs_batch /
 * sg_bc_batch teams, one PageRank per graph shared by its queries).  Queries that arrive while batches run are taken as soon as
 * a slot frees; batches of different slots overlap on the device.  Every
 * result equals the single-query call's. */
typedef struct sg_server sg_server;
enum { SG_QUERY_BFS = 0, SG_QUERY_SSSP = 1, SG_QUERY_PAGERANK = 2, SG_QUERY_BC = 3 };
typedef struct sg_server_config {
    uint64_t hbm_budget_bytes; /* admission budget for batch scratch and staging (0 = 1/4 of HBM) */
    uint32_t slots;            /* concurrent batches (default 2; measured on B200 over the mixed
                                  16-graph stream: 1 slot 274-280, 2 slots 234-261, 3 slots 174-203
                                  queries/s, with 2 keeping a long batch from holding up the rest) */
    uint32_t max_batch;        /* queries per batch (default 256) */
    uint32_t max_pending;      /* submit returns SG_ERR_BUSY beyond this (default 1<<20) */
    uint32_t msbfs_min;        /* BFS queries of one graph that go to multi-source BFS (default 4) */
    uint32_t sssp_delta;       /* SSSP two-level priority delta; 0 = each graph's 32*avg_w/avg_deg */
    uint32_t pad;
    double pr_error;           /* PageRank residual threshold (default 1e-7) */
    int32_t batch_graphs;      /* 0 = library choice (SG_BATCH_MIXED); SG_BATCH_MIXED: a batch takes the
                                  chosen query's peers of the same algorithm on any graph (one team batch
                                  across graphs: the highest throughput); SG_BATCH_ONE_GRAPH: peers on the
                                  same graph only, so a query on a small graph never waits for a large
                                  graph's traversal inside its batch */
    int32_t order;             /* with SG_BATCH_ONE_GRAPH, which pending group a free slot takes: 0 = library
                                  choice (SG_ORDER_SHORTEST_FIRST); SG_ORDER_SHORTEST_FIRST: the (algorithm,
                                  graph) group whose batches have run shortest so far (measured per group,
                                  untried groups first), unless the oldest query has waited longer than
                                  max_wait_ms, whose group then goes first; SG_ORDER_OLDEST_FIRST: the
                                  oldest query's group.  Mixed batches always start from the oldest query. */
    uint32_t max_wait_ms;      /* aging bound of SG_ORDER_SHORTEST_FIRST (0 = 500 ms) */
    uint32_t blocks_per_sm;    /* resident blocks per SM of each slot's launches (0 = 6 / slots, at least 1,
                                  for team batches; multi-source BFS / BC choose by graph and source count),
                                  at most 1/slots of what the launched kernel fits per SM, so that every
                                  slot's cooperative grid is resident beside the others' */
    int32_t reserved[4];
} sg_server_config;
#define SG_BATCH_ONE_GRAPH 1
#define SG_BATCH_MIXED 2
#define SG_ORDER_SHORTEST_FIRST 1
#define SG_ORDER_OLDEST_FIRST 2
typedef struct sg_query {
    int32_t algo;      /* SG_QUERY_* */
    uint32_t graph_id; /* from sg_server_add_graph */
    uint32_t source;   /* ignored by PageRank */
    uint32_t pad;
    void *out;         /* host buffer of nv elements: uint32 levels / distances, float ranks / bc */
    void *out2;        /* BC: optional uint64 path counts */
} sg_query;
typedef struct sg_server_stats {
    uint64_t submitted, completed, failed, batches, pending;
    double elapsed_s; /* first submit to last completion */
    double qps, mean_ms, p50_ms, p99_ms, p999_ms, max_ms;
    uint64_t hbm_budget, hbm_in_use, hbm_peak;
} sg_server_stats;
sg_status sg_server_config_default(sg_server_config *cfg);
sg_status sg_server_create(int device, const sg_server_config *cfg, sg_server **out);
sg_status sg_server_add_graph(sg_server *s, sg_graph *g, uint32_t *graph_id);
sg_status sg_server_submit(sg_server *s, const sg_query *q, uint64_t *ticket);
/* Waits for one query; *result receives its status, *latency_ms submit-to-completion. */
sg_status sg_server_wait(sg_server *s, uint64_t ticket, double timeout_s, sg_status *result, double *latency_ms);
sg_status sg_server_drain(sg_server *s, double timeout_s);
sg_status sg_server_get_stats(sg_server *s, sg_server_stats *st);
sg_status sg_server_reset_stats(sg_server *s);
sg_status sg_server_destroy(sg_server *s);
/* With the environment variable SEPGRAPH_SERVER_LOG naming a file when the
 * server is created, every batch appends one line to it: slot, algorithm,
 * queries, estimated device bytes, device-side wall time in ms. */

/* ------------------------------------------------------------------ autotuner
 * No counterpart in the reference (its variants, thresholds and grid shape are
 * command-line choices).  Times candidate options for one algorithm
 * (SG_QUERY_*) on the given graph and sources in stages, each keeping the best
 * so far: the mode (hybrid policy, forced push, forced pull; for SSSP the
 * two-level priority delta around the reference heuristic 32*avg_w/avg_deg),
 * then blocks per SM, push load balancing, local lookahead depth (BFS/SSSP)
 * and the heavy-vertex split threshold.  Every candidate must give the first
 * candidate's result (bit-exact for BFS/SSSP, PageRank L1 within
 * max(1e-6, 20 * pr_error), BC 1e-4 relative) before its time counts.  Writes
 * the fastest to *best (starting from *base, NULL = defaults); report
 * (optional) receives one line per candidate; at most max_candidates are timed
 * (0 = 64). */
typedef struct sg_tune_entry {
    sg_options options;
    double ms;       /* median device time per source */
    int32_t status;  /* sg_status of the candidate; SG_ERR_FORMAT if its result differed */
    int32_t pad;
} sg_tune_entry;
sg_status sg_autotune(sg_graph *g, int algo, const uint32_t *sources, uint32_t nsrc, const sg_options *base,
                      uint32_t max_candidates, sg_options *best, double *best_ms, sg_tune_entry *report,
                      uint32_t report_capacity, uint32_t *n_report);

/* BFS that allocates nothing, for callers that cannot call cudaMalloc (code
 * running inside another framework's memory pool or under a device-memory
 * budget).  No counterpart in the reference.  Runs the sg_bfs engine on the
 * calling thread's current device with every worklist, bitmap and control word
 * in one fixed file-scope device array (about 19 MB, held by every GPU that
 * loads it until exit).  Limits: nv <= 262144 vertices, ne <= 8388608 edges;
 * larger graphs return SG_ERR_CAPACITY before any work.  offsets/indices (CSR),
 * optional in_offsets/in_indices (CSC; pass the CSR again for a symmetric
 * graph, NULL for push-only) and levels_out are device memory of the current
 * device.  The first call on a device looks up the array's address; make it
 * before any stream capture.  Calls share the array: calls that overlap on the
 * GPU race.  opt NULL = sg_options_default(); automatic choices (load
 * balancing, blocks per SM) follow sg_bfs's rules.  stats (optional) gets
 * rounds, max_iteration_reached, rounds_by_variant, edges_processed,
 * vertices_processed and device_error; its time and reached-vertex fields and
 * n_trace are set to 0.  Blocks until done; err (optional) receives a message. */
sg_status sg_bfs_noalloc(const uint32_t *offsets, const uint32_t *indices, uint32_t nv, uint64_t ne,
                         const uint32_t *in_offsets, const uint32_t *in_indices, uint32_t source,
                         const sg_options *opt, uint32_t *levels_out, void *cuda_stream, sg_stats *stats, char *err,
                         size_t err_len);

/* ------------------------------------------------------------------ host graphs (ingest)
 * Seeded generators (the reference's generators are unseeded, traversal.h:173-189)
 * and Galois .gr I/O (src/utils/parser.cpp:409-506). */
#define SG_GEN_SYMMETRIC 0x1u      /* add reverse edges (gtools-style symmetrise) */
#define SG_GEN_KEEP_SELF_LOOPS 0x2u
#define SG_GEN_KEEP_DUPLICATES 0x4u
sg_status sg_hgraph_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                             uint32_t flags, sg_hgraph **out);
sg_status sg_hgraph_gen_grid(uint32_t rows, uint32_t cols, uint32_t flags, sg_hgraph **out);
/* Random graph of the reference's --gen_graph --gen_method 0 (CSRGraphGenerator,
 * csr_graph.h:483-541): every vertex gets U[1, gen_factor] distinct random
 * neighbours other than itself; seeded here, rows sorted. */
sg_status sg_hgraph_gen_random(uint32_t nv, uint32_t gen_factor, uint64_t seed, sg_hgraph **out);
sg_status sg_hgraph_from_csr(uint32_t nv, uint64_t ne, const uint32_t *offsets, const uint32_t *indices,
                             const uint32_t *weights, sg_hgraph **out);
/* Attach uniform weights in [lo, hi) drawn from a counter-based stream (seed, edge index). */
sg_status sg_hgraph_gen_weights(sg_hgraph *h, uint32_t lo, uint32_t hi, uint64_t seed);
sg_status sg_hgraph_read_gr(const char *path, sg_hgraph **out);
sg_status sg_hgraph_write_gr(const sg_hgraph *h, const char *path);
sg_status sg_hgraph_read_market(const char *path, int symmetrize, sg_hgraph **out);
/* METIS graph file (ReadGraph, src/utils/parser.cpp:230-396): 1-based
 * adjacency lists in file order, every undirected edge listed twice; edge
 * weights when fmt's last digit is 1; vertex sizes/weights are skipped.
 * SG_ERR_FORMAT when the entry count differs from twice the header's m. */
sg_status sg_hgraph_read_metis(const char *path, sg_hgraph **out);
/* Pointers stay valid until sg_hgraph_destroy. weights is NULL when unweighted. */
sg_status sg_hgraph_info(const sg_hgraph *h, uint32_t *nv, uint64_t *ne, const uint32_t **offsets,
                         const uint32_t **indices, const uint32_t **weights);
/* GetMaxOutDgrNode (csr_graph.h:241-259): lowest id among maximum out-degree. */
sg_status sg_hgraph_max_degree_vertex(const sg_hgraph *h, uint32_t *vertex, uint32_t *degree);
/* n seeded random vertices with out-degree > 0. */
sg_status sg_hgraph_pick_sources(const sg_hgraph *h, uint32_t n, uint64_t seed, uint32_t *out);
sg_status sg_hgraph_destroy(sg_hgraph *h);

#ifdef __cplusplus
}
#endif
#endif /* SEPGRAPH_B200_H */
