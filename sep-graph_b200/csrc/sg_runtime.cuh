// Host runtime of the B200 hybrid engine: context, device graph store,
// per-graph workspace cache, the cooperative launch of the engine kernel and
// the C++ Engine class that mirrors the reference's
// sepgraph::engine::Engine (include/framework/framework.cuh:56-797).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/sepgraph.h"
#include "sg_internal.h"
#include "sg_engine.cuh"

namespace sgb {
struct Workspace;
}

struct sg_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaDeviceProp prop{};
    std::string last_error;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint32_t pending_error = 0;
    // pinned host staging for control-block read-back
    void *pinned = nullptr;
    size_t pinned_bytes = 0;
    int live_graphs = 0;  // sg_destroy refuses while graphs of this context exist
    sgb::Workspace *batch_ws = nullptr;  // scratch of batched launches (team workspaces)
    sgb::Workspace *graph_ws = nullptr;  // scratch of single-query calls, shared by the context's graphs
    // the arena of the last released graph, reused by the next graph that fits
    // (between half its size and its size): reloading a graph costs no cudaMalloc/cudaFree
    void *spare_arena = nullptr;
    size_t spare_bytes = 0;
    bool persist_ref = false;  // holds a reference on the device's persisting-L2 set-aside
    // Contexts whose persistent launches run side by side on the device (a
    // server's slots): each launch takes at most 1/resident_share of a kernel's
    // resident blocks per SM, so that every slot's cooperative grid fits beside
    // the others' instead of waiting for one of them to end.
    uint32_t resident_share = 1;
};

namespace sgb {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

// Stream-ordered memory pool of a device, created on first use, that keeps
// freed memory for reuse (release threshold at its maximum) until a context is
// destroyed (sg_destroy trims it).  nullptr when the device offers no pool.
inline cudaMemPool_t device_pool(int device) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    if (device < 0 || device >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[device]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[device] = p;
    }
    return pools[device];
}

// Grow-only device buffers owned by one context.  Work on a context is ordered
// on its stream, so consecutive queries reuse them without reallocating.  A
// context's workspaces allocate, zero and free on the context's stream from
// the device pool: growing a buffer never waits for work that other contexts
// (a server's other slots) have in flight, as cudaFree would.  A workspace
// without a stream (a batch plan's, whose addresses a captured graph holds)
// uses cudaMalloc and cudaFree.
struct Workspace {
    std::map<std::string, DevBuf> bufs;
    const cudaStream_t *stream = nullptr;  // the owning context's current stream
    cudaMemPool_t pool = nullptr;
    Workspace() = default;
    Workspace(const cudaStream_t *s, cudaMemPool_t p) : stream(s), pool(p) {}
    Workspace(const Workspace &) = delete;
    Workspace &operator=(const Workspace &) = delete;
    bool ordered() const { return stream && pool; }
    ~Workspace() {
        for (auto &kv : bufs)
            if (kv.second.p) {
                if (ordered()) cudaFreeAsync(kv.second.p, *stream);
                else cudaFree(kv.second.p);
            }
        if (ordered()) cudaStreamSynchronize(*stream);
    }
    template <typename T>
    cudaError_t get(const char *name, size_t count, T **out, bool zero_new = false) {
        DevBuf &b = bufs[name];
        size_t bytes = count * sizeof(T);
        if (bytes == 0) bytes = 256;
        bytes = (bytes + 255) & ~size_t(255);
        if (b.bytes < bytes) {
            if (b.p) {
                if (ordered()) cudaFreeAsync(b.p, *stream);
                else cudaFree(b.p);
            }
            b.p = nullptr;
            b.bytes = 0;
            cudaError_t e = ordered() ? cudaMallocFromPoolAsync(&b.p, bytes, pool, *stream) : cudaMalloc(&b.p, bytes);
            if (e != cudaSuccess) return e;
            b.bytes = bytes;
            if (zero_new) {
                e = ordered() ? cudaMemsetAsync(b.p, 0, bytes, *stream) : cudaMemset(b.p, 0, bytes);
                if (e != cudaSuccess) return e;
            }
        }
        *out = (T *)b.p;
        return cudaSuccess;
    }
    size_t total_bytes() const {
        size_t s = 0;
        for (auto &kv : bufs) s += kv.second.bytes;
        return s;
    }
};

}  // namespace sgb

struct sg_graph {
    sg_ctx *ctx = nullptr;
    uint32_t nv = 0;
    uint64_t ne = 0;
    bool weighted = false, symmetric = false, has_csc = false;
    double weight_sum = 0.0;  // for the SSSP delta heuristic (hybrid_sssp.cu:184-197)
    void *arena = nullptr;
    size_t arena_bytes = 0;
    uint32_t *row = nullptr, *col = nullptr, *w = nullptr;
    uint32_t *crow = nullptr, *ccol = nullptr, *cw = nullptr;
};

namespace sgb {
// Scratch of single-query calls on g: the context's, grow-only and shared by
// all its graphs (work of a context is ordered on its stream), so creating
// another graph allocates no new scratch.
inline Workspace &graph_ws(sg_graph *g) {
    if (!g->ctx->graph_ws) g->ctx->graph_ws = new Workspace(&g->ctx->stream, device_pool(g->ctx->device));
    return *g->ctx->graph_ws;
}
}  // namespace sgb

namespace sgb {

inline sg_status set_error(sg_ctx *ctx, sg_status st, const char *fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        ctx->last_error = buf;
    }
    return st;
}

inline sg_status cuda_status(sg_ctx *ctx, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return SG_OK;
    set_error(ctx, e == cudaErrorMemoryAllocation ? SG_ERR_OUT_OF_MEMORY : SG_ERR_CUDA, "%s: %s", what,
              cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? SG_ERR_OUT_OF_MEMORY : SG_ERR_CUDA;
}

#define SG_TRY_CUDA(ctx, call)                                       \
    do {                                                             \
        cudaError_t _e = (call);                                     \
        if (_e != cudaSuccess) return ::sgb::cuda_status(ctx, _e, #call); \
    } while (0)

inline sg_status device_error_status(uint32_t bits) {
    using namespace sepgraph::dev;
    if (bits & kErrTimeout) return SG_ERR_TIMEOUT;
    if (bits & (kErrCapacity | kErrChunkCapacity)) return SG_ERR_CAPACITY;
    if (bits & kErrOverflow) return SG_ERR_OVERFLOW;
    if (bits & kErrUnsupported) return SG_ERR_UNSUPPORTED;
    return SG_OK;
}

// Makes `dev` current for the guard's lifetime.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// Is `p` device memory of the context's device (output written in place)?
inline bool is_device_ptr(const void *p, int device) {
    if (!p) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == device;
}

// Engine launch description shared by the algorithm entry points.
struct EngineConfig {
    int scheme = 0;
    int forced = -1;
    int lb_push = sepgraph::engine::LB_FINE;
    int lb_pull = sepgraph::engine::LB_FINE;
    int priority = 0;
    int trace = 0;
    uint32_t max_iteration = 200;
    double alpha = 15, beta = 18, edge_factor = 1.0;
    unsigned long long prio_init_raw = 0, prio_step_raw = 0;
    double timeout_s = 30.0;
    int blocks_per_sm = 0;
    uint32_t heavy_degree = 32;  // out/in-degree above which a vertex is split into chunks
    uint32_t chunk_edges = 256;
    uint32_t local_depth = 0;  // local lookahead levels in push rounds (0 = off)
    float sample_cut = 0.f;    // sampling priority cut in ASYNC_PUSH_TD rounds (0 = off)
    bool wl_sort = false;      // sort each data-driven push round's worklist by vertex id (--wl_sort)
    int worklist = 0;          // SG_WORKLIST_* (forced push DD: queues or bitmaps)
    int l2_persist = 0;        // sg_options.l2_persist: >= 0 = persistence window on the random-access array
    int pull_scan = 0;         // sg_options.pull_scan (SG_PULL_SCAN_WARP = warp-cooperative pull)
    int hub_stage = 0;         // sg_options.hub_stage (>= 0: bulk-copy staging of 256-edge hub chunks)
    bool blocking = true;
    sg_round_trace *trace_out = nullptr;
    uint32_t trace_cap = 0;
};

struct EngineResult {
    sepgraph::engine::Ctrl ctrl{};
    float ms = 0.f;
    uint32_t grid_blocks = 0;
    uint32_t device_error() const { return ctrl.error | ctrl.cnt.error; }
};

// ---------------------------------------------------------------- L2 persistence
// The persisting-L2 set-aside of a device (cudaLimitPersistingL2CacheSize) is
// raised to the device's maximum by the first context that launches with a
// persistence window and put back, with the persisting lines reset to normal,
// when the last such context of the device is destroyed.
struct PersistState {
    std::mutex mu;
    int users = 0;
    bool changed = false;
    size_t prev = 0;
};
inline PersistState &persist_state(int dev) {
    static PersistState st[64];
    return st[dev & 63];
}
inline void persist_acquire(sg_ctx *ctx) {
    if (ctx->persist_ref || ctx->prop.persistingL2CacheMaxSize <= 0 || ctx->prop.accessPolicyMaxWindowSize <= 0) return;
    PersistState &st = persist_state(ctx->device);
    std::lock_guard<std::mutex> lk(st.mu);
    if (st.users == 0) {
        size_t cur = 0;
        if (cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        const size_t want = (size_t)ctx->prop.persistingL2CacheMaxSize;
        if (cur < want) {
            if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) != cudaSuccess) {
                cudaGetLastError();
                return;
            }
            st.changed = true;
            st.prev = cur;
        }
    }
    st.users++;
    ctx->persist_ref = true;
}
inline void persist_release(sg_ctx *ctx) {
    if (!ctx->persist_ref) return;
    PersistState &st = persist_state(ctx->device);
    std::lock_guard<std::mutex> lk(st.mu);
    if (--st.users == 0 && st.changed) {
        cudaCtxResetPersistingL2Cache();
        cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, st.prev);
        cudaGetLastError();
        st.changed = false;
    }
    ctx->persist_ref = false;
}
// Access-policy window for the launches made while it lives: `bytes` from
// `base` marked persisting (as far as the set-aside reaches), then the
// stream's previous window restored.
struct PersistWindow {
    cudaStream_t s = nullptr;
    cudaStreamAttrValue old{};
    bool set = false;
    PersistWindow(sg_ctx *ctx, const void *base, size_t bytes) {
        if (!ctx->persist_ref || !base || bytes == 0) return;
        if (cudaStreamGetAttribute(ctx->stream, cudaStreamAttributeAccessPolicyWindow, &old) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        size_t lim = 0;
        if (cudaDeviceGetLimit(&lim, cudaLimitPersistingL2CacheSize) != cudaSuccess || lim == 0) {
            cudaGetLastError();
            return;
        }
        cudaStreamAttrValue v{};
        v.accessPolicyWindow.base_ptr = const_cast<void *>(base);
        v.accessPolicyWindow.num_bytes = std::min(bytes, (size_t)ctx->prop.accessPolicyMaxWindowSize);
        v.accessPolicyWindow.hitRatio = (float)std::min(1.0, (double)lim / (double)v.accessPolicyWindow.num_bytes);
        v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        if (cudaStreamSetAttribute(ctx->stream, cudaStreamAttributeAccessPolicyWindow, &v) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        s = ctx->stream;
        set = true;
    }
    ~PersistWindow() {
        if (set && cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &old) != cudaSuccess)
            cudaGetLastError();
    }
    PersistWindow(const PersistWindow &) = delete;
    PersistWindow &operator=(const PersistWindow &) = delete;
};

// Resident blocks per SM of `kernel` at `threads` threads per block, computed
// on first use and cached in `cache` (one per kernel, shared by the server's
// worker threads).
inline cudaError_t occupancy_once(std::atomic<int> &cache, const void *kernel, int threads, int *out) {
    int v = cache.load(std::memory_order_relaxed);
    if (v == 0) {
        const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kernel, threads, 0);
        if (e != cudaSuccess) return e;
        cache.store(v, std::memory_order_relaxed);
    }
    *out = v;
    return cudaSuccess;
}

// Blocks per SM a launch on ctx may take of a kernel that fits max_bps per SM:
// max_bps / ctx->resident_share (at least 1).  Any set of launches from
// resident_share such contexts then needs at most the SM's registers, shared
// memory and threads, so their grids are resident together.
inline int resident_blocks_per_sm(const sg_ctx *ctx, int max_bps) {
    return std::max(1, max_bps / (int)std::max(1u, ctx->resident_share));
}

// Resident blocks per SM of the multi-source kernels (BFS masks, BC lanes)
// when the caller does not choose: sparse high-diameter graphs are bound by
// the per-level barrier (fewer blocks), large dense ones by memory latency
// (more).  Measured on B200: 16 BFS on the 4096^2 grid 197 / 229 / 288 ms with
// 2 / 4 / 6 blocks; 64 BFS and 32 BC on symmetric RMAT-22 9.4 -> 8.2 and
// 23.3 -> 21.1 ms from 4 to 6; RMAT-16 best with 4.  On a sparse graph a
// round's work grows with the sources times the wavefront (about sqrt(V) on
// a grid), and a large one fills more blocks: push-only multi-source BFS, 64
// sources on the 4096^2 grid 1030 / 650 / 521 / 462 ms with 1 / 2 / 3 / 4
// blocks, on the 2048^2 grid 119 / 80 / 78 / 75 ms; 16 sources there 137 /
// 126 / 135 / 149 ms and 39 / 42 / 48 / 54 ms.
inline int ms_blocks_per_sm(uint32_t nv, uint64_t ne, uint32_t nsrc) {
    const double avg_deg = nv ? (double)ne / nv : 0.0;
    if (avg_deg < 8) return (double)nsrc * std::sqrt((double)nv) >= 131072.0 ? 4 : 2;
    return ne >= (1ull << 25) ? 6 : 4;
}

// Resident blocks per SM when the caller does not choose: small graphs are
// bound by per-round barrier latency, which grows with the number of blocks.
inline int auto_blocks_per_sm(uint32_t nv, uint64_t ne) {
    if (ne < (1ull << 22)) return 2;
    if (ne < (1ull << 25)) return 4;
    return 8;
}

inline cudaError_t pinned(sg_ctx *ctx, size_t bytes, void **out) {
    if (ctx->pinned_bytes < bytes) {
        if (ctx->pinned) cudaFreeHost(ctx->pinned);
        ctx->pinned = nullptr;
        ctx->pinned_bytes = 0;
        cudaError_t e = cudaMallocHost(&ctx->pinned, bytes);
        if (e != cudaSuccess) return e;
        ctx->pinned_bytes = bytes;
    }
    *out = ctx->pinned;
    return cudaSuccess;
}

// Runs the engine for functor `app` on graph `g`.  `value` and `buffer` are
// device arrays of nv elements (value may be the caller's output buffer).
template <typename App, typename TV, typename TB, typename TW>
sg_status run_engine(sg_graph *g, App app, const EngineConfig &cfg, TV *value, TB *buffer, EngineResult *res) {
    using namespace sepgraph::engine;
    sg_ctx *ctx = g->ctx;
    const uint32_t nv = g->nv;
    const uint64_t ne = g->ne;
    KArgs<TV, TB, TW> a;
    std::memset(&a, 0, sizeof a);
    a.csr.nnodes = nv;
    a.csr.nedges = (uint32_t)ne;
    a.csr.row_start = g->row;
    a.csr.edge_dst = g->col;
    a.csr.edge_weights = g->w;
    a.csc.nnodes = nv;
    a.csc.nedges = (uint32_t)ne;
    a.csc.col_start = g->crow;
    a.csc.edge_source = g->ccol;
    a.csc.edge_weights = g->cw;
    a.csc.csr_row_start = g->row;
    a.csr_w = g->w;
    a.csc_w = g->cw;
    a.value = value;
    a.buffer = buffer;

    const uint32_t nwords = (nv + 31) / 32 + 1;
    // A warp task is 32 light vertices (<= heavy_threshold edges each) or one
    // chunk of a heavy vertex (<= chunk_edges), which bounds the slowest warp
    // of a round.  Each vertex is registered at most once per round, so the
    // tables are bounded by the vertices above the threshold; there are two
    // tables, one per round parity (a push round's chunks may run at the start
    // of the next round while that round registers its own).
    const uint32_t heavy_threshold = std::max<uint32_t>(1, cfg.heavy_degree);
    // a multiple of 4: chunks start on 16-byte boundaries of the edge arrays
    const uint32_t chunk_edges = (std::max<uint32_t>(32, cfg.chunk_edges) + 3u) & ~3u;
    const uint32_t heavy_cap = (uint32_t)std::min<uint64_t>(nv, ne / heavy_threshold) + 2;
    // chunks are cut on the 4-edge grid (chunk_span): at most two more per
    // heavy vertex than its degree / chunk_edges
    const uint32_t chunk_cap = (uint32_t)(ne / chunk_edges + 2ull * heavy_cap + 2);
    auto &ws = sgb::graph_ws(g);
    SG_TRY_CUDA(ctx, ws.get("tmp", nv, &a.tmp));
    SG_TRY_CUDA(ctx, ws.get("q0", nv, &a.queue[0]));
    SG_TRY_CUDA(ctx, ws.get("q1", nv, &a.queue[1]));
    SG_TRY_CUDA(ctx, ws.get("q2", nv, &a.queue[2]));
    SG_TRY_CUDA(ctx, ws.get("bm0", nwords, &a.bitmap[0]));
    SG_TRY_CUDA(ctx, ws.get("bm1", nwords, &a.bitmap[1]));
    SG_TRY_CUDA(ctx, ws.get("fl0", nwords, &a.qflag[0]));
    SG_TRY_CUDA(ctx, ws.get("fl1", nwords, &a.qflag[1]));
    SG_TRY_CUDA(ctx, ws.get("fl2", nwords, &a.qflag[2]));
    SG_TRY_CUDA(ctx, ws.get("middle", nv, &a.middle));
    SG_TRY_CUDA(ctx, ws.get("heavy", 2ull * heavy_cap, &a.heavy, true));
    SG_TRY_CUDA(ctx, ws.get("chunk", 2ull * chunk_cap, &a.chunk_owner, true));
    SG_TRY_CUDA(ctx, ws.get("ctrl", 1, &a.ctrl));
    if (cfg.trace && cfg.trace_cap) SG_TRY_CUDA(ctx, ws.get("trace", cfg.trace_cap, &a.trace));
    a.queue_cap = nv;
    a.nwords = nwords;
    a.heavy_cap = heavy_cap;
    a.chunk_cap = chunk_cap;
    a.trace_cap = cfg.trace ? cfg.trace_cap : 0;

    Params &p = a.p;
    p.scheme = cfg.scheme;
    p.forced = cfg.forced;
    p.lb_push = cfg.lb_push;
    p.lb_pull = cfg.lb_pull;
    p.priority = cfg.priority;
    p.trace = cfg.trace;
    p.collect = (cfg.forced < 0 || cfg.trace) ? 1 : 0;
    p.has_csc = g->has_csc;
    p.max_iteration = cfg.max_iteration ? cfg.max_iteration : 200;
    p.heavy_threshold = heavy_threshold;
    p.chunk_edges = chunk_edges;
    p.pull_warp_threshold = 32;
    p.local_depth = cfg.local_depth;
    p.sample_cut = cfg.sample_cut;
    p.bitmap_frontier = use_bitmap_frontier(cfg.forced, cfg.lb_push, cfg.wl_sort, cfg.worklist);
    p.pull_coop = cfg.pull_scan == SG_PULL_SCAN_WARP;
    p.stage_chunks = cfg.hub_stage >= 0;
    p.alpha = cfg.alpha;
    p.beta = cfg.beta;
    p.total_workload0 = (long long)((double)ne * cfg.edge_factor);
    p.prio_init_raw = cfg.prio_init_raw;
    p.prio_step_raw = cfg.prio_step_raw;
    p.timeout_ns = (unsigned long long)((cfg.timeout_s > 0 ? cfg.timeout_s : 30.0) * 1e9);

    // the functor sees the graph like AppBase members are set in Engine::InitGraph (framework.cuh:162-166)
    app.m_csr_graph = a.csr;
    app.m_csc_graph = a.csc;
    app.m_nnodes = nv;
    app.m_nedges = (uint32_t)ne;
    app.m_p_current_round = &a.ctrl->rs.round;

    auto kernel = hybrid_engine_kernel<App, TV, TB, TW>;
    static std::atomic<int> occupancy{0};  // one per template instantiation
    int max_blocks_per_sm = 0;
    SG_TRY_CUDA(ctx, occupancy_once(occupancy, (const void *)kernel, kBlockThreads, &max_blocks_per_sm));
    if (max_blocks_per_sm <= 0) return set_error(ctx, SG_ERR_NO_DEVICE, "engine kernel cannot be resident");
    int bps = cfg.blocks_per_sm > 0 ? cfg.blocks_per_sm : auto_blocks_per_sm(nv, ne);
    bps = std::max(1, std::min(bps, resident_blocks_per_sm(ctx, max_blocks_per_sm)));
    dim3 grid(ctx->prop.multiProcessorCount * bps), block(kBlockThreads);
    res->grid_blocks = grid.x;
    if (cfg.wl_sort) SG_TRY_CUDA(ctx, ws.get("sort", grid.x, &a.sort_counts));
    // edge-tiled topology-driven pull (functors with PullReduce): a row index per
    // 256 in-edges, found once at the launch's start
    if constexpr (has_pull_reduce<App, TB>::value && std::is_same<TW, sepgraph::graphs::NoWeight>::value) {
        const bool td_pull = cfg.forced < 0 || cfg.forced == V_SYNC_PULL_TD;
        if (g->has_csc && td_pull && cfg.lb_pull != LB_NONE && nv > 0)
            SG_TRY_CUDA(ctx, ws.get("pull_tiles", (ne + kPullTileEdges - 1) / kPullTileEdges + 1, &a.tile_row));
    }

    SG_TRY_CUDA(ctx, cudaMemsetAsync(a.ctrl, 0, sizeof(Ctrl), ctx->stream));
    SG_TRY_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    void *args[] = {(void *)&app, (void *)&a};
    {
        // the array the rounds touch at random stays in L2 while the graph arrays stream past it:
        // the pulled values of a topology-driven pull, the tentative values otherwise
        if (cfg.l2_persist >= 0) persist_acquire(ctx);
        const bool td_pull = cfg.forced == V_SYNC_PULL_TD && a.tile_row;
        PersistWindow pw(ctx, td_pull ? (const void *)a.tmp : (const void *)a.buffer,
                         cfg.l2_persist >= 0 ? sizeof(TB) * (size_t)nv : 0);
        SG_TRY_CUDA(ctx, cudaLaunchCooperativeKernel((const void *)kernel, grid, block, args, 0, ctx->stream));
    }
    SG_TRY_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    if (!cfg.blocking) return SG_OK;

    void *h = nullptr;
    SG_TRY_CUDA(ctx, pinned(ctx, sizeof(Ctrl) + sizeof(sg_round_trace) * a.trace_cap, &h));
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(h, a.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, ctx->stream));
    if (a.trace_cap)
        SG_TRY_CUDA(ctx, cudaMemcpyAsync((char *)h + sizeof(Ctrl), a.trace, sizeof(sg_round_trace) * a.trace_cap,
                                         cudaMemcpyDeviceToHost, ctx->stream));
    SG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::memcpy(&res->ctrl, h, sizeof(Ctrl));
    if (a.trace_cap && cfg.trace_out)
        std::memcpy(cfg.trace_out, (char *)h + sizeof(Ctrl),
                    sizeof(sg_round_trace) * std::min<uint32_t>(res->ctrl.n_trace, cfg.trace_cap));
    SG_TRY_CUDA(ctx, cudaEventElapsedTime(&res->ms, ctx->ev0, ctx->ev1));
    const sg_status st = device_error_status(res->device_error());
    if (st != SG_OK) return set_error(ctx, st, "device error bits 0x%x", res->device_error());
    return SG_OK;
}



inline void fill_stats(sg_stats *s, const EngineResult &r) {
    if (!s) return;
    s->rounds = r.ctrl.round;
    s->max_iteration_reached = r.ctrl.max_iteration_reached;
    for (int i = 0; i < 8; ++i) s->rounds_by_variant[i] = r.ctrl.rounds_by_variant[i];
    s->time_kernel_ms = r.ms;
    s->time_total_ms = r.ms;
    s->edges_processed = r.ctrl.cnt.edges_processed;
    s->vertices_processed = r.ctrl.vertices_processed;
    s->device_error = r.device_error();
    s->n_trace = s->trace ? std::min<uint32_t>(r.ctrl.n_trace, s->trace_capacity) : 0;
}

}  // namespace sgb

// ---------------------------------------------------------------- Engine
// C++ mirror of the reference's Engine for custom functors.  Same lifecycle:
// Engine(AlgoType) -> SetOptions -> LoadGraph -> InitGraph(data...) -> Start ->
// GatherValue / GatherBuffer / PrintInfo.  LoadGraph takes the device graph
// (the reference reads the graph named by --graphfile, framework.cuh:99-133).
namespace sepgraph {
namespace engine {

template <typename TValue, typename TBuffer, typename TWeight,
          template <typename, typename, typename, typename...> class TAppImpl, typename... UnusedData>
class Engine {
    using AppImpl = TAppImpl<TValue, TBuffer, TWeight, UnusedData...>;
    policy::AlgoType m_algo_type;
    common::EngineOptions m_opt;
    sg_graph *m_graph = nullptr;
    std::unique_ptr<AppImpl> m_app;
    TValue *m_value = nullptr;
    TBuffer *m_buffer = nullptr;
    std::vector<TValue> m_value_host;
    std::vector<TBuffer> m_buffer_host;
    sgb::EngineResult m_res;
    sg_status m_status = SG_OK;

   public:
    int max_iteration = 200;
    double alpha = 15, beta = 18, edge_factor = 1.0;

    explicit Engine(policy::AlgoType algo_type) : m_algo_type(algo_type) {}
    void SetOptions(common::EngineOptions &o) { m_opt = o; }
    void LoadGraph(sg_graph *g) { m_graph = g; }
    void InitGraph(UnusedData &...data) { m_app.reset(new AppImpl(data...)); }

    sg_status Start() {
        if (!m_graph || !m_app) return SG_ERR_INVALID_ARG;
        auto &ws = sgb::graph_ws(m_graph);
        if (ws.get("engine_value", m_graph->nv, &m_value) != cudaSuccess ||
            ws.get("engine_buffer", m_graph->nv, &m_buffer) != cudaSuccess)
            return SG_ERR_OUT_OF_MEMORY;
        sgb::EngineConfig cfg;
        cfg.scheme = m_algo_type == policy::AlgoType::TRAVERSAL_SCHEME ? 0 : 1;
        cfg.forced = m_opt.IsForceVariant() ? m_opt.GetAlgoVariant().Id() : -1;
        const double avg_deg = m_graph->nv ? (double)m_graph->ne / m_graph->nv : 0;
        cfg.lb_push = m_opt.IsForceLoadBalancing(common::MsgPassing::PUSH)
                          ? (int)m_opt.GetLoadBalancing(common::MsgPassing::PUSH)
                          : (avg_deg >= 5 ? LB_FINE : LB_NONE);  // LoadOptions (framework.cuh:402-443)
        cfg.lb_pull = m_opt.IsForceLoadBalancing(common::MsgPassing::PULL)
                          ? (int)m_opt.GetLoadBalancing(common::MsgPassing::PULL)
                          : (avg_deg >= 5 ? LB_FINE : LB_NONE);
        cfg.priority = m_opt.GetPriorityType() == common::Priority::LOW_HIGH;
        if (m_opt.GetPriorityType() == common::Priority::SAMPLING) cfg.sample_cut = (float)m_opt.GetCutThreshold();
        cfg.prio_init_raw = to_raw<TBuffer>((TBuffer)m_opt.GetPriorityThreshold());
        cfg.prio_step_raw = cfg.prio_init_raw;
        cfg.max_iteration = max_iteration;
        cfg.alpha = alpha;
        cfg.beta = beta;
        cfg.edge_factor = edge_factor;
        if (alpha == 0) cfg.forced = V_ASYNC_PUSH_DD;
        m_status = sgb::run_engine<AppImpl, TValue, TBuffer, TWeight>(m_graph, *m_app, cfg, m_value, m_buffer, &m_res);
        return m_status;
    }
    // GatherValue / GatherBuffer (framework.cuh:385-391): copied on the engine's
    // stream (the graph's context stream), after the launch it ordered.
    const std::vector<TValue> &GatherValue() {
        m_value_host.resize(m_graph->nv);
        gather(m_value_host.data(), m_value, sizeof(TValue));
        return m_value_host;
    }
    const std::vector<TBuffer> &GatherBuffer() {
        m_buffer_host.resize(m_graph->nv);
        gather(m_buffer_host.data(), m_buffer, sizeof(TBuffer));
        return m_buffer_host;
    }
    cudaStream_t getStream() const { return m_graph ? m_graph->ctx->stream : nullptr; }
    void PrintInfo() const {
        std::printf("Kernel time: %f\nTotal rounds: %u\n", m_res.ms, m_res.ctrl.round);
        for (int v = 0; v < 8; ++v)
            if (m_res.ctrl.rounds_by_variant[v])
                std::printf("  %s rounds: %u\n", common::AlgoVariant::FromId(v).ToString().c_str(),
                            m_res.ctrl.rounds_by_variant[v]);
    }
    const sgb::EngineResult &Result() const { return m_res; }

   private:
    void gather(void *dst, const void *src, size_t elem) {
        if (!m_graph || !src) return;
        cudaStream_t s = m_graph->ctx->stream;
        if (cudaMemcpyAsync(dst, src, elem * m_graph->nv, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            m_status = SG_ERR_CUDA;
    }
};

}  // namespace engine
}  // namespace sepgraph
