// C ABI of libsepgraph_b200 (declarations and reference citations in
// include/sepgraph.h).  Instantiates the engine for the four reference
// algorithms and adds the BC backward pass and small reduction kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "host/sg_hgraph.h"
#include "sg_apps.cuh"
#include "sg_bc.cuh"
#include "sg_runtime.cuh"

using namespace sepgraph;
using sgb::set_error;

namespace {

using sgb::DeviceGuard;

// Checks an uploaded CSR (offsets start at 0, end at ne and never decrease;
// every index < nv) and sums the weights, so that a graph whose edges need no
// host-side work never goes through a host loop.
struct CsrCheck {
    uint32_t ends_bad, first_bad_offset;
    unsigned long long first_bad_edge;
    double weight_sum;  // exact: at most 2^32 weights below 2^32
};

__global__ void validate_csr_kernel(const uint32_t *row, const uint32_t *col, const uint32_t *w, uint32_t nv,
                                    unsigned long long ne, CsrCheck *chk) {
    const unsigned long long tid = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    const unsigned long long nt = (unsigned long long)gridDim.x * blockDim.x;
    if (tid == 0 && (row[0] != 0 || row[nv] != ne)) chk->ends_bad = 1;
    for (unsigned long long v = tid; v < nv; v += nt)
        if (__ldg(row + v + 1) < __ldg(row + v)) atomicMin(&chk->first_bad_offset, (uint32_t)v);
    double sum = 0;
    for (unsigned long long e = tid; e < ne; e += nt) {
        if (__ldg(col + e) >= nv) atomicMin(&chk->first_bad_edge, e);
        if (w) sum += __ldg(w + e);
    }
    sum = dev::warp_sum(sum);
    if (w && dev::lane_id() == 0 && sum != 0) atomicAdd(&chk->weight_sum, sum);
}

// Sum of out-degrees and count of vertices whose value differs from `unreached`
// (GTEPS numerator over the reached component), plus the maximum finite value.
__global__ void reached_stats_kernel(const uint32_t *row, const uint32_t *value, uint32_t nv, uint32_t unreached,
                                     unsigned long long *out /* [edges, vertices, max] */) {
    unsigned long long e = 0, n = 0;
    uint32_t mx = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const uint32_t x = value[v];
        if (x != unreached) {
            e += __ldg(row + v + 1) - __ldg(row + v);
            n += 1;
            mx = max(mx, x);
        }
    }
    e = dev::warp_sum(e);
    n = dev::warp_sum(n);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) mx = max(mx, __shfl_xor_sync(dev::kFullMask, mx, d));
    if ((threadIdx.x & 31) == 0) {
        if (e) atomicAdd(out, e);
        if (n) atomicAdd(out + 1, n);
        if (mx) atomicMax(out + 2, (unsigned long long)mx);
    }
}

// ---------------------------------------------------------------- BC backward
// One query over the whole cooperative grid (sg_bc.cuh has the pass itself).
using bc::BCBackArgs;
using bc::kBcBigDegree;
using bc::kBcChunk;

__global__ void __launch_bounds__(256) bc_backward_kernel(BCBackArgs a) {
    auto sync = [&] { return dev::grid_barrier(a.bar, a.bar + 1, a.err, a.timeout_ns, [] {}); };
    bc::backward(a, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, sync);
}

__global__ void bc_scale_kernel(const float *delta, float *out, uint32_t nv) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
        out[v] = delta[v] * 0.5f;
}

sg_options default_options() {
    sg_options o;
    std::memset(&o, 0, sizeof o);
    o.variant = SG_VARIANT_AUTO;
    o.lb_push = SG_LB_AUTO;
    o.lb_pull = SG_LB_AUTO;
    o.priority = SG_PRIORITY_NONE;
    o.priority_delta = 0;
    o.cut_threshold = 0;
    o.alpha = 15;
    o.beta = 18;
    o.edge_factor = 1.0;
    o.max_iteration = 200;
    o.fused = 0;
    o.block_size = 0;
    o.non_atomic = 1;
    o.trace = 0;
    o.pr_error = 0.01;
    o.timeout_s = 30.0;
    o.blocking = 1;
    return o;
}

sgb::EngineConfig make_config(const sg_graph *g, const sg_options &o, int scheme, int default_lb_pull,
                              sg_stats *stats) {
    sgb::EngineConfig c;
    c.scheme = scheme;
    c.forced = o.variant;
    const double avg_deg = g->nv ? (double)g->ne / g->nv : 0;
    // LoadOptions (framework.cuh:402-443): average degree >= 5 selects FINE_GRAINED
    c.lb_push = o.lb_push >= 0 ? o.lb_push : (avg_deg >= 5 ? engine::LB_FINE : engine::LB_NONE);
    c.lb_pull = o.lb_pull >= 0 ? o.lb_pull : default_lb_pull;
    c.max_iteration = o.max_iteration > 0 ? (uint32_t)o.max_iteration : 200u;
    c.alpha = o.alpha;
    c.beta = o.beta > 0 ? o.beta : 18;
    c.edge_factor = o.edge_factor;
    if (o.alpha == 0) c.forced = engine::V_ASYNC_PUSH_DD;  // framework.cuh:445-448
    c.timeout_s = o.timeout_s;
    c.blocks_per_sm = o.blocks_per_sm;
    if (o.heavy_degree > 0) c.heavy_degree = (uint32_t)o.heavy_degree;
    if (o.chunk_edges > 0) c.chunk_edges = (uint32_t)o.chunk_edges;
    if (o.local_depth > 0) c.local_depth = (uint32_t)o.local_depth;
    c.wl_sort = o.wl_sort != 0;
    c.worklist = o.worklist;
    c.l2_persist = o.l2_persist;
    c.pull_scan = o.pull_scan;
    c.hub_stage = o.hub_stage;
    // SetSampleBasedPriority (common.h:229-233; hybrid_pr.cu:135-137 sets it when --cut_threshold > 0)
    if (o.priority == SG_PRIORITY_SAMPLING && o.cut_threshold > 0) c.sample_cut = (float)std::min(o.cut_threshold, 1.0);
    c.blocking = o.blocking != 0;
    if (o.trace && stats && stats->trace && stats->trace_capacity) {
        c.trace = 1;
        c.trace_out = stats->trace;
        c.trace_cap = stats->trace_capacity;
    } else if (o.trace) {
        c.trace = 1;
    }
    return c;
}

sg_status check_graph(sg_graph *g) {
    if (!g || !g->ctx) return SG_ERR_INVALID_ARG;
    return SG_OK;
}

// Copies a device result to the caller's buffer when it is not device memory.
template <typename T>
sg_status deliver(sg_ctx *ctx, T *out, const T *dev_src, uint32_t n, bool out_is_dev) {
    if (!out || out_is_dev) return SG_OK;
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(out, dev_src, sizeof(T) * n, cudaMemcpyDeviceToHost, ctx->stream));
    return SG_OK;
}

sg_status reached_stats(sg_graph *g, const uint32_t *value, sg_stats *stats) {
    if (!stats) return SG_OK;
    sg_ctx *ctx = g->ctx;
    unsigned long long *d = nullptr;
    SG_TRY_CUDA(ctx, sgb::graph_ws(g).get("reach_stats", 3, &d));
    SG_TRY_CUDA(ctx, cudaMemsetAsync(d, 0, 3 * sizeof(unsigned long long), ctx->stream));
    const int blocks = std::max(1, std::min<int>((g->nv + 255) / 256, ctx->prop.multiProcessorCount * 8));
    reached_stats_kernel<<<blocks, 256, 0, ctx->stream>>>(g->row, value, g->nv, apps::kInf, d);
    SG_TRY_CUDA(ctx, cudaGetLastError());
    unsigned long long h[3];
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    SG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    stats->edges_reached = h[0];
    stats->vertices_reached = (uint32_t)h[1];
    stats->search_depth = (uint32_t)h[2];
    return SG_OK;
}

sg_status finish(sg_ctx *ctx, sg_status st, const sgb::EngineResult &res, const sgb::EngineConfig &cfg,
                 sg_stats *stats) {
    if (!cfg.blocking) return st;
    if (stats) sgb::fill_stats(stats, res);
    return st;
}

}  // namespace

extern "C" {

const char *sg_status_string(sg_status s) {
    switch (s) {
        case SG_OK: return "ok";
        case SG_ERR_INVALID_ARG: return "invalid argument";
        case SG_ERR_CUDA: return "CUDA error";
        case SG_ERR_OUT_OF_MEMORY: return "out of memory";
        case SG_ERR_TIMEOUT: return "device wait timed out";
        case SG_ERR_CAPACITY: return "worklist capacity exceeded";
        case SG_ERR_UNSUPPORTED: return "unsupported variant";
        case SG_ERR_OVERFLOW: return "path count overflow";
        case SG_ERR_NO_DEVICE: return "no usable CUDA device";
        case SG_ERR_IO: return "I/O error";
        case SG_ERR_FORMAT: return "malformed graph file";
        case SG_ERR_BUSY: return "busy";
    }
    return "unknown status";
}

int sg_abi_version(void) { return SG_ABI_VERSION; }

sg_status sg_init(int device, sg_ctx **out) {
    if (!out) return SG_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return SG_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) return SG_ERR_INVALID_ARG;
    sg_ctx *ctx = new (std::nothrow) sg_ctx;
    if (!ctx) return SG_ERR_OUT_OF_MEMORY;
    ctx->device = device;
    DeviceGuard dg(device);
    int coop = 0;
    if (cudaGetDeviceProperties(&ctx->prop, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess || !coop ||
        cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return SG_ERR_NO_DEVICE;
    }
    ctx->stream = ctx->own_stream;
    *out = ctx;
    return SG_OK;
}

sg_status sg_destroy(sg_ctx *ctx) {
    if (!ctx) return SG_ERR_INVALID_ARG;
    if (ctx->live_graphs > 0)
        return set_error(ctx, SG_ERR_BUSY, "%d graph(s) of this context still exist", ctx->live_graphs);
    DeviceGuard dg(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    sgb::persist_release(ctx);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    if (ctx->spare_arena) cudaFree(ctx->spare_arena);
    delete ctx->batch_ws;  // frees on the context's stream and waits for it
    delete ctx->graph_ws;
    if (cudaMemPool_t pool = sgb::device_pool(ctx->device)) cudaMemPoolTrimTo(pool, 0);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return SG_OK;
}

sg_status sg_ctx_set_stream(sg_ctx *ctx, void *s) {
    if (!ctx) return SG_ERR_INVALID_ARG;
    // the context's scratch is freed and reused in the order of its stream:
    // work queued on the old stream ends before the new one can reuse it
    cudaStreamSynchronize(ctx->stream);
    ctx->stream = s ? (cudaStream_t)s : ctx->own_stream;
    return SG_OK;
}

sg_status sg_ctx_get_stream(sg_ctx *ctx, void **s) {
    if (!ctx || !s) return SG_ERR_INVALID_ARG;
    *s = (void *)ctx->stream;
    return SG_OK;
}

sg_status sg_ctx_synchronize(sg_ctx *ctx) {
    if (!ctx) return SG_ERR_INVALID_ARG;
    DeviceGuard dg(ctx->device);
    SG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SG_OK;
}

const char *sg_last_error(const sg_ctx *ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

sg_status sg_device_info(sg_ctx *ctx, int *sm_count, uint64_t *hbm_bytes, uint64_t *l2_bytes, char *name,
                         size_t name_len) {
    if (!ctx) return SG_ERR_INVALID_ARG;
    if (sm_count) *sm_count = ctx->prop.multiProcessorCount;
    if (hbm_bytes) *hbm_bytes = ctx->prop.totalGlobalMem;
    if (l2_bytes) *l2_bytes = ctx->prop.l2CacheSize;
    if (name && name_len) {
        std::strncpy(name, ctx->prop.name, name_len - 1);
        name[name_len - 1] = 0;
    }
    return SG_OK;
}

sg_status sg_options_default(sg_options *opt) {
    if (!opt) return SG_ERR_INVALID_ARG;
    *opt = default_options();
    return SG_OK;
}

}  // extern "C"

namespace sgb {

// Every graph is uploaded as it is (host or device inputs, one copy each),
// checked on the device by one validation kernel, and gets its in-edge (CSC)
// view from the device transpose: no host loop over the edges.
sg_status create_graph(sg_ctx *ctx, uint32_t nv, uint64_t ne, const uint32_t *offsets, const uint32_t *indices,
                       const uint32_t *weights, uint32_t flags, sg_graph **out) {
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const bool has_csc = !(flags & SG_GRAPH_NO_CSC), symmetric = (flags & SG_GRAPH_SYMMETRIC) != 0;
    const bool full_csc = has_csc && !symmetric;
    const size_t b_row = al(4ull * (nv + 1)), b_col = al(4ull * std::max<uint64_t>(ne, 1));
    const size_t b_w = weights ? b_col : 0;
    const size_t b_csr = b_row + b_col + b_w;
    const size_t total = b_csr * (full_csc ? 2 : 1) + al(sizeof(CsrCheck));
    sg_graph *g = new (std::nothrow) sg_graph;
    if (!g) return SG_ERR_OUT_OF_MEMORY;
    g->ctx = ctx;
    g->nv = nv;
    g->ne = ne;
    g->weighted = weights != nullptr;
    g->symmetric = symmetric;
    g->has_csc = has_csc;
    cudaError_t e = cudaSuccess;
    if (ctx->spare_arena && ctx->spare_bytes >= total && ctx->spare_bytes / 2 <= total) {
        g->arena = ctx->spare_arena;  // stream-ordered after the released graph's work
        g->arena_bytes = ctx->spare_bytes;
        ctx->spare_arena = nullptr;
        ctx->spare_bytes = 0;
    } else {
        e = cudaMalloc(&g->arena, total);
        if (e != cudaSuccess) {
            delete g;
            return sgb::cuda_status(ctx, e, "graph arena");
        }
        g->arena_bytes = total;
    }
    char *p = (char *)g->arena;
    auto carve = [&](size_t bytes) {
        uint32_t *q = (uint32_t *)p;
        p += bytes;
        return q;
    };
    g->row = carve(b_row);
    g->col = carve(b_col);
    if (weights) g->w = carve(b_w);
    if (full_csc) {
        g->crow = carve(b_row);
        g->ccol = carve(b_col);
        if (weights) g->cw = carve(b_w);
    } else if (has_csc) {  // symmetric: CSC aliases CSR (csr_graph.h:405-410)
        g->crow = g->row;
        g->ccol = g->col;
        g->cw = g->w;
    }
    CsrCheck *dchk = (CsrCheck *)p;
    const cudaStream_t s = ctx->stream;
    CsrCheck hchk{0u, 0xffffffffu, ~0ull, 0.0};
    uint32_t bad_dst = 0;
    auto fail = [&](sg_status st) {
        cudaStreamSynchronize(s);
        cudaFree(g->arena);
        delete g;
        return st;
    };
    e = cudaMemcpyAsync(g->row, offsets, 4ull * (nv + 1), cudaMemcpyDefault, s);
    if (e == cudaSuccess && ne) e = cudaMemcpyAsync(g->col, indices, 4ull * ne, cudaMemcpyDefault, s);
    if (e == cudaSuccess && weights && ne) e = cudaMemcpyAsync(g->w, weights, 4ull * ne, cudaMemcpyDefault, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dchk, &hchk, sizeof hchk, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return fail(sgb::cuda_status(ctx, e, "graph upload"));
    const uint64_t work = std::max<uint64_t>(nv, ne);
    const unsigned blocks = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((work + 255) / 256, 148ull * 16));
    validate_csr_kernel<<<blocks, 256, 0, s>>>(g->row, g->col, g->w, nv, ne, dchk);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hchk, dchk, sizeof hchk, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(sgb::cuda_status(ctx, e, "graph check"));
    if (hchk.ends_bad) return fail(set_error(ctx, SG_ERR_INVALID_ARG, "offsets[0] must be 0 and offsets[nv] == ne"));
    if (hchk.first_bad_offset != 0xffffffffu)
        return fail(set_error(ctx, SG_ERR_INVALID_ARG, "offsets not monotone at %u", hchk.first_bad_offset));
    if (hchk.first_bad_edge != ~0ull) {
        cudaMemcpy(&bad_dst, g->col + hchk.first_bad_edge, 4, cudaMemcpyDeviceToHost);
        return fail(set_error(ctx, SG_ERR_INVALID_ARG, "edge %llu points to vertex %u >= nv", hchk.first_bad_edge, bad_dst));
    }
    g->weight_sum = weights ? hchk.weight_sum : (double)ne;
    sg_status st = SG_OK;
    if (full_csc) st = device_transpose(ctx, nv, ne, g->row, g->col, g->w, g->crow, g->ccol, g->cw);
    else if (has_csc && weights) st = symmetric_weighted_csc(ctx, g);
    if (st == SG_OK) st = sgb::cuda_status(ctx, cudaStreamSynchronize(s), "graph transpose");
    if (st != SG_OK) return fail(st);
    ctx->live_graphs++;
    *out = g;
    return SG_OK;
}

}  // namespace sgb

extern "C" {

sg_status sg_graph_create(sg_ctx *ctx, uint32_t nv, uint64_t ne, const uint32_t *offsets, const uint32_t *indices,
                          const uint32_t *weights, uint32_t flags, sg_graph **out) {
    if (!ctx || !out || !offsets || (ne && !indices) || nv == 0) return SG_ERR_INVALID_ARG;
    if (ne >= (1ull << 32)) return set_error(ctx, SG_ERR_INVALID_ARG, "edge count %llu exceeds uint32", (unsigned long long)ne);
    *out = nullptr;
    DeviceGuard dg(ctx->device);
    return sgb::create_graph(ctx, nv, ne, offsets, indices, weights, flags, out);
}

sg_status sg_graph_create_from_host(sg_ctx *ctx, const sg_hgraph *h, uint32_t flags, sg_graph **out) {
    if (!h) return SG_ERR_INVALID_ARG;
    return sg_graph_create(ctx, h->nv, h->ne, h->offsets.data(), h->indices.data(),
                           h->weights.empty() ? nullptr : h->weights.data(), flags, out);
}

sg_status sg_graph_destroy(sg_graph *g) {
    if (!g) return SG_ERR_INVALID_ARG;
    sg_ctx *ctx = g->ctx;
    DeviceGuard dg(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (g->arena) {
        // keep the larger of this arena and the context's spare for the next graph
        if (!ctx->spare_arena || ctx->spare_bytes < g->arena_bytes) {
            if (ctx->spare_arena) cudaFree(ctx->spare_arena);
            ctx->spare_arena = g->arena;
            ctx->spare_bytes = g->arena_bytes;
        } else {
            cudaFree(g->arena);
        }
    }
    ctx->live_graphs--;
    delete g;
    return SG_OK;
}

sg_status sg_ctx_release_cached(sg_ctx *ctx) {
    if (!ctx) return SG_ERR_INVALID_ARG;
    DeviceGuard dg(ctx->device);
    SG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->spare_arena) cudaFree(ctx->spare_arena);
    ctx->spare_arena = nullptr;
    ctx->spare_bytes = 0;
    delete ctx->graph_ws;
    ctx->graph_ws = nullptr;
    delete ctx->batch_ws;
    ctx->batch_ws = nullptr;
    return SG_OK;
}

}  // extern "C"

sg_ctx *sgb::graph_context(const sg_graph *g) { return g ? g->ctx : nullptr; }
double sgb::graph_weight_sum(const sg_graph *g) { return g ? g->weight_sum : 0.0; }

void sgb::set_resident_share(sg_ctx *ctx, uint32_t share) {
    if (ctx) ctx->resident_share = std::max(1u, share);
}

sg_graph *sgb::graph_view(sg_graph *g, sg_ctx *ctx) {
    if (!g || !ctx || g->ctx->device != ctx->device) return nullptr;
    sg_graph *v = new (std::nothrow) sg_graph;
    if (!v) return nullptr;
    v->ctx = ctx;
    v->nv = g->nv;
    v->ne = g->ne;
    v->weighted = g->weighted;
    v->symmetric = g->symmetric;
    v->has_csc = g->has_csc;
    v->weight_sum = g->weight_sum;
    v->arena = nullptr;  // the arrays stay owned by g
    v->row = g->row;
    v->col = g->col;
    v->w = g->w;
    v->crow = g->crow;
    v->ccol = g->ccol;
    v->cw = g->cw;
    return v;
}

void sgb::graph_view_destroy(sg_graph *view) {
    if (!view) return;
    DeviceGuard dg(view->ctx->device);
    cudaStreamSynchronize(view->ctx->stream);
    delete view;  // the arrays stay with the graph, the scratch with the context
}

extern "C" {

sg_status sg_graph_info(const sg_graph *g, uint32_t *nv, uint64_t *ne, uint64_t *device_bytes, int *weighted) {
    if (!g) return SG_ERR_INVALID_ARG;
    if (nv) *nv = g->nv;
    if (ne) *ne = g->ne;
    if (device_bytes) *device_bytes = g->arena_bytes;
    if (weighted) *weighted = g->weighted;
    return SG_OK;
}

sg_status sg_graph_copy_out(const sg_graph *g, int csc, uint32_t *offsets, uint32_t *indices, uint32_t *weights) {
    if (!g || !g->ctx) return SG_ERR_INVALID_ARG;
    sg_ctx *ctx = g->ctx;
    if (csc && !g->has_csc) return set_error(ctx, SG_ERR_UNSUPPORTED, "graph was created without a CSC view");
    if (weights && !g->weighted) return set_error(ctx, SG_ERR_INVALID_ARG, "graph has no weights");
    DeviceGuard dg(ctx->device);
    const uint32_t *row = csc ? g->crow : g->row, *col = csc ? g->ccol : g->col, *w = csc ? g->cw : g->w;
    SG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (offsets) SG_TRY_CUDA(ctx, cudaMemcpy(offsets, row, 4ull * (g->nv + 1), cudaMemcpyDefault));
    if (indices && g->ne) SG_TRY_CUDA(ctx, cudaMemcpy(indices, col, 4ull * g->ne, cudaMemcpyDefault));
    if (weights && g->ne) SG_TRY_CUDA(ctx, cudaMemcpy(weights, w, 4ull * g->ne, cudaMemcpyDefault));
    return SG_OK;
}

sg_status sg_bfs(sg_graph *g, uint32_t source, const sg_options *opt, uint32_t *levels_out, sg_stats *stats) {
    if (check_graph(g) != SG_OK || source >= g->nv) return SG_ERR_INVALID_ARG;
    sg_ctx *ctx = g->ctx;
    DeviceGuard dg(ctx->device);
    const sg_options o = opt ? *opt : default_options();
    sgb::EngineConfig cfg = make_config(g, o, 0, engine::LB_FINE, stats);
    const bool out_dev = sgb::is_device_ptr(levels_out, ctx->device);
    uint32_t *value = nullptr, *buffer = nullptr;
    if (out_dev)
        value = levels_out;
    else
        SG_TRY_CUDA(ctx, sgb::graph_ws(g).get("value_u32", g->nv, &value));
    SG_TRY_CUDA(ctx, sgb::graph_ws(g).get("buffer_u32", g->nv, &buffer));
    // local lookahead mixes levels inside a round, which needs the atomic minimum
    apps::BFS<uint32_t, uint32_t, graphs::NoWeight> app(source, o.non_atomic != 0 && o.local_depth <= 0);
    sgb::EngineResult res;
    sg_status st = sgb::run_engine<decltype(app), uint32_t, uint32_t, graphs::NoWeight>(g, app, cfg, value, buffer, &res);
    if (st == SG_OK) st = deliver(ctx, levels_out, value, g->nv, out_dev);
    if (st == SG_OK && cfg.blocking) st = reached_stats(g, value, stats);
    return finish(ctx, st, res, cfg, stats);
}

sg_status sg_sssp(sg_graph *g, uint32_t source, const sg_options *opt, uint32_t *dist_out, sg_stats *stats) {
    if (check_graph(g) != SG_OK || source >= g->nv) return SG_ERR_INVALID_ARG;
    sg_ctx *ctx = g->ctx;
    DeviceGuard dg(ctx->device);
    const sg_options o = opt ? *opt : default_options();
    sgb::EngineConfig cfg = make_config(g, o, 0, engine::LB_FINE, stats);
    if (o.priority == SG_PRIORITY_LOW_HIGH) {
        // Delta = 32 * avg weight / avg degree (hybrid_sssp.cu:184-197) unless given
        double delta = o.priority_delta;
        if (delta <= 0) {
            const double avg_w = g->ne ? g->weight_sum / (double)g->ne : 1.0;
            const double avg_d = g->nv ? (double)g->ne / (double)g->nv : 1.0;
            delta = std::floor(32.0 * avg_w / avg_d);
            if (delta < 1) delta = 1;
        }
        cfg.priority = 1;
        cfg.prio_init_raw = engine::to_raw<uint32_t>((uint32_t)delta);
        cfg.prio_step_raw = cfg.prio_init_raw;
        if (cfg.forced < 0) cfg.forced = engine::V_ASYNC_PUSH_DD;  // two-level priority runs push-only (--sparse)
        if (cfg.forced != engine::V_ASYNC_PUSH_DD)
            return set_error(ctx, SG_ERR_UNSUPPORTED, "two-level priority requires ASYNC_PUSH_DD");
    }
    const bool out_dev = sgb::is_device_ptr(dist_out, ctx->device);
    uint32_t *value = nullptr, *buffer = nullptr;
    if (out_dev)
        value = dist_out;
    else
        SG_TRY_CUDA(ctx, sgb::graph_ws(g).get("value_u32", g->nv, &value));
    SG_TRY_CUDA(ctx, sgb::graph_ws(g).get("buffer_u32", g->nv, &buffer));
    apps::SSSP<uint32_t, uint32_t, uint32_t> app(source);
    sgb::EngineResult res;
    sg_status st = sgb::run_engine<decltype(app), uint32_t, uint32_t, uint32_t>(g, app, cfg, value, buffer, &res);
    if (st == SG_OK) st = deliver(ctx, dist_out, value, g->nv, out_dev);
    if (st == SG_OK && cfg.blocking) st = reached_stats(g, value, stats);
    return finish(ctx, st, res, cfg, stats);
}

sg_status sg_pagerank(sg_graph *g, const sg_options *opt, float *ranks_out, float *residual_out, sg_stats *stats) {
    if (check_graph(g) != SG_OK) return SG_ERR_INVALID_ARG;
    sg_ctx *ctx = g->ctx;
    DeviceGuard dg(ctx->device);
    const sg_options o = opt ? *opt : default_options();
    sgb::EngineConfig cfg = make_config(g, o, 1, engine::LB_FINE, stats);
    const bool out_dev = sgb::is_device_ptr(ranks_out, ctx->device);
    const bool res_dev = sgb::is_device_ptr(residual_out, ctx->device);
    float *value = nullptr, *buffer = nullptr;
    if (out_dev)
        value = ranks_out;
    else
        SG_TRY_CUDA(ctx, sgb::graph_ws(g).get("value_f32", g->nv, &value));
    if (res_dev)
        buffer = residual_out;
    else
        SG_TRY_CUDA(ctx, sgb::graph_ws(g).get("buffer_f32", g->nv, &buffer));
    apps::PageRank<float, float, graphs::NoWeight> app(o.pr_error);
    sgb::EngineResult res;
    sg_status st = sgb::run_engine<decltype(app), float, float, graphs::NoWeight>(g, app, cfg, value, buffer, &res);
    if (st == SG_OK) st = deliver(ctx, ranks_out, value, g->nv, out_dev);
    if (st == SG_OK) st = deliver(ctx, residual_out, buffer, g->nv, res_dev);
    if (st == SG_OK && cfg.blocking) {
        SG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (stats) {
            stats->edges_reached = g->ne;
            stats->vertices_reached = g->nv;
        }
    }
    return finish(ctx, st, res, cfg, stats);
}

sg_status sg_bc(sg_graph *g, uint32_t source, const sg_options *opt, float *bc_out, uint64_t *sigma_out,
                sg_stats *stats) {
    if (check_graph(g) != SG_OK || source >= g->nv) return SG_ERR_INVALID_ARG;
    sg_ctx *ctx = g->ctx;
    DeviceGuard dg(ctx->device);
    const sg_options o = opt ? *opt : default_options();
    // HybridBC forces FINE_GRAINED for both directions (hybrid_bc.cu:335-336)
    sgb::EngineConfig cfg = make_config(g, o, 0, engine::LB_FINE, stats);
    if (o.lb_push < 0) cfg.lb_push = engine::LB_FINE;
    cfg.blocking = true;  // the backward pass needs the forward depth on the host
    const uint32_t nv = g->nv;
    const uint32_t max_levels = cfg.max_iteration + 2;
    uint32_t *level = nullptr, *buffer = nullptr, *stack = nullptr, *misc = nullptr, *ends = nullptr;
    unsigned long long *sigma = nullptr;
    float *delta = nullptr, *bcv = nullptr;
    const bool sig_dev = sgb::is_device_ptr(sigma_out, ctx->device);
    const bool bc_dev = sgb::is_device_ptr(bc_out, ctx->device);
    auto &ws = sgb::graph_ws(g);
    SG_TRY_CUDA(ctx, ws.get("value_u32", nv, &level));
    SG_TRY_CUDA(ctx, ws.get("buffer_u32", nv, &buffer));
    SG_TRY_CUDA(ctx, ws.get("bc_stack", nv, &stack));
    SG_TRY_CUDA(ctx, ws.get("bc_ends", max_levels, &ends));
    SG_TRY_CUDA(ctx, ws.get("bc_misc", 8, &misc));  // 0 count, 1 nlevels, 2 search depth, 3 err, 4-5 barrier
    if (sig_dev)
        sigma = (unsigned long long *)sigma_out;
    else
        SG_TRY_CUDA(ctx, ws.get("bc_sigma", nv, &sigma));
    SG_TRY_CUDA(ctx, ws.get("bc_delta", nv, &delta));
    if (bc_dev)
        bcv = bc_out;
    else
        SG_TRY_CUDA(ctx, ws.get("bc_out", nv, &bcv));
    SG_TRY_CUDA(ctx, cudaMemsetAsync(misc, 0, 8 * sizeof(uint32_t), ctx->stream));
    SG_TRY_CUDA(ctx, cudaMemsetAsync(sigma, 0, nv * sizeof(unsigned long long), ctx->stream));
    SG_TRY_CUDA(ctx, cudaMemsetAsync(delta, 0, nv * sizeof(float), ctx->stream));
    static const unsigned long long one = 1;  // sigma[source] = 1 (hybrid_bc.cu:325-326)
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(sigma + source, &one, sizeof one, cudaMemcpyHostToDevice, ctx->stream));

    apps::LevelStack stk{stack, misc + 0, ends, misc + 1, nv, max_levels, misc + 3};
    apps::BCForward<uint32_t, uint32_t, graphs::NoWeight> app(source, sigma, misc + 2, stk);
    sgb::EngineResult res;
    sg_status st = sgb::run_engine<decltype(app), uint32_t, uint32_t, graphs::NoWeight>(g, app, cfg, level, buffer, &res);
    if (st != SG_OK) return finish(ctx, st, res, cfg, stats);
    uint32_t hm[4];
    SG_TRY_CUDA(ctx, cudaMemcpy(hm, misc, sizeof hm, cudaMemcpyDeviceToHost));
    if (hm[3] & dev::kErrOverflow) return set_error(ctx, SG_ERR_OVERFLOW, "BC path count exceeds uint64");
    if (hm[3]) return set_error(ctx, sgb::device_error_status(hm[3]), "BC forward error bits 0x%x", hm[3]);
    const uint32_t search_depth = hm[2], nlevels = hm[1];
    float bw_ms = 0.f;
    if (search_depth >= 2) {
        const uint32_t max_depth = std::min(search_depth - 1, nlevels ? nlevels - 1 : 0);
        const uint32_t chunk_cap = (uint32_t)(g->ne / kBcChunk + g->ne / kBcBigDegree + 2);
        uint4 *chunks = nullptr;
        uint32_t *ccount = nullptr;
        SG_TRY_CUDA(ctx, ws.get("bc_chunks", chunk_cap, &chunks));
        SG_TRY_CUDA(ctx, ws.get("bc_ccount", max_levels, &ccount));
        SG_TRY_CUDA(ctx, cudaMemsetAsync(ccount, 0, max_levels * sizeof(uint32_t), ctx->stream));
        BCBackArgs ba;
        ba.row = g->row;
        ba.col = g->col;
        ba.level = level;
        ba.sigma = sigma;
        ba.delta = delta;
        ba.bc_out = bcv;
        ba.stack = stack;
        ba.ends = ends;
        ba.nlevels = nlevels;
        ba.max_depth = max_depth;
        ba.nv = nv;
        ba.chunks = chunks;
        ba.chunk_cap = chunk_cap;
        ba.chunk_count = ccount;
        ba.bar = misc + 4;
        ba.err = misc + 3;
        ba.timeout_ns = (unsigned long long)((o.timeout_s > 0 ? o.timeout_s : 30.0) * 1e9);
        static std::atomic<int> occupancy{0};
        int bps = 0;
        SG_TRY_CUDA(ctx, sgb::occupancy_once(occupancy, (const void *)bc_backward_kernel, 256, &bps));
        dim3 grid(ctx->prop.multiProcessorCount * sgb::resident_blocks_per_sm(ctx, bps));
        void *args[] = {&ba};
        SG_TRY_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
        SG_TRY_CUDA(ctx, cudaLaunchCooperativeKernel((const void *)bc_backward_kernel, grid, dim3(256), args, 0, ctx->stream));
        SG_TRY_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
        SG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        SG_TRY_CUDA(ctx, cudaEventElapsedTime(&bw_ms, ctx->ev0, ctx->ev1));
        SG_TRY_CUDA(ctx, cudaMemcpy(hm, misc, sizeof hm, cudaMemcpyDeviceToHost));
        if (hm[3]) return set_error(ctx, sgb::device_error_status(hm[3]), "BC backward error bits 0x%x", hm[3]);
    } else {
        bc_scale_kernel<<<std::max(1u, std::min((nv + 255) / 256, 4096u)), 256, 0, ctx->stream>>>(delta, bcv, nv);
        SG_TRY_CUDA(ctx, cudaGetLastError());
    }
    st = deliver(ctx, bc_out, bcv, nv, bc_dev);
    if (st == SG_OK && sigma_out && !sig_dev)
        SG_TRY_CUDA(ctx, cudaMemcpyAsync(sigma_out, sigma, nv * sizeof(uint64_t), cudaMemcpyDeviceToHost, ctx->stream));
    if (st == SG_OK) st = reached_stats(g, level, stats);
    st = finish(ctx, st, res, cfg, stats);
    if (stats) {
        stats->time_total_ms = res.ms + bw_ms;
        stats->edges_reached *= 2;  // two traversals
    }
    return st;
}

// ---------------------------------------------------------------- host graphs
sg_status sg_hgraph_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                             uint32_t flags, sg_hgraph **out) {
    if (!out) return SG_ERR_INVALID_ARG;
    sg_hgraph *h = new (std::nothrow) sg_hgraph;
    if (!h) return SG_ERR_OUT_OF_MEMORY;
    sg_status st = sgb::gen_rmat(scale, edge_factor, a, b, c, seed, flags, *h);
    if (st != SG_OK) {
        delete h;
        return st;
    }
    *out = h;
    return SG_OK;
}

sg_status sg_hgraph_gen_grid(uint32_t rows, uint32_t cols, uint32_t flags, sg_hgraph **out) {
    if (!out) return SG_ERR_INVALID_ARG;
    sg_hgraph *h = new (std::nothrow) sg_hgraph;
    if (!h) return SG_ERR_OUT_OF_MEMORY;
    sg_status st = sgb::gen_grid(rows, cols, flags, *h);
    if (st != SG_OK) {
        delete h;
        return st;
    }
    *out = h;
    return SG_OK;
}

sg_status sg_hgraph_gen_random(uint32_t nv, uint32_t gen_factor, uint64_t seed, sg_hgraph **out) {
    if (!out) return SG_ERR_INVALID_ARG;
    sg_hgraph *h = new (std::nothrow) sg_hgraph;
    if (!h) return SG_ERR_OUT_OF_MEMORY;
    sg_status st = sgb::gen_random(nv, gen_factor, seed, *h);
    if (st != SG_OK) {
        delete h;
        return st;
    }
    *out = h;
    return SG_OK;
}

sg_status sg_hgraph_from_csr(uint32_t nv, uint64_t ne, const uint32_t *offsets, const uint32_t *indices,
                             const uint32_t *weights, sg_hgraph **out) {
    if (!out) return SG_ERR_INVALID_ARG;
    sg_hgraph *h = new (std::nothrow) sg_hgraph;
    if (!h) return SG_ERR_OUT_OF_MEMORY;
    sg_status st = sgb::from_csr(nv, ne, offsets, indices, weights, *h);
    if (st != SG_OK) {
        delete h;
        return st;
    }
    *out = h;
    return SG_OK;
}

sg_status sg_hgraph_gen_weights(sg_hgraph *h, uint32_t lo, uint32_t hi, uint64_t seed) {
    if (!h) return SG_ERR_INVALID_ARG;
    return sgb::gen_weights(*h, lo, hi, seed);
}

sg_status sg_hgraph_read_gr(const char *path, sg_hgraph **out) {
    if (!path || !out) return SG_ERR_INVALID_ARG;
    sg_hgraph *h = new (std::nothrow) sg_hgraph;
    if (!h) return SG_ERR_OUT_OF_MEMORY;
    sg_status st = sgb::read_gr(path, *h);
    if (st != SG_OK) {
        delete h;
        return st;
    }
    *out = h;
    return SG_OK;
}

sg_status sg_hgraph_write_gr(const sg_hgraph *h, const char *path) {
    if (!h || !path) return SG_ERR_INVALID_ARG;
    return sgb::write_gr(*h, path);
}

sg_status sg_hgraph_read_metis(const char *path, sg_hgraph **out) {
    if (!path || !out) return SG_ERR_INVALID_ARG;
    sg_hgraph *h = new (std::nothrow) sg_hgraph;
    if (!h) return SG_ERR_OUT_OF_MEMORY;
    sg_status st = sgb::read_metis(path, *h);
    if (st != SG_OK) {
        delete h;
        return st;
    }
    *out = h;
    return SG_OK;
}

sg_status sg_hgraph_read_market(const char *path, int symmetrize, sg_hgraph **out) {
    if (!path || !out) return SG_ERR_INVALID_ARG;
    sg_hgraph *h = new (std::nothrow) sg_hgraph;
    if (!h) return SG_ERR_OUT_OF_MEMORY;
    sg_status st = sgb::read_market(path, symmetrize != 0, *h);
    if (st != SG_OK) {
        delete h;
        return st;
    }
    *out = h;
    return SG_OK;
}

sg_status sg_hgraph_info(const sg_hgraph *h, uint32_t *nv, uint64_t *ne, const uint32_t **offsets,
                         const uint32_t **indices, const uint32_t **weights) {
    if (!h) return SG_ERR_INVALID_ARG;
    if (nv) *nv = h->nv;
    if (ne) *ne = h->ne;
    if (offsets) *offsets = h->offsets.data();
    if (indices) *indices = h->indices.data();
    if (weights) *weights = h->weights.empty() ? nullptr : h->weights.data();
    return SG_OK;
}

sg_status sg_hgraph_max_degree_vertex(const sg_hgraph *h, uint32_t *vertex, uint32_t *degree) {
    if (!h) return SG_ERR_INVALID_ARG;
    return sgb::max_degree_vertex(*h, vertex, degree);
}

sg_status sg_hgraph_pick_sources(const sg_hgraph *h, uint32_t n, uint64_t seed, uint32_t *out) {
    if (!h) return SG_ERR_INVALID_ARG;
    return sgb::pick_sources(*h, n, seed, out);
}

sg_status sg_hgraph_destroy(sg_hgraph *h) {
    if (!h) return SG_ERR_INVALID_ARG;
    delete h;
    return SG_OK;
}

}  // extern "C"
