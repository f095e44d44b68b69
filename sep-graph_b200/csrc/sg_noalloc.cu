// sg_bfs_noalloc: BFS for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: code that runs inside
// another framework's memory pool or under a strict memory budget, plugins
// whose host process forbids new device allocations after start-up, and code
// paths that must not allocate while the device is being shared.  For them
// this entry point runs the same hybrid BFS engine as sg_bfs, but every
// worklist, bitmap and control word lives in one file-scope device array of
// fixed size (kNoAllocScratchBytes, about 19 MB), so the call allocates
// nothing.  The caller passes the graph (device CSR, optionally the device
// in-edge CSC) and the device output array.
//
// Limits: at most kNoAllocMaxVertices vertices and kNoAllocMaxEdges edges; larger
// inputs are rejected with SG_ERR_CAPACITY before anything runs.  Every GPU
// that loads this part of the library holds the array until the process exits.
// The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture.  All calls share the array and it keeps the last
// call's contents, so calls whose work overlaps on the GPU (different streams,
// or different host threads on one device) race and must be serialised by the
// caller.
//
// Options: opt == NULL means sg_options_default(), and every automatic choice
// (load balancing from the average degree, resident blocks per SM from the
// graph's size) is made as sg_bfs makes it, so both run the same rounds.
// Statistics filled: rounds, max_iteration_reached, rounds_by_variant,
// edges_processed, vertices_processed and device_error.  The call creates no
// timing events, so time_total_ms and time_kernel_ms are set to 0, as are the
// reached-vertex fields (edges_reached, vertices_reached, search_depth) and
// n_trace (no trace is recorded).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "sg_apps.cuh"
#include "sg_engine.cuh"
#include "sg_runtime.cuh"

namespace {

using namespace sepgraph;
using engine::Ctrl;
using engine::HeavyItem;

constexpr uint32_t kNoAllocMaxVertices = 1u << 18;
constexpr uint32_t kNoAllocMaxEdges = 1u << 23;
constexpr uint32_t kHeavyDegree = 32;
constexpr uint32_t kChunkEdges = 256;

constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr uint32_t kWords = kNoAllocMaxVertices / 32 + 1;
constexpr uint32_t kHeavyCap = (kNoAllocMaxVertices < kNoAllocMaxEdges / kHeavyDegree ? kNoAllocMaxVertices
                                                                                      : kNoAllocMaxEdges / kHeavyDegree) +
                               2;
constexpr uint32_t kChunkCap = kNoAllocMaxEdges / kChunkEdges + 2 * kHeavyCap + 2;

// Byte offsets of the regions inside the scratch array.
constexpr size_t kOffBuffer = 0;
constexpr size_t kOffTmp = kOffBuffer + align256(4ull * kNoAllocMaxVertices);
constexpr size_t kOffQueue = kOffTmp + align256(4ull * kNoAllocMaxVertices);
constexpr size_t kOffMiddle = kOffQueue + 3 * align256(4ull * kNoAllocMaxVertices);
constexpr size_t kOffBitmap = kOffMiddle + align256(4ull * kNoAllocMaxVertices);
constexpr size_t kOffFlag = kOffBitmap + 2 * align256(4ull * kWords);
constexpr size_t kOffHeavy = kOffFlag + 3 * align256(4ull * kWords);
// two heavy-vertex tables and two chunk tables (one per round parity)
constexpr size_t kOffChunk = kOffHeavy + align256(2 * sizeof(HeavyItem<uint32_t>) * kHeavyCap);
constexpr size_t kOffCtrl = kOffChunk + align256(2 * 4ull * kChunkCap);
constexpr size_t kNoAllocScratchBytes = kOffCtrl + align256(sizeof(Ctrl));

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char *g_scratch_addr[kMaxDevices] = {};

using BfsApp = apps::BFS<uint32_t, uint32_t, graphs::NoWeight>;

sg_status fail(char *err, size_t err_len, sg_status st, const char *msg) {
    if (err && err_len) {
        std::strncpy(err, msg, err_len - 1);
        err[err_len - 1] = 0;
    }
    return st;
}

bool on_device(const void *p, int dev) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == dev;
}

}  // namespace

extern "C" sg_status sg_bfs_noalloc(const uint32_t *offsets, const uint32_t *indices, uint32_t nv, uint64_t ne,
                                    const uint32_t *in_offsets, const uint32_t *in_indices, uint32_t source,
                                    const sg_options *opt, uint32_t *levels_out, void *stream, sg_stats *stats,
                                    char *err, size_t err_len) {
    char msg[256];
    if (nv == 0 || nv > kNoAllocMaxVertices || ne > kNoAllocMaxEdges) {
        std::snprintf(msg, sizeof msg, "sg_bfs_noalloc: graph of %u vertices / %llu edges exceeds the fixed scratch "
                                       "limit of %u vertices / %u edges",
                      nv, (unsigned long long)ne, kNoAllocMaxVertices, kNoAllocMaxEdges);
        return fail(err, err_len, nv == 0 ? SG_ERR_INVALID_ARG : SG_ERR_CAPACITY, msg);
    }
    if (!offsets || (ne && !indices) || !levels_out || source >= nv || (!in_offsets) != (!in_indices))
        return fail(err, err_len, SG_ERR_INVALID_ARG, "sg_bfs_noalloc: null pointer or source out of range");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(err, err_len, SG_ERR_NO_DEVICE, "sg_bfs_noalloc: no current CUDA device");
    if (!on_device(offsets, dev) || (ne && !on_device(indices, dev)) || !on_device(levels_out, dev) ||
        (in_offsets && (!on_device(in_offsets, dev) || (ne && !on_device(in_indices, dev)))))
        return fail(err, err_len, SG_ERR_INVALID_ARG, "sg_bfs_noalloc: graph and output must be device memory of "
                                                      "the current device");
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!g_scratch_addr[dev]) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                std::snprintf(msg, sizeof msg, "sg_bfs_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
                return fail(err, err_len, SG_ERR_CUDA, msg);
            }
            g_scratch_addr[dev] = (unsigned char *)p;
        }
        base = g_scratch_addr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    sg_options o;
    if (opt)
        o = *opt;
    else
        sg_options_default(&o);
    const bool has_csc = in_offsets != nullptr;
    if (!has_csc && o.variant >= 0 && (o.variant >> 1) & 1)
        return fail(err, err_len, SG_ERR_UNSUPPORTED, "sg_bfs_noalloc: pull variants need the in-edge arrays");

    engine::KArgs<uint32_t, uint32_t, graphs::NoWeight> a;
    std::memset(&a, 0, sizeof a);
    a.csr.nnodes = nv;
    a.csr.nedges = (uint32_t)ne;
    a.csr.row_start = offsets;
    a.csr.edge_dst = indices;
    a.csc.nnodes = nv;
    a.csc.nedges = (uint32_t)ne;
    a.csc.col_start = has_csc ? in_offsets : offsets;
    a.csc.edge_source = has_csc ? in_indices : indices;
    a.csc.csr_row_start = offsets;
    a.value = levels_out;
    a.buffer = (uint32_t *)(base + kOffBuffer);
    a.tmp = (uint32_t *)(base + kOffTmp);
    for (int k = 0; k < 3; ++k) a.queue[k] = (uint32_t *)(base + kOffQueue + k * align256(4ull * kNoAllocMaxVertices));
    a.queue_cap = nv;
    for (int k = 0; k < 2; ++k) a.bitmap[k] = (uint32_t *)(base + kOffBitmap + k * align256(4ull * kWords));
    for (int k = 0; k < 3; ++k) a.qflag[k] = (uint32_t *)(base + kOffFlag + k * align256(4ull * kWords));
    a.nwords = nv / 32 + 1;
    a.middle = (uint32_t *)(base + kOffMiddle);
    a.heavy = (HeavyItem<uint32_t> *)(base + kOffHeavy);
    a.heavy_cap = kHeavyCap;
    a.chunk_owner = (uint32_t *)(base + kOffChunk);
    a.chunk_cap = kChunkCap;
    a.ctrl = (Ctrl *)(base + kOffCtrl);
    engine::Params &p = a.p;
    p.scheme = 0;
    p.forced = o.variant;
    if (o.alpha == 0) p.forced = engine::V_ASYNC_PUSH_DD;
    if (!has_csc && p.forced < 0) p.forced = engine::V_ASYNC_PUSH_DD;
    const double avg_deg = (double)ne / nv;
    p.lb_push = o.lb_push >= 0 ? o.lb_push : (avg_deg >= 5 ? engine::LB_FINE : engine::LB_NONE);
    p.lb_pull = o.lb_pull >= 0 ? o.lb_pull : engine::LB_FINE;
    p.collect = p.forced < 0 ? 1 : 0;
    p.has_csc = 1;  // without in-edges the variant is forced to push above
    p.max_iteration = o.max_iteration > 0 ? (uint32_t)o.max_iteration : 200u;
    p.heavy_threshold = kHeavyDegree;
    p.chunk_edges = kChunkEdges;
    p.pull_warp_threshold = 32;
    p.local_depth = o.local_depth > 0 ? (uint32_t)o.local_depth : 0u;
    p.sample_cut = 0.f;
    p.bitmap_frontier = engine::use_bitmap_frontier(p.forced, p.lb_push, false, o.worklist);
    p.alpha = o.alpha;
    p.beta = o.beta > 0 ? o.beta : 18;
    p.total_workload0 = (long long)((double)ne * (o.edge_factor > 0 ? o.edge_factor : 1.0));
    p.timeout_ns = (unsigned long long)((o.timeout_s > 0 ? o.timeout_s : 30.0) * 1e9);

    BfsApp app(source, o.non_atomic != 0 && o.local_depth <= 0);  // lookahead needs the atomic minimum
    app.m_csr_graph = a.csr;
    app.m_csc_graph = a.csc;
    app.m_nnodes = nv;
    app.m_nedges = (uint32_t)ne;
    app.m_p_current_round = &a.ctrl->rs.round;

    // State that must start at zero: the control block and the heavy-vertex
    // tables (bitmaps are cleared by the kernel's first phase).
    cudaError_t e = cudaMemsetAsync(base + kOffHeavy, 0, kOffCtrl + sizeof(Ctrl) - kOffHeavy, s);
    auto kernel = engine::hybrid_engine_kernel<BfsApp, uint32_t, uint32_t, graphs::NoWeight>;
    int bps = 0, sms = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kernel, engine::kBlockThreads, 0);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) {
        const int want = o.blocks_per_sm > 0 ? o.blocks_per_sm : sgb::auto_blocks_per_sm(nv, ne);
        dim3 grid(sms * (bps < want ? bps : want)), block(engine::kBlockThreads);
        void *args[] = {(void *)&app, (void *)&a};
        e = cudaLaunchCooperativeKernel((const void *)kernel, grid, block, args, 0, s);
    }
    Ctrl c;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&c, a.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        std::snprintf(msg, sizeof msg, "sg_bfs_noalloc: %s", cudaGetErrorString(e));
        return fail(err, err_len, SG_ERR_CUDA, msg);
    }
    const uint32_t bits = c.error | c.cnt.error;
    if (stats) {
        stats->time_total_ms = 0;
        stats->time_kernel_ms = 0;
        stats->edges_reached = 0;
        stats->vertices_reached = 0;
        stats->search_depth = 0;
        stats->rounds = c.round;
        stats->max_iteration_reached = c.max_iteration_reached;
        for (int k = 0; k < 8; ++k) stats->rounds_by_variant[k] = c.rounds_by_variant[k];
        stats->edges_processed = c.cnt.edges_processed;
        stats->vertices_processed = c.vertices_processed;
        stats->device_error = bits;
        stats->n_trace = 0;
    }
    if (bits & dev::kErrTimeout) return fail(err, err_len, SG_ERR_TIMEOUT, "sg_bfs_noalloc: device wait timed out");
    if (bits & (dev::kErrCapacity | dev::kErrChunkCapacity))
        return fail(err, err_len, SG_ERR_CAPACITY, "sg_bfs_noalloc: worklist capacity exceeded");
    if (bits & dev::kErrUnsupported) return fail(err, err_len, SG_ERR_UNSUPPORTED, "sg_bfs_noalloc: unsupported variant");
    return SG_OK;
}
