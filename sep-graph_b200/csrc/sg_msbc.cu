// Multi-source betweenness centrality: up to 32 sources of one graph in one
// persistent launch.
//
// Single-source BC (StageOne/StageTwo of samples/hybrid_bc/hybrid_bc.cu,
// host form hybrid_bc_host.cpp:16-92) runs a BFS that counts shortest paths
// (sigma), then accumulates dependencies deepest level first:
//   delta[v] = sum over v->w with level[w] == level[v]+1 of sigma[v]/sigma[w] * (1 + delta[w])
// and reports delta * 0.5.  Here the 32 sources advance together, one warp
// lane per source: per vertex a 32-bit mask of the sources whose frontier it
// is in, rows of 32 path counts (uint64) and 32 dependencies (float).
//
// Forward, level d -> d+1 (pull over in-edges): a vertex that some source has
// not reached ORs its in-neighbours' frontier masks; for the new bits the
// warp sums the in-neighbours' path counts lane by lane, eight row loads in
// flight (no atomics except on split hubs).  Work is tiered by in-degree: a
// thread finds the new bits of a
// vertex with <= 64 in-edges and its warp then sums the counts of those
// vertices one at a time; vertices with more in-edges are listed once for a
// warp each, and those above 512 are split into 256-edge chunks whose
// partial sums are added atomically.  The level's discoveries are appended
// to a list as (vertex, mask) pairs.
//
// Backward, level d (deepest first): the masks of levels d+1 (successors) and
// d (the vertices themselves) are scattered into dense arrays from the level
// lists; a warp takes a vertex of level d, reads 32 out-edges at a time, keeps
// the edges whose head has one of the vertex's sources at depth d+1 and sums
// q(w) = (1 + delta(w)) / sigma(w) lane by lane, so that
// delta(v) = sigma(v) * sum q(w) (the single-source sum with sigma(v)
// factored out: one float row per edge instead of two rows and a division).
// The sources keep delta 0 (depth-0 entries are never accumulated), as in the
// single-source pass.
// No reference counterpart: the reference runs one source per Engine.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cstring>

#include "sg_runtime.cuh"

namespace {

using namespace sepgraph;
using engine::Ctrl;

constexpr int kMbThreads = 256;
constexpr uint32_t kMbThreadDeg = 64;  // in-degree up to this: a thread finds the new sources
constexpr uint32_t kMbSplit = 512;     // degree above this: split into chunks
constexpr uint32_t kMbChunk = 256;     // edges per chunk
constexpr uint32_t kMbSources = 32;

struct MbArgs {
    const uint32_t *row, *col;    // CSR: successors (backward)
    const uint32_t *crow, *ccol;  // CSC: predecessors (forward; may alias the CSR)
    uint32_t nv, nsrc, full;
    uint32_t *seen, *fr, *nx;       // per-vertex source masks
    uint32_t *fm_next, *fm_cur;     // backward: masks of levels d+1 and d
    unsigned long long *sigma;      // nv x 32
    float *delta;                   // nv x 32
    float *q;                       // nv x 32: (1 + delta) / sigma of finished levels
    uint2 *list;                    // (vertex, mask) per level, concatenated
    uint32_t list_cap;
    uint32_t *ends;                 // ends[d+1] = end of level d's entries; ends[0] = 0
    uint32_t max_levels;
    uint32_t *wlist;                // in-degree kMbThreadDeg+1 .. kMbSplit (forward warp tier)
    uint4 *chunks[2];               // (v, first edge, edges, -): [0] in-edges (forward), [1] out-edges (backward)
    uint32_t chunk_cap;
    uint32_t *counts;               // [0] wlist size, [1],[2] chunk counts, [3] level appends
    const uint32_t *sources;
    float *bc;                      // nsrc rows of nv
    Ctrl *ctrl;
    unsigned long long timeout_ns;
};

__device__ __forceinline__ uint32_t gthread() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint32_t nthreads() { return gridDim.x * blockDim.x; }

__device__ __forceinline__ void add_checked(unsigned long long &acc, unsigned long long x, bool &ovf) {
    const unsigned long long r = acc + x;
    ovf |= r < acc;
    acc = r;
}

constexpr int kMbGather = 8;  // row loads in flight per gather step

// The next up to kMbGather set bits of the warp-uniform mask m (32 = none).
__device__ __forceinline__ void take_bits(uint32_t &m, uint32_t (&j)[kMbGather]) {
#pragma unroll
    for (int t = 0; t < kMbGather; ++t) {
        j[t] = m ? (uint32_t)__ffs(m) - 1 : 32u;
        if (m) m &= m - 1;
    }
}

// Sum, lane by lane, the path counts of the in-neighbours in [b, b+deg) whose
// frontier mask has a bit of `want`; returns the OR of those masks (& want).
// Up to kMbGather rows are loaded before they are added.
__device__ __forceinline__ uint32_t pull_counts(const MbArgs &a, uint32_t b, uint32_t deg, uint32_t want,
                                                unsigned long long &acc, bool &ovf) {
    const uint32_t lane = dev::lane_id();
    uint32_t got = 0;
    for (uint32_t k = 0; k < deg; k += 32) {
        uint32_t u = 0, f = 0;
        if (k + lane < deg) {
            u = __ldg(a.ccol + b + k + lane);
            f = __ldcg(a.fr + u) & want;
        }
        uint32_t m = __ballot_sync(dev::kFullMask, f != 0);
        while (m) {
            uint32_t j[kMbGather];
            take_bits(m, j);
            unsigned long long x[kMbGather];
#pragma unroll
            for (int t = 0; t < kMbGather; ++t) {
                const uint32_t src = j[t] < 32 ? j[t] : 0u;
                const uint32_t uj = __shfl_sync(dev::kFullMask, u, src);
                const uint32_t fj = j[t] < 32 ? __shfl_sync(dev::kFullMask, f, src) : 0u;
                got |= fj;
                x[t] = ((fj >> lane) & 1u) ? __ldcg(a.sigma + (size_t)uj * kMbSources + lane) : 0ull;
            }
#pragma unroll
            for (int t = 0; t < kMbGather; ++t) add_checked(acc, x[t], ovf);
        }
    }
    return got;
}

// Brandes' dependency factored per successor: delta(v) = sigma(v) * sum over
// successors w one level deeper of q(w), q(w) = (1 + delta(w)) / sigma(w),
// stored once per (w, source) when w's level is finished.  Sums q over the
// out-edges [b, b+deg) whose head has a source of `act` one level deeper.
__device__ __forceinline__ float sum_q(const MbArgs &a, uint32_t b, uint32_t deg, uint32_t act) {
    const uint32_t lane = dev::lane_id();
    float acc = 0.f;
    for (uint32_t k = 0; k < deg; k += 32) {
        uint32_t w = 0, f = 0;
        if (k + lane < deg) {
            w = __ldg(a.col + b + k + lane);
            f = __ldcg(a.fm_next + w) & act;
        }
        uint32_t m = __ballot_sync(dev::kFullMask, f != 0);
        while (m) {
            uint32_t j[kMbGather];
            take_bits(m, j);
            float x[kMbGather];
#pragma unroll
            for (int t = 0; t < kMbGather; ++t) {
                const uint32_t src = j[t] < 32 ? j[t] : 0u;
                const uint32_t wj = __shfl_sync(dev::kFullMask, w, src);
                const uint32_t fj = j[t] < 32 ? __shfl_sync(dev::kFullMask, f, src) : 0u;
                x[t] = ((fj >> lane) & 1u) ? __ldcg(a.q + (size_t)wj * kMbSources + lane) : 0.f;
            }
#pragma unroll
            for (int t = 0; t < kMbGather; ++t) acc += x[t];
        }
    }
    return acc;
}

// Finishes (v, source lane) of a level: delta = sigma * sum, q = (1 + delta) / sigma.
__device__ __forceinline__ void finish_dep(const MbArgs &a, uint32_t v, float sum) {
    const size_t k = (size_t)v * kMbSources + dev::lane_id();
    const float sv = (float)__ldcg(a.sigma + k);
    const float d = sv * sum;
    a.delta[k] = d;
    a.q[k] = (1.0f + d) / sv;
}

__global__ void __launch_bounds__(kMbThreads) msbc_kernel(MbArgs a) {
    Ctrl *c = a.ctrl;
    engine::set_team(blockIdx.x, gridDim.x, c);
    engine::Counters *n = &c->cnt;
    const uint32_t lane = dev::lane_id();
    const uint32_t gw = gthread() >> 5, nw = nthreads() >> 5;
    auto nop = [] {};
    __shared__ uint32_t s_level, s_done, s_e;
    __shared__ float tile[kMbThreads / 32][32][33];

    // init: masks, rows, tier lists
    for (uint32_t v = gthread(); v < a.nv; v += nthreads()) {
        a.seen[v] = a.fr[v] = a.nx[v] = 0;
        a.fm_next[v] = a.fm_cur[v] = 0;
        const uint32_t ib = __ldg(a.crow + v), ideg = __ldg(a.crow + v + 1) - ib;
        if (ideg > kMbThreadDeg && ideg <= kMbSplit) a.wlist[atomicAdd(a.counts, 1u)] = v;
        for (int dir = 0; dir < 2; ++dir) {
            const uint32_t *off = dir == 0 ? a.crow : a.row;
            const uint32_t b = __ldg(off + v), deg = __ldg(off + v + 1) - b;
            if (deg <= kMbSplit) continue;
            const uint32_t nch = (deg + kMbChunk - 1) / kMbChunk;
            const uint32_t c0 = atomicAdd(a.counts + 1 + dir, nch);
            for (uint32_t k = 0; k < nch; ++k) {
                if (c0 + k < a.chunk_cap)
                    a.chunks[dir][c0 + k] = make_uint4(v, b + k * kMbChunk, min(kMbChunk, deg - k * kMbChunk), 0);
                else
                    atomicOr(&n->error, dev::kErrChunkCapacity);
            }
        }
    }
    const uint64_t rows = (uint64_t)a.nv * kMbSources;
    for (uint64_t k = gthread(); k < rows; k += nthreads()) {
        a.sigma[k] = 0;
        a.delta[k] = 0.f;
    }
    if (!engine::grid_sync(c, a.timeout_ns, nop)) return;
    if (gthread() < a.nsrc) {
        const uint32_t s = gthread(), v = a.sources[s];
        atomicOr(a.seen + v, 1u << s);
        atomicOr(a.nx + v, 1u << s);
        a.sigma[(size_t)v * kMbSources + s] = 1;
    }
    if (!engine::grid_sync(c, a.timeout_ns, nop)) return;
    // level 0 = the sources (warp-uniform loop: every lane reaches the ballot)
    for (uint32_t base0 = gw * 32; base0 < a.nv; base0 += nw * 32) {
        const uint32_t v = base0 + lane;
        const uint32_t m = v < a.nv ? a.nx[v] : 0u;
        const bool put = m != 0;
        const uint32_t bm = __ballot_sync(dev::kFullMask, put);
        if (bm) {
            uint32_t base = 0;
            if (lane == __ffs(bm) - 1) base = atomicAdd(a.counts + 3, (uint32_t)__popc(bm));
            base = __shfl_sync(dev::kFullMask, base, __ffs(bm) - 1);
            if (put) {
                a.fr[v] = m;
                a.nx[v] = 0;
                const uint32_t p = base + __popc(bm & dev::lanemask_lt());
                if (p < a.list_cap) a.list[p] = make_uint2(v, m);
                else atomicOr(&n->error, dev::kErrCapacity);
            }
        }
    }
    auto close_level = [&] {  // leader: end of the level just appended
        const uint32_t d = c->round;
        const uint32_t cnt = dev::ld_l2(a.counts + 3);
        a.ends[d + 1] = a.ends[d] + cnt;  // level d's entries end here
        a.counts[3] = 0;
        c->round = d + 1;
        c->rs.done = cnt == 0 || d + 2 >= a.max_levels ? 1u : 0u;
        if (cnt != 0 && d + 2 >= a.max_levels) atomicOr(&n->error, dev::kErrCapacity);
    };
    if (!engine::grid_sync(c, a.timeout_ns, [&] {
            a.ends[0] = 0;
            c->round = 0;
            close_level();
        }))
        return;

    // ---------------------------------------------------------------- forward
    bool ovf = false;
    for (;;) {
        if (threadIdx.x == 0) {
            s_level = dev::ld_l2(&c->round);  // next depth to discover
            s_done = dev::ld_l2(&c->rs.done);
            s_e = dev::ld_l2(a.ends + s_level);
        }
        __syncthreads();
        if (s_done) break;
        const uint32_t nwl = min(dev::ld_l2(a.counts), a.nv);
        const uint32_t nch = min(dev::ld_l2(a.counts + 1), a.chunk_cap);
        // thread tier: new bits of vertices with <= kMbThreadDeg in-edges
        for (uint32_t base = gw * 32; base < a.nv; base += nw * 32) {
            const uint32_t v = base + lane;
            uint32_t want = 0, nm = 0, b = 0, deg = 0;
            if (v < a.nv) {
                b = __ldg(a.crow + v);
                deg = __ldg(a.crow + v + 1) - b;
                if (deg <= kMbThreadDeg) want = a.full & ~__ldcg(a.seen + v);
                if (want) {
                    for (uint32_t e = b; e < b + deg; ++e) {
                        nm |= __ldcg(a.fr + __ldg(a.ccol + e));
                        if ((nm & want) == want) break;
                    }
                    nm &= want;
                }
            }
            uint32_t m = __ballot_sync(dev::kFullMask, nm != 0);
            while (m) {
                const uint32_t j = __ffs(m) - 1;
                m &= m - 1;
                const uint32_t vj = __shfl_sync(dev::kFullMask, v, j), nj = __shfl_sync(dev::kFullMask, nm, j);
                const uint32_t bj = __shfl_sync(dev::kFullMask, b, j), dj = __shfl_sync(dev::kFullMask, deg, j);
                unsigned long long acc = 0;
                pull_counts(a, bj, dj, nj, acc, ovf);
                if ((nj >> lane) & 1u) a.sigma[(size_t)vj * kMbSources + lane] = acc;
                if (lane == 0) a.nx[vj] = nj;
            }
        }
        // warp tier
        for (uint32_t i = gw; i < nwl; i += nw) {
            const uint32_t v = __ldg(a.wlist + i);
            const uint32_t want = a.full & ~__ldcg(a.seen + v);
            if (!want) continue;
            const uint32_t b = __ldg(a.crow + v), deg = __ldg(a.crow + v + 1) - b;
            unsigned long long acc = 0;
            const uint32_t got = pull_counts(a, b, deg, want, acc, ovf);
            if ((got >> lane) & 1u) a.sigma[(size_t)v * kMbSources + lane] = acc;
            if (lane == 0 && got) a.nx[v] = got;
        }
        // chunks of split vertices: partial sums added atomically
        for (uint32_t i = gw; i < nch; i += nw) {
            const uint4 ch = a.chunks[0][i];
            const uint32_t want = a.full & ~__ldcg(a.seen + ch.x);
            if (!want) continue;
            unsigned long long acc = 0;
            const uint32_t got = pull_counts(a, ch.y, ch.z, want, acc, ovf);
            if ((got >> lane) & 1u) {
                const unsigned long long old = atomicAdd(a.sigma + (size_t)ch.x * kMbSources + lane, acc);
                ovf |= old + acc < old;
            }
            if (lane == 0 && got) atomicOr(a.nx + ch.x, got);
        }
        if (!engine::grid_sync(c, a.timeout_ns, nop)) return;
        // commit: the new bits become the frontier and a level-list entry
        for (uint32_t base0 = gw * 32; base0 < a.nv; base0 += nw * 32) {
            const uint32_t v = base0 + lane;
            const uint32_t m = v < a.nv ? __ldcg(a.nx + v) : 0u;
            const bool put = m != 0;
            if (!put && v < a.nv && __ldcg(a.fr + v)) a.fr[v] = 0;
            const uint32_t bm = __ballot_sync(dev::kFullMask, put);
            if (!bm) continue;
            uint32_t base = 0;
            if (lane == __ffs(bm) - 1) base = atomicAdd(a.counts + 3, (uint32_t)__popc(bm));
            base = __shfl_sync(dev::kFullMask, base, __ffs(bm) - 1);
            if (put) {
                a.nx[v] = 0;
                a.fr[v] = m;
                a.seen[v] |= m;
                const uint32_t p = s_e + base + __popc(bm & dev::lanemask_lt());
                if (p < a.list_cap) a.list[p] = make_uint2(v, m);
                else atomicOr(&n->error, dev::kErrCapacity);
            }
        }
        if (!engine::grid_sync(c, a.timeout_ns, close_level)) return;
    }
    if (ovf) atomicOr(&n->error, dev::kErrOverflow);
    // A level list that ran out of room is incomplete and its level ends point
    // past the entries written: the host retries with the full bound, so this
    // launch stops here.  Every block reads the same bit (nothing sets it
    // after the forward pass's last barrier) and returns before the backward
    // pass's first barrier.
    if (dev::ld_l2(&n->error) & dev::kErrCapacity) return;

    // ---------------------------------------------------------------- backward
    // levels 0 .. L-1 hold entries (the last appended level was empty); the
    // deepest level has delta 0, so q = 1 / sigma there.  Level ends are
    // clamped to the list's capacity as a second guard.
    auto end_of = [&](uint32_t d) { return min(dev::ld_l2(a.ends + d), a.list_cap); };
    const uint32_t L = dev::ld_l2(&c->round) - 1;
    const uint32_t nch1 = min(dev::ld_l2(a.counts + 2), a.chunk_cap);
    if (L >= 2) {
        const uint32_t b0 = end_of(L - 1), e0 = end_of(L);
        for (uint32_t i = b0 + gw; i < e0; i += nw) {
            const uint2 en = a.list[i];
            if ((en.y >> lane) & 1u) finish_dep(a, en.x, 0.f);
        }
    }
    for (int d = (int)L - 2; d >= 1; --d) {
        const uint32_t b0 = end_of(d), e0 = end_of(d + 1), e1 = end_of(d + 2);
        // masks of level d+1 and level d, dense
        for (uint32_t i = b0 + gthread(); i < e1; i += nthreads()) {
            const uint2 en = a.list[i];
            if (i < e0) a.fm_cur[en.x] = en.y;
            else a.fm_next[en.x] = en.y;
        }
        if (!engine::grid_sync(c, a.timeout_ns, nop)) return;
        for (uint32_t i = b0 + gw; i < e0; i += nw) {
            const uint2 en = a.list[i];
            const uint32_t b = __ldg(a.row + en.x), deg = __ldg(a.row + en.x + 1) - b;
            if (deg > kMbSplit) continue;  // chunks below
            const float sum = sum_q(a, b, deg, en.y);
            if ((en.y >> lane) & 1u) finish_dep(a, en.x, sum);
        }
        // split vertices: partial sums of q collect in delta, finished below
        for (uint32_t i = gw; i < nch1; i += nw) {
            const uint4 ch = a.chunks[1][i];
            const uint32_t act = __ldcg(a.fm_cur + ch.x);
            if (!act) continue;
            const float sum = sum_q(a, ch.y, ch.z, act);
            if ((act >> lane) & 1u) atomicAdd(a.delta + (size_t)ch.x * kMbSources + lane, sum);
        }
        if (!engine::grid_sync(c, a.timeout_ns, nop)) return;
        for (uint32_t i = b0 + gw; i < e0; i += nw) {
            const uint2 en = a.list[i];
            if (__ldg(a.row + en.x + 1) - __ldg(a.row + en.x) > kMbSplit && ((en.y >> lane) & 1u))
                finish_dep(a, en.x, __ldcg(a.delta + (size_t)en.x * kMbSources + lane));
        }
        for (uint32_t i = b0 + gthread(); i < e1; i += nthreads()) {
            const uint2 en = a.list[i];
            if (i < e0) a.fm_cur[en.x] = 0;
            else a.fm_next[en.x] = 0;
        }
        if (!engine::grid_sync(c, a.timeout_ns, nop)) return;
    }

    // ---------------------------------------------------------------- output
    // bc[s][v] = delta[v][s] * 0.5, transposed through shared memory
    float(*t)[33] = tile[threadIdx.x >> 5];
    for (uint32_t base = gw * 32; base < a.nv; base += nw * 32) {
        for (uint32_t r = 0; r < 32; ++r) {
            const uint32_t v = base + r;
            t[r][lane] = v < a.nv ? __ldcg(a.delta + (size_t)v * kMbSources + lane) : 0.f;
        }
        __syncwarp();
        const uint32_t v = base + lane;
        if (v < a.nv)
            for (uint32_t s = 0; s < a.nsrc; ++s) a.bc[(size_t)s * a.nv + v] = t[lane][s] * 0.5f;
        __syncwarp();
    }
}

}  // namespace

namespace sgb {

// Multi-source BC into bc_out (nsrc rows of nv) or, when row_outs is given,
// row i to row_outs[i] (host or device, nv floats each).
sg_status msbc_rows(sg_graph *g, const uint32_t *sources, uint32_t nsrc, const sg_options *opt, float *bc_out,
                    float *const *row_outs, sg_stats *stats) {
    if (!g || !g->ctx || !sources || (!bc_out && !row_outs) || nsrc == 0 || nsrc > kMbSources)
        return SG_ERR_INVALID_ARG;
    sg_ctx *ctx = g->ctx;
    for (uint32_t i = 0; i < nsrc; ++i)
        if (sources[i] >= g->nv) return sgb::set_error(ctx, SG_ERR_INVALID_ARG, "source %u out of range", sources[i]);
    if (!g->has_csc && !g->symmetric)
        return sgb::set_error(ctx, SG_ERR_UNSUPPORTED, "multi-source BC pulls over in-edges: graph has no CSC view");
    sgb::DeviceGuard dg(ctx->device);
    const sg_options o = opt ? *opt : sg_options{};
    const uint32_t nv = g->nv;
    sgb::Workspace &ws = sgb::graph_ws(g);
    MbArgs a{};
    a.row = g->row;
    a.col = g->col;
    a.crow = g->has_csc ? g->crow : g->row;
    a.ccol = g->has_csc ? g->ccol : g->col;
    a.nv = nv;
    a.nsrc = nsrc;
    a.full = nsrc == 32 ? 0xffffffffu : ((1u << nsrc) - 1);
    SG_TRY_CUDA(ctx, ws.get("mb_seen", nv, &a.seen));
    SG_TRY_CUDA(ctx, ws.get("mb_fr", nv, &a.fr));
    SG_TRY_CUDA(ctx, ws.get("mb_nx", nv, &a.nx));
    SG_TRY_CUDA(ctx, ws.get("mb_fm_next", nv, &a.fm_next));
    SG_TRY_CUDA(ctx, ws.get("mb_fm_cur", nv, &a.fm_cur));
    SG_TRY_CUDA(ctx, ws.get("mb_sigma", (size_t)nv * kMbSources, &a.sigma));
    SG_TRY_CUDA(ctx, ws.get("mb_delta", (size_t)nv * kMbSources, &a.delta));
    SG_TRY_CUDA(ctx, ws.get("mb_q", (size_t)nv * kMbSources, &a.q));
    SG_TRY_CUDA(ctx, ws.get("mb_wlist", nv, &a.wlist));
    a.chunk_cap = (uint32_t)std::min<uint64_t>(2 * (g->ne / kMbChunk) + 2, 0xffffffffu);
    SG_TRY_CUDA(ctx, ws.get("mb_chunks_in", a.chunk_cap, &a.chunks[0]));
    SG_TRY_CUDA(ctx, ws.get("mb_chunks_out", a.chunk_cap, &a.chunks[1]));
    SG_TRY_CUDA(ctx, ws.get("mb_counts", 4, &a.counts));
    a.max_levels = nv + 2;  // depths are < nv
    SG_TRY_CUDA(ctx, ws.get("mb_ends", (size_t)a.max_levels + 1, &a.ends));
    SG_TRY_CUDA(ctx, ws.get("ctrl", 1, &a.ctrl));
    uint32_t *dsrc = nullptr;
    SG_TRY_CUDA(ctx, ws.get("mb_sources", kMbSources, &dsrc));
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(dsrc, sources, 4 * nsrc, cudaMemcpyHostToDevice, ctx->stream));
    a.sources = dsrc;
    const bool out_dev = !row_outs && sgb::is_device_ptr(bc_out, ctx->device);
    if (out_dev) a.bc = bc_out;
    else SG_TRY_CUDA(ctx, ws.get("mb_bc", (size_t)nsrc * nv, &a.bc));
    a.timeout_ns = (unsigned long long)((o.timeout_s > 0 ? o.timeout_s : 30.0) * 1e9);

    static std::atomic<int> occupancy{0};
    int bps = 0;
    SG_TRY_CUDA(ctx, sgb::occupancy_once(occupancy, (const void *)msbc_kernel, kMbThreads, &bps));
    if (bps <= 0) return sgb::set_error(ctx, SG_ERR_NO_DEVICE, "multi-source BC kernel cannot be resident");
    const int want = o.blocks_per_sm > 0 ? o.blocks_per_sm : sgb::ms_blocks_per_sm(nv, g->ne, nsrc);
    const dim3 grid(ctx->prop.multiProcessorCount * std::max(1, std::min(sgb::resident_blocks_per_sm(ctx, bps), want)));
    // a vertex appears once per depth at which some source reaches it; start
    // with 8 depths per vertex and retry with the bound of 32
    Ctrl h{};
    float ms = 0.f;
    for (uint32_t per : {8u, kMbSources}) {
        a.list_cap = (uint32_t)std::min<uint64_t>((uint64_t)nv * per, 0xffffffffu);
        SG_TRY_CUDA(ctx, ws.get(per == 8 ? "mb_list8" : "mb_list32", a.list_cap, &a.list));
        SG_TRY_CUDA(ctx, cudaMemsetAsync(a.ctrl, 0, sizeof(Ctrl), ctx->stream));
        SG_TRY_CUDA(ctx, cudaMemsetAsync(a.counts, 0, 4 * sizeof(uint32_t), ctx->stream));
        SG_TRY_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
        void *args[] = {&a};
        SG_TRY_CUDA(ctx, cudaLaunchCooperativeKernel((const void *)msbc_kernel, grid, dim3(kMbThreads), args, 0,
                                                     ctx->stream));
        SG_TRY_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
        SG_TRY_CUDA(ctx, cudaMemcpyAsync(&h, a.ctrl, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
        SG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (!(h.cnt.error & dev::kErrCapacity) || per == kMbSources) break;
    }
    SG_TRY_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    if (row_outs) {
        for (uint32_t i = 0; i < nsrc; ++i)
            SG_TRY_CUDA(ctx, cudaMemcpy(row_outs[i], a.bc + (size_t)i * nv, 4ull * nv, cudaMemcpyDefault));
    } else if (!out_dev) {
        SG_TRY_CUDA(ctx, cudaMemcpy(bc_out, a.bc, 4ull * nsrc * nv, cudaMemcpyDeviceToHost));
    }
    const uint32_t bits = h.cnt.error;
    if (stats) {
        std::memset(stats, 0, offsetof(sg_stats, trace));
        stats->rounds = h.round;
        stats->search_depth = h.round > 1 ? h.round - 2 : 0;
        stats->time_total_ms = stats->time_kernel_ms = ms;
        stats->device_error = bits;
    }
    const sg_status st = sgb::device_error_status(bits);
    if (st != SG_OK) return sgb::set_error(ctx, st, "multi-source BC device error bits 0x%x", bits);
    return SG_OK;
}

}  // namespace sgb

extern "C" sg_status sg_msbc(sg_graph *g, const uint32_t *sources, uint32_t nsrc, const sg_options *opt,
                             float *bc_out, sg_stats *stats) {
    if (!bc_out) return SG_ERR_INVALID_ARG;
    return sgb::msbc_rows(g, sources, nsrc, opt, bc_out, nullptr, stats);
}
