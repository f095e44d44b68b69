// Batched traversals: many BFS sources in one persistent launch.
//
// Multi-source BFS with 64-bit per-vertex source masks (bit i = source i).
// Each round: expand the active vertices' masks to their neighbours (push,
// atomicOr of the bits the neighbour has not seen) or let every vertex that
// still misses some source OR its in-neighbours' masks (pull, early exit once
// every missing bit is covered), then fix the newly seen bits, write their
// levels and build the next active list.  A vertex reached by several
// sources in the same round is expanded once for all of them, so 64 BFSs cost
// a few passes over the graph instead of 64.  Work is balanced in three tiers
// by degree: a thread per vertex up to 32 edges, a warp per vertex up to 256,
// and 256-edge chunks of bigger vertices (listed once per launch) spread over
// all warps, so one hub never holds up a round.  The direction switch uses the
// single-source engine's rule (scout count against the in-edges of vertices
// some source has not reached yet / alpha, and beta for leaving pull,
// include/framework/hybrid_policy.h:265-288).  No reference counterpart: the
// reference runs one source per Engine.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include <cmath>
#include <cstddef>

#include <type_traits>

#include "sg_apps.cuh"
#include "sg_bc.cuh"
#include "sg_runtime.cuh"

namespace {

using namespace sepgraph;
using engine::Ctrl;

constexpr int kMsThreads = 256;
constexpr uint32_t kMsWarp = 32;     // vertices above this degree are scanned by a whole warp
constexpr uint32_t kMsChunk = 256;   // vertices above this degree are split into chunks of this many edges
constexpr uint32_t kNoVertex = 0xffffffffu;  // an empty edge slot (vertex ids are below nv < 2^32 - 1)

// The vertices' masks: seen (the sources that reached it), next (bits ORed
// into it this round) and the frontier masks of the current and the next
// round (fr[qin], fr[qin ^ 1]).  Two layouts, chosen per launch:
//  - interleaved, a vertex's four masks in 32 bytes (one sector): a push round
//    touches all of a neighbour's masks together.  Measured on B200, 64 BFS on
//    the 4096^2 grid 1048 -> 759 ms, on the 2048^2 grid 241 -> 183 ms.
//  - one dense array per mask: a pull round reads the frontier masks of random
//    in-neighbours, and the 8-byte-per-vertex array of a graph of a few
//    million vertices stays in L2 (64 BFS on directed RMAT-22 7.7 ms dense,
//    8.8 ms interleaved).
// Sparse high-diameter graphs (average degree below 8) run push rounds, so
// they take the interleaved layout (the push-only kernel below keeps seen and
// the two round parities' next masks there; the two-phase kernel, when pull
// is forced on such a graph, its four masks).
enum : uint32_t { kSeen = 0, kNext = 1, kFr0 = 2 };
struct MsMasks {
    unsigned long long *base;
    uint64_t fstride;  // between a vertex's masks: 1 interleaved, nv dense
    uint32_t vstride;  // between vertices: 4 interleaved, 1 dense
    __device__ __forceinline__ unsigned long long *at(uint32_t field, uint32_t v) const {
        return base + field * fstride + (uint64_t)v * vstride;
    }
    // seen and next of v (one 16-byte load when interleaved)
    __device__ __forceinline__ void seen_next(uint32_t v, unsigned long long &seen, unsigned long long &next) const {
        if (vstride == 4) {
            const uint4 q = __ldcg(reinterpret_cast<const uint4 *>(base + 4ull * v));
            seen = (unsigned long long)q.x | ((unsigned long long)q.y << 32);
            next = (unsigned long long)q.z | ((unsigned long long)q.w << 32);
        } else {
            seen = __ldcg(at(kSeen, v));
            next = __ldcg(at(kNext, v));
        }
    }
};

struct MsArgs {
    const uint32_t *row, *col;    // CSR
    const uint32_t *crow, *ccol;  // CSC (may alias CSR)
    uint32_t nv, nsrc;
    unsigned long long full;      // mask of the nsrc source bits
    MsMasks m;  // nv vertices' masks (4 * nv words)
    uint32_t *active[2], *touched;
    const uint32_t *sources;
    uint32_t *levels;  // nsrc rows of nv
    // Chunks (v, first edge, edges, -) of the vertices above kMsChunk out-edges
    // (CSR, [0]) and in-edges (CSC, [1]), listed once at the start of the
    // launch; every round spreads them over all warps (push: chunks of frontier
    // vertices, pull: chunks of vertices that still miss a source).
    uint4 *chunks[2];
    uint32_t chunk_cap;
    uint32_t *n_chunks;  // [2], zero at launch
    Ctrl *ctrl;
    uint32_t max_rounds;
    double alpha, beta;
    long long total_edges;
    unsigned long long timeout_ns;
    int force_dir;  // -1 auto, 0 push, 1 pull
};

// Round snapshot in the control block's RoundState: variant = 0 push / 1 pull,
// qin = active slot, F = active count, round, done.
struct MsLeader {
    long long unexplored;
    uint32_t rounds_push, rounds_pull;
};

__device__ __forceinline__ uint32_t gthread() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint32_t nthreads() { return gridDim.x * blockDim.x; }

__global__ void __launch_bounds__(kMsThreads) msbfs_kernel(MsArgs a) {
    Ctrl *c = a.ctrl;
    engine::set_team(blockIdx.x, gridDim.x, c);
    __shared__ engine::RoundState s;
    engine::Counters *n = &c->cnt;
    const uint32_t lane = dev::lane_id();
    const uint32_t gw = gthread() >> 5, nw = nthreads() >> 5;
    MsLeader L;
    engine::PolicyState ps;  // leader's round state (block 0, thread 0)
    auto nop = [] {};

    // init: masks cleared, levels INF, sources seeded
    for (uint32_t v = gthread(); v < a.nv; v += nthreads()) {
        for (uint32_t f = 0; f < 4; ++f) *a.m.at(f, v) = 0;
    }
    const uint64_t total_lv = (uint64_t)a.nsrc * a.nv;
    for (uint64_t k = gthread(); k < total_lv; k += nthreads()) a.levels[k] = 0xffffffffu;
    for (uint32_t v = gthread(); v < a.nv; v += nthreads()) {
        for (int dir = 0; dir < 2; ++dir) {
            const uint32_t *off = dir == 0 ? a.row : a.crow;
            const uint32_t b = __ldg(off + v), deg = __ldg(off + v + 1) - b;
            if (deg <= kMsChunk) continue;
            const uint32_t nch = (deg + kMsChunk - 1) / kMsChunk;
            const uint32_t c0 = atomicAdd(a.n_chunks + dir, nch);
            for (uint32_t k = 0; k < nch; ++k) {
                if (c0 + k < a.chunk_cap)
                    a.chunks[dir][c0 + k] = make_uint4(v, b + k * kMsChunk, min(kMsChunk, deg - k * kMsChunk), 0);
                else
                    atomicOr(&n->error, dev::kErrChunkCapacity);
            }
        }
    }
    if (!engine::grid_sync(c, a.timeout_ns, nop)) return;
    if (gthread() < a.nsrc) {
        const uint32_t v = a.sources[gthread()];
        const unsigned long long bit = 1ull << gthread();
        atomicOr(a.m.at(kSeen, v), bit);
        const unsigned long long old = atomicOr(a.m.at(kFr0, v), bit);
        if (old == 0) a.active[0][atomicAdd(&n->qcount[0], 1u)] = v;
        a.levels[(uint64_t)gthread() * a.nv + v] = 0;
    }
    auto start = [&] {
        memset(&ps, 0, sizeof ps);
        ps.rs.round = 1;
        ps.rs.qin = 0;
        ps.rs.F = dev::ld_l2(&n->qcount[0]);
        ps.rs.variant = a.force_dir == 1 ? 1 : 0;
        L.unexplored = a.total_edges;
        L.rounds_push = L.rounds_pull = 0;
        const uint4 *src = reinterpret_cast<const uint4 *>(&ps.rs);
        for (int k = 0; k < 4; ++k) __stcg(reinterpret_cast<uint4 *>(&c->rs) + k, src[k]);
    };
    if (!engine::grid_sync(c, a.timeout_ns, start)) return;

    for (;;) {
        if (threadIdx.x < 4)
            reinterpret_cast<uint4 *>(&s)[threadIdx.x] = __ldcg(reinterpret_cast<const uint4 *>(&c->rs) + threadIdx.x);
        __syncthreads();
        if (s.done) break;
        const uint32_t cur = s.qin, nxt = cur ^ 1u;
        unsigned long long edges = 0;
        // ---- phase 1: expand
        // OR a frontier mask into up to four neighbours, col[e + k * stride] for
        // e + k * stride < end: their loads, then their ORs, are in flight
        // together; returns the bits k whose OR was the vertex's first this
        // round (its first writer lists it for phase 2, with one atomic per warp)
        auto push4 = [&](uint32_t e, uint32_t end, uint32_t stride, unsigned long long f, uint32_t(&u)[4]) {
            unsigned long long sn[4], nx[4], old[4];
#pragma unroll
            for (int k = 0; k < 4; ++k)
                u[k] = (uint64_t)e + k * stride < end ? __ldg(a.col + e + k * stride) : kNoVertex;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                sn[k] = nx[k] = ~0ull;
                if (u[k] != kNoVertex) a.m.seen_next(u[k], sn[k], nx[k]);
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const unsigned long long add = f & ~sn[k];
                old[k] = add && (nx[k] & add) != add ? atomicOr(a.m.at(kNext, u[k]), add) : 1ull;
            }
            uint32_t first = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) first |= (old[k] == 0 ? 1u : 0u) << k;
            return first;
        };
        auto warp_or = [](unsigned long long x) {
            for (int d = 16; d > 0; d >>= 1) x |= __shfl_xor_sync(dev::kFullMask, x, d);
            return x;
        };
        const uint32_t n_ch = min(__ldcg(a.n_chunks + s.variant), a.chunk_cap);
        const uint4 *chunks = a.chunks[s.variant];
        if (s.variant == 0) {
            const uint32_t *act = a.active[cur];
            uint32_t u4[4];
            for (uint32_t base = gw * 32; base < s.F; base += nw * 32) {
                const uint32_t i = base + lane;
                uint32_t v = 0, beg = 0, deg = 0;
                unsigned long long f = 0;
                if (i < s.F) {
                    v = __ldcg(act + i);
                    f = __ldcg(a.m.at(kFr0 + cur, v));
                    beg = __ldg(a.row + v);
                    deg = __ldg(a.row + v + 1) - beg;
                }
                if (deg > kMsChunk) deg = 0;  // its chunks are expanded below
                const bool mid = deg > kMsWarp;
                // a thread per vertex, four of its edges per step (all lanes step together)
                const uint32_t mine = mid ? 0u : deg;
                const uint32_t steps = __reduce_max_sync(dev::kFullMask, (mine + 3u) >> 2);
                for (uint32_t st = 0; st < steps; ++st) {
                    const uint32_t first = push4(beg + 4 * st, beg + mine, 1, f, u4);
                    dev::warp_append4(a.touched, &n->middle_count, a.nv, first, u4, &n->error);
                }
                edges += mine;
                uint32_t m = __ballot_sync(dev::kFullMask, mid);
                while (m) {
                    const uint32_t j = __ffs(m) - 1;
                    m &= m - 1;
                    const uint32_t bj = __shfl_sync(dev::kFullMask, beg, j), dj = __shfl_sync(dev::kFullMask, deg, j);
                    const unsigned long long fj = __shfl_sync(dev::kFullMask, f, j);
                    for (uint32_t off = 0; off < dj; off += 128) {
                        const uint32_t first = push4(bj + off + lane, bj + dj, 32, fj, u4);
                        dev::warp_append4(a.touched, &n->middle_count, a.nv, first, u4, &n->error);
                    }
                    if (lane == 0) edges += dj;
                }
            }
            for (uint32_t ch = gw; ch < n_ch; ch += nw) {
                const uint4 c4 = chunks[ch];
                const unsigned long long f = __ldcg(a.m.at(kFr0 + cur, c4.x));
                if (!f) continue;  // not in this round's frontier (the whole warp reads the same chunk)
                for (uint32_t off = 0; off < c4.z; off += 128) {
                    const uint32_t first = push4(c4.y + off + lane, c4.y + c4.z, 32, f, u4);
                    dev::warp_append4(a.touched, &n->middle_count, a.nv, first, u4, &n->error);
                }
                if (lane == 0) edges += c4.z;
            }
        } else {
            // pull: every vertex that misses a source ORs its in-neighbours'
            // frontier masks, stopping once every missing bit is covered
            for (uint32_t base = gw * 32; base < a.nv; base += nw * 32) {
                const uint32_t u = base + lane;
                unsigned long long miss = 0;
                uint32_t b = 0, deg = 0;
                if (u < a.nv) {
                    miss = a.full & ~__ldcg(a.m.at(kSeen, u));
                    if (miss) {
                        b = __ldg(a.crow + u);
                        deg = __ldg(a.crow + u + 1) - b;
                        if (deg > kMsChunk) miss = 0;  // its chunks are scanned below
                    }
                }
                const bool mid = miss && deg > kMsWarp;
                bool hit = false;
                if (miss && !mid) {
                    unsigned long long acc = 0;
                    uint32_t k = b;
                    for (; k < b + deg; ++k) {
                        acc |= __ldcg(a.m.at(kFr0 + cur, __ldg(a.ccol + k)));
                        if ((acc & miss) == miss) {
                            ++k;
                            break;
                        }
                    }
                    edges += k - b;
                    if (acc & miss) {
                        *a.m.at(kNext, u) = acc & miss;
                        hit = true;
                    }
                }
                dev::warp_append(a.touched, &n->middle_count, a.nv, hit, u, &n->error);
                uint32_t m = __ballot_sync(dev::kFullMask, mid);
                while (m) {
                    const uint32_t j = __ffs(m) - 1;
                    m &= m - 1;
                    const uint32_t uj = __shfl_sync(dev::kFullMask, u, j);
                    const uint32_t bj = __shfl_sync(dev::kFullMask, b, j), dj = __shfl_sync(dev::kFullMask, deg, j);
                    const unsigned long long mj = __shfl_sync(dev::kFullMask, miss, j);
                    unsigned long long acc = 0;
                    uint32_t scanned = 0;
                    for (uint32_t off = 0; off < dj; off += 32) {
                        if (off + lane < dj) acc |= __ldcg(a.m.at(kFr0 + cur, __ldg(a.ccol + bj + off + lane)));
                        scanned = min(dj, off + 32);
                        acc = warp_or(acc);
                        if ((acc & mj) == mj) break;
                    }
                    if (lane == 0) {
                        edges += scanned;
                        if (acc & mj) {
                            *a.m.at(kNext, uj) = acc & mj;
                            a.touched[atomicAdd(&n->middle_count, 1u)] = uj;
                        }
                    }
                }
            }
            for (uint32_t ch = gw; ch < n_ch; ch += nw) {
                const uint4 c4 = chunks[ch];
                const unsigned long long miss = a.full & ~__ldcg(a.m.at(kSeen, c4.x));
                if (!miss) continue;
                unsigned long long acc = 0;
                uint32_t scanned = 0;
                for (uint32_t off = 0; off < c4.z; off += 32) {
                    if (off + lane < c4.z) acc |= __ldcg(a.m.at(kFr0 + cur, __ldg(a.ccol + c4.y + off + lane)));
                    scanned = min(c4.z, off + 32);
                    acc = warp_or(acc);
                    if ((acc & miss) == miss) break;
                }
                if (lane == 0) {
                    edges += scanned;
                    if (acc & miss) {
                        const unsigned long long old = atomicOr(a.m.at(kNext, c4.x), acc & miss);
                        if (old == 0) a.touched[atomicAdd(&n->middle_count, 1u)] = c4.x;
                    }
                }
            }
        }
        edges = dev::warp_sum(edges);
        if (lane == 0 && edges) atomicAdd(&n->edges_processed, edges);
        if (!engine::grid_sync(c, a.timeout_ns, nop)) return;
        // ---- phase 2: clear the old frontier, settle the new bits, build the next active list
        {
            const uint32_t *act = a.active[cur];
            for (uint32_t i = gthread(); i < s.F; i += nthreads()) *a.m.at(kFr0 + cur, __ldcg(act + i)) = 0;
            const uint32_t T = __ldcg(&n->middle_count);
            unsigned long long scout = 0, explored = 0;
            for (uint32_t base = gw * 32; base < T; base += nw * 32) {
                const uint32_t i = base + lane;
                uint32_t u = 0;
                unsigned long long nb = 0;
                if (i < T) {
                    u = __ldcg(a.touched + i);  // listed once per round
                    unsigned long long was, nx;
                    a.m.seen_next(u, was, nx);
                    nb = nx & ~was;
                    *a.m.at(kNext, u) = 0;
                    if (nb) {
                        *a.m.at(kSeen, u) = was | nb;
                        *a.m.at(kFr0 + nxt, u) = nb;
                        scout += __ldg(a.row + u + 1) - __ldg(a.row + u);
                        // u now seen by every source: a pull round no longer scans its in-edges
                        if ((was | nb) == a.full) explored += __ldg(a.crow + u + 1) - __ldg(a.crow + u);
                        for (unsigned long long m = nb; m; m &= m - 1)
                            a.levels[(uint64_t)(__ffsll(m) - 1) * a.nv + u] = s.round;
                    }
                }
                dev::warp_append(a.active[nxt], &n->qcount[nxt], a.nv, nb != 0, u, &n->error);
            }
            scout = dev::warp_sum(scout);
            explored = dev::warp_sum(explored);
            if (lane == 0 && scout) atomicAdd(&n->scout[nxt], scout);
            if (lane == 0 && explored) atomicAdd(&n->scout[2], explored);
        }
        auto end_round = [&] {
            const uint32_t F2 = dev::ld_l2(&n->qcount[nxt]);
            const unsigned long long sc = dev::ld_l2(&n->scout[nxt]);
            const unsigned long long ex = dev::ld_l2(&n->scout[2]);
            const bool was_pull = ps.rs.variant == 1;
            if (was_pull) ++L.rounds_pull; else ++L.rounds_push;
            L.unexplored -= (long long)ex;
            if (L.unexplored < 0) L.unexplored = 0;
            n->qcount[cur] = 0;
            n->scout[cur] = 0;
            n->scout[2] = 0;
            n->middle_count = 0;
            ps.rs.qin = nxt;
            ps.rs.F = F2;
            ps.rs.round++;
            if (a.force_dir >= 0)
                ps.rs.variant = a.force_dir;
            else  // the engine's traversal rule (hybrid_policy.h:265-288): stay in pull while the
                  // frontier is large, switch to pull when its edges outweigh the edges a pull
                  // round would scan (in-edges of the vertices some source has not reached)
                ps.rs.variant = ((was_pull && (double)F2 > (double)a.nv / a.beta) ||
                                 (double)sc > (double)L.unexplored / a.alpha) ? 1 : 0;
            if (F2 == 0 || ps.rs.round > a.max_rounds) {
                ps.rs.done = 1;
                c->round = ps.rs.round - 1;
                c->rounds_by_variant[engine::V_ASYNC_PUSH_DD] = L.rounds_push;
                c->rounds_by_variant[engine::V_ASYNC_PULL_DD] = L.rounds_pull;
                c->max_iteration_reached = F2 != 0;
            }
            const uint4 *src = reinterpret_cast<const uint4 *>(&ps.rs);
            for (int k = 0; k < 4; ++k) __stcg(reinterpret_cast<uint4 *>(&c->rs) + k, src[k]);
        };
        if (!engine::grid_sync(c, a.timeout_ns, end_round)) return;
    }
}

// Push-only multi-source BFS with one barrier per round, for sparse graphs
// (average degree below 8: grids, road networks), where push rounds are the
// only ones that pay and hubs are absent.  The vertices discovered in round k
// (list T[p], their new bits pending in next[p]) are settled in round k + 1
// by the thread that expands them: it fixes their seen mask and levels and
// ORs their new bits straight into their neighbours' next[p ^ 1], so the
// two-phase kernel's separate settle pass and its barrier disappear.  A
// neighbour's seen mask read while another thread settles that neighbour may
// miss the bits being settled; the OR then carries bits the neighbour already
// has, which its own settle drops (nb = next & ~seen), so levels are exact.
// Each vertex enters T[p ^ 1] at most once a round (the OR that found its
// next[p ^ 1] zero lists it), and its settle zeroes next[p] again.  Masks:
// fields kSeen and kNext + p (the record's third word holds next[1]).  Round
// state: qin = p, F = |T[p]|, pile = 1 for the settle-only round that ends a
// launch at max_rounds.
__global__ void __launch_bounds__(kMsThreads) msbfs_fused_kernel(MsArgs a) {
    Ctrl *c = a.ctrl;
    engine::set_team(blockIdx.x, gridDim.x, c);
    __shared__ engine::RoundState s;
    engine::Counters *n = &c->cnt;
    const uint32_t lane = dev::lane_id();
    const uint32_t gw = gthread() >> 5, nw = nthreads() >> 5;
    engine::PolicyState ps;  // leader's round state (block 0, thread 0)
    auto nop = [] {};

    for (uint32_t v = gthread(); v < a.nv; v += nthreads()) {
        for (uint32_t f = 0; f < 4; ++f) *a.m.at(f, v) = 0;
    }
    const uint64_t total_lv = (uint64_t)a.nsrc * a.nv;
    for (uint64_t k = gthread(); k < total_lv; k += nthreads()) a.levels[k] = 0xffffffffu;
    if (!engine::grid_sync(c, a.timeout_ns, nop)) return;
    if (gthread() < a.nsrc) {  // the sources' bits pending in next[0], each vertex listed once in T[0]
        const uint32_t v = a.sources[gthread()];
        const unsigned long long old = atomicOr(a.m.at(kNext, v), 1ull << gthread());
        if (old == 0) a.active[0][atomicAdd(&n->qcount[0], 1u)] = v;
    }
    auto start = [&] {
        memset(&ps, 0, sizeof ps);
        ps.rs.round = 0;
        ps.rs.qin = 0;
        ps.rs.F = dev::ld_l2(&n->qcount[0]);
        ps.rs.pile = a.max_rounds == 0 ? 1u : 0u;
        const uint4 *src = reinterpret_cast<const uint4 *>(&ps.rs);
        for (int k = 0; k < 4; ++k) __stcg(reinterpret_cast<uint4 *>(&c->rs) + k, src[k]);
    };
    if (!engine::grid_sync(c, a.timeout_ns, start)) return;

    uint32_t u4[4];
    for (;;) {
        if (threadIdx.x < 4)
            reinterpret_cast<uint4 *>(&s)[threadIdx.x] = __ldcg(reinterpret_cast<const uint4 *>(&c->rs) + threadIdx.x);
        __syncthreads();
        if (s.done) break;
        const uint32_t p = s.qin, q = p ^ 1u;
        const bool expand = s.pile == 0;
        const uint32_t *T = a.active[p];
        unsigned long long edges = 0;
        // OR f into up to four neighbours col[e + k * stride] (e + k * stride < end)
        // of next[q]; returns the bits k whose OR was that vertex's first (it is
        // listed in T[q])
        auto push4 = [&](uint32_t e, uint32_t end, uint32_t stride, unsigned long long f) {
            unsigned long long sn[4], nx[4], old[4];
#pragma unroll
            for (int k = 0; k < 4; ++k)
                u4[k] = (uint64_t)e + k * stride < end ? __ldg(a.col + e + k * stride) : kNoVertex;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                sn[k] = nx[k] = ~0ull;
                if (u4[k] != kNoVertex) {
                    sn[k] = __ldcg(a.m.at(kSeen, u4[k]));
                    nx[k] = __ldcg(a.m.at(kNext + q, u4[k]));
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const unsigned long long add = f & ~sn[k];
                old[k] = add && (nx[k] & add) != add ? atomicOr(a.m.at(kNext + q, u4[k]), add) : 1ull;
            }
            uint32_t first = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) first |= (old[k] == 0 ? 1u : 0u) << k;
            return first;
        };
        for (uint32_t base = gw * 32; base < s.F; base += nw * 32) {
            const uint32_t i = base + lane;
            uint32_t u = 0, beg = 0, deg = 0;
            unsigned long long nb = 0;
            if (i < s.F) {
                u = __ldcg(T + i);
                const unsigned long long was = __ldcg(a.m.at(kSeen, u));
                const unsigned long long nx = __ldcg(a.m.at(kNext + p, u));
                nb = nx & ~was;
                *a.m.at(kNext + p, u) = 0;
                if (nb) {
                    *a.m.at(kSeen, u) = was | nb;
                    for (unsigned long long m = nb; m; m &= m - 1)
                        a.levels[(uint64_t)(__ffsll(m) - 1) * a.nv + u] = s.round;
                    if (expand) {
                        beg = __ldg(a.row + u);
                        deg = __ldg(a.row + u + 1) - beg;
                    }
                }
            }
            // a thread per vertex up to kMsWarp edges, four per step (all lanes step together)
            const bool mid = deg > kMsWarp;
            const uint32_t mine = mid ? 0u : deg;
            const uint32_t steps = __reduce_max_sync(dev::kFullMask, (mine + 3u) >> 2);
            for (uint32_t st = 0; st < steps; ++st) {
                const uint32_t first = push4(beg + 4 * st, beg + mine, 1, nb);
                dev::warp_append4(a.active[q], &n->qcount[q], a.nv, first, u4, &n->error);
            }
            edges += mine;
            // larger lists: a whole warp per vertex
            uint32_t m = __ballot_sync(dev::kFullMask, mid);
            while (m) {
                const uint32_t j = __ffs(m) - 1;
                m &= m - 1;
                const uint32_t bj = __shfl_sync(dev::kFullMask, beg, j), dj = __shfl_sync(dev::kFullMask, deg, j);
                const unsigned long long fj = __shfl_sync(dev::kFullMask, nb, j);
                for (uint32_t off = 0; off < dj; off += 128) {
                    const uint32_t first = push4(bj + off + lane, bj + dj, 32, fj);
                    dev::warp_append4(a.active[q], &n->qcount[q], a.nv, first, u4, &n->error);
                }
                if (lane == 0) edges += dj;
            }
        }
        edges = dev::warp_sum(edges);
        if (lane == 0 && edges) atomicAdd(&n->edges_processed, edges);
        auto end_round = [&] {
            const uint32_t F2 = dev::ld_l2(&n->qcount[q]);
            const uint32_t F_in = ps.rs.F;
            n->qcount[p] = 0;
            const bool settle_only = ps.rs.pile != 0;
            ps.rs.qin = q;
            ps.rs.F = F2;
            ps.rs.round++;
            ps.rs.pile = ps.rs.round >= a.max_rounds ? 1u : 0u;  // the last round settles without expanding
            if (F2 == 0 || settle_only) {
                ps.rs.done = 1;
                c->round = settle_only ? ps.rs.round - 1 : ps.rs.round;  // expanding rounds
                c->rounds_by_variant[engine::V_ASYNC_PUSH_DD] = c->round;
                c->max_iteration_reached = settle_only && F_in != 0;
            }
            const uint4 *src = reinterpret_cast<const uint4 *>(&ps.rs);
            for (int k = 0; k < 4; ++k) __stcg(reinterpret_cast<uint4 *>(&c->rs) + k, src[k]);
        };
        if (!engine::grid_sync(c, a.timeout_ns, end_round)) return;
    }
}

// Edges of the reached component summed over sources: sum_v popcount(seen[v]) * deg(v).
__global__ void msbfs_reach_kernel(const uint32_t *row, MsMasks m, uint32_t nv, unsigned long long *out) {
    unsigned long long e = 0;
    for (uint32_t v = gthread(); v < nv; v += nthreads())
        e += (unsigned long long)__popcll(*m.at(kSeen, v)) * (__ldg(row + v + 1) - __ldg(row + v));
    e = dev::warp_sum(e);
    if ((threadIdx.x & 31) == 0 && e) atomicAdd(out, e);
}

}  // namespace

extern "C" sg_status sg_msbfs(sg_graph *g, const uint32_t *sources, uint32_t nsrc, const sg_options *opt,
                              uint32_t *levels_out, sg_stats *stats) {
    if (!g || !g->ctx) return SG_ERR_INVALID_ARG;
    return sgb::msbfs_on(g->ctx, g, sources, nsrc, opt, levels_out, stats);
}

extern "C" sg_status sg_msbfs_on(sg_ctx *ctx, sg_graph *g, const uint32_t *sources, uint32_t nsrc,
                                 const sg_options *opt, uint32_t *levels_out, sg_stats *stats) {
    if (!ctx || !g || !g->ctx || g->ctx->device != ctx->device) return SG_ERR_INVALID_ARG;
    return sgb::msbfs_on(ctx, g, sources, nsrc, opt, levels_out, stats);
}

// Multi-source BFS on any context of the graph's device; scratch comes from
// that context, so concurrent calls on different contexts never share state.
// With row_outs, row i goes to row_outs[i] (host or device, nv uint32 each)
// and levels_out is ignored.
sg_status sgb::msbfs_on(sg_ctx *ctx, sg_graph *g, const uint32_t *sources, uint32_t nsrc, const sg_options *opt,
                        uint32_t *levels_out, sg_stats *stats, uint32_t *const *row_outs) {
    if (!ctx || !g || !sources || nsrc == 0 || nsrc > 64 || (!levels_out && !row_outs)) return SG_ERR_INVALID_ARG;
    if (row_outs)
        for (uint32_t i = 0; i < nsrc; ++i)
            if (!row_outs[i]) return SG_ERR_INVALID_ARG;
    if (!ctx->batch_ws) ctx->batch_ws = new sgb::Workspace(&ctx->stream, sgb::device_pool(ctx->device));
    for (uint32_t i = 0; i < nsrc; ++i)
        if (sources[i] >= g->nv) return sgb::set_error(ctx, SG_ERR_INVALID_ARG, "source %u out of range", sources[i]);
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != ctx->device) cudaSetDevice(ctx->device);
    struct Restore {
        int p, d;
        ~Restore() {
            if (p >= 0 && p != d) cudaSetDevice(p);
        }
    } restore{prev, ctx->device};
    sg_options o;
    if (opt)
        o = *opt;
    else
        sg_options_default(&o);
    const uint32_t nv = g->nv;
    auto &ws = *ctx->batch_ws;
    MsArgs a;
    std::memset(&a, 0, sizeof a);
    a.row = g->row;
    a.col = g->col;
    a.crow = g->has_csc ? g->crow : g->row;
    a.ccol = g->has_csc ? g->ccol : g->col;
    a.nv = nv;
    a.nsrc = nsrc;
    a.full = nsrc == 64 ? ~0ull : ((1ull << nsrc) - 1);
    SG_TRY_CUDA(ctx, ws.get("ms_masks", 4ull * nv, &a.m.base));
    const bool interleaved = g->ne < 8ull * nv;  // average degree below 8
    a.m.fstride = interleaved ? 1 : nv;
    a.m.vstride = interleaved ? 4 : 1;
    SG_TRY_CUDA(ctx, ws.get("q0", nv, &a.active[0]));
    SG_TRY_CUDA(ctx, ws.get("q1", nv, &a.active[1]));
    SG_TRY_CUDA(ctx, ws.get("middle", nv, &a.touched));
    SG_TRY_CUDA(ctx, ws.get("ctrl", 1, &a.ctrl));
    // at most sum over split vertices of (deg / kMsChunk + 1) <= 2 * E / kMsChunk chunks per direction
    a.chunk_cap = (uint32_t)std::min<uint64_t>(2 * (g->ne / kMsChunk) + 2, 0xffffffffu);
    SG_TRY_CUDA(ctx, ws.get("ms_chunks_out", a.chunk_cap, &a.chunks[0]));
    SG_TRY_CUDA(ctx, ws.get("ms_chunks_in", a.chunk_cap, &a.chunks[1]));
    SG_TRY_CUDA(ctx, ws.get("ms_n_chunks", 2, &a.n_chunks));
    SG_TRY_CUDA(ctx, cudaMemsetAsync(a.n_chunks, 0, 2 * sizeof(uint32_t), ctx->stream));
    uint32_t *dsrc = nullptr;
    SG_TRY_CUDA(ctx, ws.get("ms_sources", 64, &dsrc));
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(dsrc, sources, 4 * nsrc, cudaMemcpyHostToDevice, ctx->stream));
    a.sources = dsrc;
    const bool out_dev = !row_outs && sgb::is_device_ptr(levels_out, ctx->device);
    if (out_dev)
        a.levels = levels_out;
    else
        SG_TRY_CUDA(ctx, ws.get("ms_levels", (size_t)nsrc * nv, &a.levels));
    a.max_rounds = o.max_iteration > 0 ? (uint32_t)o.max_iteration : 200u;
    a.alpha = o.alpha > 0 ? o.alpha : 15;
    a.beta = o.beta > 0 ? o.beta : 18;
    a.total_edges = (long long)g->ne;
    a.timeout_ns = (unsigned long long)((o.timeout_s > 0 ? o.timeout_s : 30.0) * 1e9);
    a.force_dir = o.variant == SG_ASYNC_PUSH_DD ? 0 : (o.variant == SG_ASYNC_PULL_DD ? 1 : -1);
    if (!g->has_csc && !g->symmetric) a.force_dir = 0;

    // sparse graphs run push-only with one barrier per round (msbfs_fused_kernel)
    // unless pull is forced; the rest take the two-phase push/pull kernel
    const bool fused = interleaved && a.force_dir != 1;
    const void *kernel = fused ? (const void *)msbfs_fused_kernel : (const void *)msbfs_kernel;
    static std::atomic<int> occupancy[2] = {{0}, {0}};
    int bps = 0;
    SG_TRY_CUDA(ctx, sgb::occupancy_once(occupancy[fused ? 1 : 0], kernel, kMsThreads, &bps));
    const int want = o.blocks_per_sm > 0 ? o.blocks_per_sm : sgb::ms_blocks_per_sm(nv, g->ne, nsrc);
    dim3 grid(ctx->prop.multiProcessorCount * std::max(1, std::min(sgb::resident_blocks_per_sm(ctx, bps), want)));
    SG_TRY_CUDA(ctx, cudaMemsetAsync(a.ctrl, 0, sizeof(Ctrl), ctx->stream));
    SG_TRY_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    void *args[] = {&a};
    SG_TRY_CUDA(ctx, cudaLaunchCooperativeKernel(kernel, grid, dim3(kMsThreads), args, 0, ctx->stream));
    SG_TRY_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    if (!o.blocking) return SG_OK;
    Ctrl h;
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(&h, a.ctrl, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    if (row_outs) {
        for (uint32_t i = 0; i < nsrc; ++i)
            SG_TRY_CUDA(ctx, cudaMemcpyAsync(row_outs[i], a.levels + (size_t)i * nv, 4ull * nv, cudaMemcpyDefault,
                                             ctx->stream));
    } else if (!out_dev) {
        SG_TRY_CUDA(ctx, cudaMemcpyAsync(levels_out, a.levels, 4ull * nsrc * nv, cudaMemcpyDeviceToHost, ctx->stream));
    }
    unsigned long long *dr = nullptr, reach = 0;
    SG_TRY_CUDA(ctx, ws.get("reach_stats", 3, &dr));
    SG_TRY_CUDA(ctx, cudaMemsetAsync(dr, 0, 8, ctx->stream));
    msbfs_reach_kernel<<<ctx->prop.multiProcessorCount * 4, 256, 0, ctx->stream>>>(g->row, a.m, nv, dr);
    SG_TRY_CUDA(ctx, cudaGetLastError());
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(&reach, dr, 8, cudaMemcpyDeviceToHost, ctx->stream));
    SG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    SG_TRY_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    const uint32_t bits = h.cnt.error;
    if (stats) {
        stats->rounds = h.round;
        stats->max_iteration_reached = h.max_iteration_reached;
        for (int k = 0; k < 8; ++k) stats->rounds_by_variant[k] = h.rounds_by_variant[k];
        stats->time_total_ms = stats->time_kernel_ms = ms;
        stats->edges_processed = h.cnt.edges_processed;
        stats->edges_reached = reach;
        stats->device_error = bits;
    }
    const sg_status st = sgb::device_error_status(bits);
    if (st != SG_OK) return sgb::set_error(ctx, st, "msbfs device error bits 0x%x", bits);
    return SG_OK;
}

// ---------------------------------------------------------------- many queries, one launch
namespace {

// Edges of the reached component of each query's value array (unreached = UINT32_MAX).
__global__ void batch_reach_kernel(const uint32_t *const *rows, const uint32_t *const *vals, const uint32_t *nvs,
                                   unsigned long long *out) {
    const uint32_t q = blockIdx.y;
    const uint32_t *row = rows[q], *val = vals[q];
    const uint32_t nv = nvs[q];
    unsigned long long e = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
        if (val[v] != 0xffffffffu) e += __ldg(row + v + 1) - __ldg(row + v);
    e = dev::warp_sum(e);
    if ((threadIdx.x & 31) == 0 && e) atomicAdd(out + q, e);
}

// ---------------------------------------------------------------- batched BC
// Per-team state of Brandes' two passes, sized for the largest graph.
struct BCTeam {
    uint32_t *level;  // forward levels (the engine's value array)
    unsigned long long *sigma;
    float *delta;
    uint32_t *stack, *ends, *misc, *ccount;  // misc: 0 stack count, 1 levels closed, 2 search depth, 3 error bits
    uint4 *chunks;
    uint32_t chunk_cap, max_levels;
};

using BCApp = apps::BCForward<uint32_t, uint32_t, graphs::NoWeight>;

// Each team claims a query, runs the hybrid forward pass (BCForward through the
// same round loop as a single query) and then the backward pass over its own
// level stack with team barriers, and writes delta * 0.5 to the query's
// output.  Forward and backward of different queries overlap across teams.
__global__ void __launch_bounds__(engine::kBlockThreads)
    batched_bc_kernel(const engine::BatchQuery<BCApp, uint32_t> *queries, uint32_t nq,
                      const engine::TeamSpace<uint32_t> *spaces, const BCTeam *bcs, float *const *outs,
                      uint32_t team_blocks, uint32_t *next_query, engine::BatchResult *results, engine::Params p) {
    using namespace engine;
    const uint32_t team = blockIdx.x / team_blocks;
    const TeamSpace<uint32_t> &sp = spaces[team];
    const BCTeam bt = bcs[team];
    Ctrl *c = sp.ctrl;
    set_team(blockIdx.x % team_blocks, team_blocks, c);
    const uint32_t gt = g_team_rank * blockDim.x + threadIdx.x, nt = g_team_size * blockDim.x;
    __shared__ uint32_t s_q, s_misc[4];
    auto nop = [] {};
    for (;;) {
        auto claim = [&] {
            const uint32_t q = atomicAdd(next_query, 1u);
            unsigned char *z = reinterpret_cast<unsigned char *>(&c->rs);
            memset(z, 0, sizeof(Ctrl) - offsetof(Ctrl, rs));
            c->pad0 = q;
            for (int k = 0; k < 4; ++k) bt.misc[k] = 0;
        };
        if (!grid_sync(c, p.timeout_ns, claim)) return;
        if (threadIdx.x == 0) s_q = dev::ld_l2(&c->pad0);
        __syncthreads();
        const uint32_t q = s_q;
        if (q >= nq) return;
        const BatchQuery<BCApp, uint32_t> &bq = queries[q];
        const uint32_t nv = bq.csr.nnodes;
        // sigma[source] = 1, every other path count and dependency 0 (hybrid_bc.cu:325-326);
        // the engine's first team barrier orders these writes before the forward pass
        for (uint32_t v = gt; v < nv; v += nt) {
            bt.sigma[v] = v == bq.app.m_source_node ? 1ull : 0ull;
            bt.delta[v] = 0.f;
        }
        for (uint32_t k = gt; k < bt.max_levels; k += nt) bt.ccount[k] = 0;
        KArgs<uint32_t, uint32_t, graphs::NoWeight> a;
        a.csr = bq.csr;
        a.csc = bq.csc;
        a.csr_w = bq.csr_w;
        a.csc_w = bq.csc_w;
        a.value = bt.level;
        a.buffer = sp.buffer;
        a.tmp = sp.tmp;
        for (int k = 0; k < 3; ++k) {
            a.queue[k] = sp.queue[k];
            a.qflag[k] = sp.qflag[k];
        }
        a.bitmap[0] = sp.bitmap[0];
        a.bitmap[1] = sp.bitmap[1];
        a.queue_cap = nv;
        a.nwords = nv / 32 + 1;
        a.middle = sp.middle;
        a.heavy = sp.heavy;
        a.heavy_cap = sp.heavy_cap;
        a.chunk_owner = sp.chunk_owner;
        a.chunk_cap = sp.chunk_cap;
        a.ctrl = c;
        a.trace = nullptr;
        a.trace_cap = 0;
        a.p = p;
        a.p.total_workload0 = (long long)bq.csr.nedges;
        BCApp app = bq.app;
        app.m_sigmas = bt.sigma;
        app.m_p_search_depth = bt.misc + 2;
        app.m_stack = apps::LevelStack{bt.stack, bt.misc + 0, bt.ends, bt.misc + 1, nv, bt.max_levels, bt.misc + 3};
        app.m_p_current_round = &c->rs.round;
        if (!run_instance<BCApp, uint32_t, uint32_t, graphs::NoWeight>(app, a)) return;
        if (threadIdx.x < 4) s_misc[threadIdx.x] = dev::ld_l2(bt.misc + threadIdx.x);
        __syncthreads();
        const uint32_t nlevels = s_misc[1], depth = s_misc[2], ferr = s_misc[3];
        // reached edges of the forward traversal (GTEPS numerator)
        unsigned long long e = 0;
        for (uint32_t v = gt; v < nv; v += nt)
            if (__ldcg(bt.level + v) != 0xffffffffu) e += bq.csr.end_edge(v) - bq.csr.begin_edge(v);
        e = dev::warp_sum(e);
        if (dev::lane_id() == 0 && e) atomicAdd(&results[q].reached, e);
        bc::BCBackArgs ba;
        ba.row = bq.csr.row_start;
        ba.col = bq.csr.edge_dst;
        ba.level = bt.level;
        ba.sigma = bt.sigma;
        ba.delta = bt.delta;
        ba.bc_out = outs[q];
        ba.stack = bt.stack;
        ba.ends = bt.ends;
        ba.nlevels = nlevels;
        ba.max_depth = (ferr == 0 && depth >= 2) ? min(depth - 1, nlevels ? nlevels - 1 : 0u) : 0u;
        ba.nv = nv;
        ba.chunks = bt.chunks;
        ba.chunk_cap = bt.chunk_cap;
        ba.chunk_count = bt.ccount;
        ba.bar = nullptr;
        ba.err = bt.misc + 3;
        ba.timeout_ns = p.timeout_ns;
        auto sync = [&] { return grid_sync(c, p.timeout_ns, nop); };
        if (!bc::backward(ba, gt, nt, sync)) return;
        // the result record follows every block's output writes
        auto record = [&] { write_result(results + q, c, team, dev::ld_l2(bt.misc + 3), dev::globaltimer_ns()); };
        if (!grid_sync(c, p.timeout_ns, record)) return;
    }
}

template <typename T>
sg_status ws_get(sg_ctx *ctx, sgb::Workspace &ws, const char *name, size_t n, T **out) {
    SG_TRY_CUDA(ctx, ws.get(name, n, out));
    return SG_OK;
}

// Everything one batched launch needs once its descriptors are on the device:
// the kernel, its grid and argument values (their addresses are the launch's
// argument array, so a Build must stay put while it is enqueued or captured),
// the buffers to zero before each launch and the host-side bookkeeping.
struct BatchBuild {
    const void *kernel = nullptr;
    uint32_t n = 0, n_teams = 0, team_blocks = 0;
    void *dq = nullptr, *dsp = nullptr, *dbc = nullptr, *douts = nullptr;
    uint32_t *counter = nullptr;
    engine::BatchResult *dres = nullptr;
    engine::Params p{};
    void *args[9] = {};
    struct Zero {
        void *ptr;
        size_t bytes;
    };
    std::vector<Zero> zero;
    std::vector<uint32_t> order;         // launch position -> query index
    std::vector<sg_graph *> graphs;      // by query index
    std::vector<void *> outs, vptr;      // caller output, device array written by the kernel
    std::vector<bool> out_dev;
    bool bc = false;
    size_t value_bytes = 4;
};

// Zeroes the per-launch state and launches; no host synchronisation (capturable).
sg_status enqueue_batch(sg_ctx *ctx, BatchBuild &B, cudaStream_t s) {
    for (auto &z : B.zero) SG_TRY_CUDA(ctx, cudaMemsetAsync(z.ptr, 0, z.bytes, s));
    SG_TRY_CUDA(ctx, cudaLaunchCooperativeKernel(B.kernel, dim3(B.n_teams * B.team_blocks), dim3(engine::kBlockThreads),
                                                 B.args, 0, s));
    return SG_OK;
}

// Plans n queries of one functor type as one batched launch: team sizing,
// team workspaces and query descriptors in `ws`, outputs in place (device) or
// through a staging array (host).  With device_outputs_only, host outputs are
// rejected (a captured launch cannot copy to pageable memory).
template <typename App, typename TV, typename TB, typename TW>
sg_status prepare_batch(sg_ctx *ctx, sgb::Workspace &ws, std::vector<engine::BatchQuery<App, TV>> qs,
                        const std::vector<sg_graph *> &graphs, const std::vector<void *> &outs, const sg_options &o,
                        engine::Params p, bool device_outputs_only, BatchBuild &B) {
    using namespace engine;
    const uint32_t n = (uint32_t)qs.size();
    B.n = n;
    B.graphs = graphs;
    B.outs = outs;
    // largest graphs first (longest-processing-time order)
    B.order.resize(n);
    for (uint32_t i = 0; i < n; ++i) B.order[i] = i;
    std::stable_sort(B.order.begin(), B.order.end(), [&](uint32_t x, uint32_t y) { return graphs[x]->ne > graphs[y]->ne; });
    uint32_t nv_max = 0;
    uint64_t ne_max = 0;
    for (auto *g : graphs) {
        nv_max = std::max(nv_max, g->nv);
        ne_max = std::max(ne_max, g->ne);
    }
    constexpr bool kBC = std::is_same<App, BCApp>::value;
    B.bc = kBC;
    B.value_bytes = sizeof(TV);
    B.kernel = kBC ? (const void *)batched_bc_kernel : (const void *)batched_engine_kernel<App, TV, TB, TW>;
    static std::atomic<int> occupancy{0};  // one per template instantiation
    int max_bps = 0;
    SG_TRY_CUDA(ctx, sgb::occupancy_once(occupancy, B.kernel, kBlockThreads, &max_bps));
    const int bps =
        std::max(1, std::min(sgb::resident_blocks_per_sm(ctx, max_bps), o.blocks_per_sm > 0 ? o.blocks_per_sm : 4));
    const uint32_t total_blocks = (uint32_t)(ctx->prop.multiProcessorCount * bps);
    // Automatic team size.  Equal teams claim queries largest first, so the
    // batch lasts at least as long as its largest query on one team: a team
    // gets 4x its edge-proportional share of the grid, blocks * 4 * ne_max /
    // sum(ne), and at least one block per 2M edges of the largest graph; but
    // the grid keeps at least min(n, 16) teams, because queries on
    // high-diameter graphs are bound by their round count, not their edges,
    // and gain from running side by side.  Measured on B200 (592 blocks): 256
    // SSSP queries over RMAT scales 12-20 ran in 27-30 ms with 24-49 blocks
    // per team against 72 ms with 7; 256 on RMAT-14 fastest with 8-10; 64 BFS
    // on RMAT-22 flat from 24 to 148; mixed RMAT/grid server batches lost half
    // their throughput with one or two large teams.
    uint32_t team_blocks = (uint32_t)o.team_blocks;
    if (o.team_blocks <= 0) {
        uint64_t sum_ne = 0;
        for (auto *g : graphs) sum_ne += g->ne;
        const uint64_t share = (4ull * total_blocks * ne_max + sum_ne - 1) / std::max<uint64_t>(1, sum_ne);
        const uint64_t cap = std::max<uint64_t>(1, total_blocks / std::min(n, 16u));
        team_blocks = (uint32_t)std::max<uint64_t>(1, std::min(std::max(ne_max >> 21, share), cap));
    }
    team_blocks = std::max(1u, std::min(team_blocks, total_blocks));
    const uint32_t n_teams = std::max(1u, std::min(n, total_blocks / team_blocks));
    B.team_blocks = team_blocks;
    B.n_teams = n_teams;

    // team workspaces
    const uint32_t nwords = nv_max / 32 + 1;
    const uint32_t heavy_cap = (uint32_t)std::min<uint64_t>(nv_max, ne_max / std::max(1u, p.heavy_threshold)) + 2;
    // chunks are cut on the 4-edge grid: at most one more per heavy vertex than deg / chunk_edges rounded up
    const uint32_t chunk_cap = (uint32_t)(ne_max / p.chunk_edges + 2ull * heavy_cap + 2);
    TB *buf, *tmp;
    uint32_t *qq, *bm, *fl, *mid, *chunk, *counter;
    HeavyItem<TB> *heavy;
    Ctrl *ctrl;
    const size_t T = n_teams;
    sg_status st;
    if ((st = ws_get(ctx, ws, "b_buf", T * nv_max, &buf)) != SG_OK) return st;
    if ((st = ws_get(ctx, ws, "b_tmp", T * nv_max, &tmp)) != SG_OK) return st;
    if ((st = ws_get(ctx, ws, "b_q", T * 3 * nv_max, &qq)) != SG_OK) return st;
    if ((st = ws_get(ctx, ws, "b_bm", T * 2 * nwords, &bm)) != SG_OK) return st;
    if ((st = ws_get(ctx, ws, "b_fl", T * 3 * nwords, &fl)) != SG_OK) return st;
    if ((st = ws_get(ctx, ws, "b_mid", T * nv_max, &mid)) != SG_OK) return st;
    // two heavy-vertex tables per team (one per round parity)
    if ((st = ws_get(ctx, ws, "b_heavy", T * 2 * heavy_cap, &heavy)) != SG_OK) return st;
    if ((st = ws_get(ctx, ws, "b_chunk", T * 2 * chunk_cap, &chunk)) != SG_OK) return st;
    if ((st = ws_get(ctx, ws, "b_ctrl", T, &ctrl)) != SG_OK) return st;
    if ((st = ws_get(ctx, ws, "b_counter", 1, &counter)) != SG_OK) return st;
    // heavy/chunk tables start zeroed so that a stale chunk never names an out-of-range item
    B.zero.push_back({heavy, T * 2 * heavy_cap * sizeof(HeavyItem<TB>)});
    B.zero.push_back({ctrl, T * sizeof(Ctrl)});
    B.zero.push_back({counter, sizeof(uint32_t)});
    B.counter = counter;
    std::vector<TeamSpace<TB>> spaces(T);
    for (size_t t = 0; t < T; ++t) {
        TeamSpace<TB> &s = spaces[t];
        s.buffer = buf + t * nv_max;
        s.tmp = tmp + t * nv_max;
        for (int k = 0; k < 3; ++k) {
            s.queue[k] = qq + (t * 3 + k) * nv_max;
            s.qflag[k] = fl + (t * 3 + k) * nwords;
        }
        s.bitmap[0] = bm + (t * 2) * nwords;
        s.bitmap[1] = bm + (t * 2 + 1) * nwords;
        s.middle = mid + t * nv_max;
        s.heavy = heavy + t * 2 * heavy_cap;
        s.chunk_owner = chunk + t * 2 * chunk_cap;
        s.ctrl = ctrl + t;
        s.trace = nullptr;
        s.cap_v = nv_max;
        s.heavy_cap = heavy_cap;
        s.chunk_cap = chunk_cap;
        s.trace_cap = 0;
    }
    // BC: levels, path counts, dependencies, level stack and chunk table per team
    if constexpr (kBC) {
        const uint32_t max_levels = std::min(p.max_iteration, nv_max) + 2;  // a level holds at least one vertex
        const uint32_t bchunk_cap = (uint32_t)(ne_max / bc::kBcChunk + ne_max / bc::kBcBigDegree + 2);
        uint32_t *lv, *stk, *ends, *misc, *cc;
        unsigned long long *sig;
        float *dl;
        uint4 *bch;
        BCTeam *dbc;
        if ((st = ws_get(ctx, ws, "bc_level", T * nv_max, &lv)) != SG_OK) return st;
        if ((st = ws_get(ctx, ws, "bc_sigma", T * nv_max, &sig)) != SG_OK) return st;
        if ((st = ws_get(ctx, ws, "bc_delta", T * nv_max, &dl)) != SG_OK) return st;
        if ((st = ws_get(ctx, ws, "bc_stack", T * nv_max, &stk)) != SG_OK) return st;
        if ((st = ws_get(ctx, ws, "bc_ends", T * max_levels, &ends)) != SG_OK) return st;
        if ((st = ws_get(ctx, ws, "bc_ccount", T * max_levels, &cc)) != SG_OK) return st;
        if ((st = ws_get(ctx, ws, "bc_misc", T * 4, &misc)) != SG_OK) return st;
        if ((st = ws_get(ctx, ws, "bc_chunks", T * bchunk_cap, &bch)) != SG_OK) return st;
        std::vector<BCTeam> bts(T);
        for (size_t t = 0; t < T; ++t)
            bts[t] = BCTeam{lv + t * nv_max, sig + t * nv_max, dl + t * nv_max, stk + t * nv_max, ends + t * max_levels,
                            misc + t * 4, cc + t * max_levels, bch + t * bchunk_cap, bchunk_cap, max_levels};
        if ((st = ws_get(ctx, ws, "bc_teams", T, &dbc)) != SG_OK) return st;
        SG_TRY_CUDA(ctx, cudaMemcpyAsync(dbc, bts.data(), T * sizeof(BCTeam), cudaMemcpyHostToDevice, ctx->stream));
        B.dbc = dbc;
    }
    // outputs: device outputs are written in place, host outputs go through a staging array
    B.out_dev.assign(n, false);
    TV *stage = nullptr;
    size_t stage_elems = 0;
    for (uint32_t i = 0; i < n; ++i) {
        B.out_dev[i] = sgb::is_device_ptr(outs[i], ctx->device);
        if (!B.out_dev[i]) {
            if (device_outputs_only) return sgb::set_error(ctx, SG_ERR_INVALID_ARG, "batch plan output %u is not device memory", i);
            stage_elems += graphs[i]->nv;
        }
    }
    if (stage_elems && (st = ws_get(ctx, ws, "b_stage", stage_elems, &stage)) != SG_OK) return st;
    B.vptr.assign(n, nullptr);
    {
        size_t off = 0;
        for (uint32_t i = 0; i < n; ++i) {
            B.vptr[i] = B.out_dev[i] ? outs[i] : (void *)(stage + off);
            if (!B.out_dev[i]) off += graphs[i]->nv;
        }
    }
    std::vector<BatchQuery<App, TV>> qd;
    qd.reserve(n);
    std::vector<float *> fouts(n);
    for (uint32_t k = 0; k < n; ++k) {
        qd.push_back(qs[B.order[k]]);
        qd.back().value = (TV *)B.vptr[B.order[k]];
        fouts[k] = reinterpret_cast<float *>(B.vptr[B.order[k]]);  // BC writes 4-byte floats in the same slots
    }
    if constexpr (kBC) {
        float **douts;
        if ((st = ws_get(ctx, ws, "bc_outs", n, &douts)) != SG_OK) return st;
        SG_TRY_CUDA(ctx, cudaMemcpyAsync(douts, fouts.data(), n * sizeof(float *), cudaMemcpyHostToDevice, ctx->stream));
        B.douts = douts;
    }
    BatchQuery<App, TV> *dq;
    TeamSpace<TB> *dsp;
    if ((st = ws_get(ctx, ws, "b_queries", n, &dq)) != SG_OK) return st;
    if ((st = ws_get(ctx, ws, "b_spaces", T, &dsp)) != SG_OK) return st;
    if ((st = ws_get(ctx, ws, "b_results", n, &B.dres)) != SG_OK) return st;
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(dq, qd.data(), n * sizeof(qd[0]), cudaMemcpyHostToDevice, ctx->stream));
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(dsp, spaces.data(), T * sizeof(spaces[0]), cudaMemcpyHostToDevice, ctx->stream));
    B.zero.push_back({B.dres, n * sizeof(BatchResult)});
    B.dq = dq;
    B.dsp = dsp;
    B.p = p;
    if (kBC) {
        void *a[] = {&B.dq, &B.n, &B.dsp, &B.dbc, &B.douts, &B.team_blocks, &B.counter, &B.dres, &B.p};
        std::copy(a, a + 9, B.args);
    } else {
        void *a[] = {&B.dq, &B.n, &B.dsp, &B.team_blocks, &B.counter, &B.dres, &B.p};
        std::copy(a, a + 7, B.args);
    }
    return SG_OK;
}

// After a launch: outputs to the host, per-query results, aggregate stats.
sg_status finish_batch(sg_ctx *ctx, sgb::Workspace &ws, BatchBuild &B, bool copy_outputs, sg_stats *stats,
                       float *per_query_ms) {
    using namespace engine;
    const uint32_t n = B.n;
    sg_status st;
    std::vector<BatchResult> res(n);
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(res.data(), B.dres, n * sizeof(BatchResult), cudaMemcpyDeviceToHost, ctx->stream));
    if (copy_outputs)
        for (uint32_t i = 0; i < n; ++i)
            if (!B.out_dev[i])
                SG_TRY_CUDA(ctx, cudaMemcpyAsync(B.outs[i], B.vptr[i], B.graphs[i]->nv * B.value_bytes,
                                                 cudaMemcpyDeviceToHost, ctx->stream));
    // reached edges per query (GTEPS numerator)
    unsigned long long reached = 0;
    if (stats && !B.bc) {
        const uint32_t **rows, **vals;
        uint32_t *nvs;
        unsigned long long *dr;
        if ((st = ws_get(ctx, ws, "b_rows", n, (const uint32_t ***)&rows)) != SG_OK) return st;
        if ((st = ws_get(ctx, ws, "b_vals", n, (const uint32_t ***)&vals)) != SG_OK) return st;
        if ((st = ws_get(ctx, ws, "b_nvs", n, &nvs)) != SG_OK) return st;
        if ((st = ws_get(ctx, ws, "b_reach", n, &dr)) != SG_OK) return st;
        std::vector<const uint32_t *> hr(n), hv(n);
        std::vector<uint32_t> hn(n);
        for (uint32_t i = 0; i < n; ++i) {
            hr[i] = B.graphs[i]->row;
            hv[i] = (const uint32_t *)B.vptr[i];
            hn[i] = B.graphs[i]->nv;
        }
        SG_TRY_CUDA(ctx, cudaMemcpyAsync(rows, hr.data(), n * sizeof(void *), cudaMemcpyHostToDevice, ctx->stream));
        SG_TRY_CUDA(ctx, cudaMemcpyAsync(vals, hv.data(), n * sizeof(void *), cudaMemcpyHostToDevice, ctx->stream));
        SG_TRY_CUDA(ctx, cudaMemcpyAsync(nvs, hn.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
        SG_TRY_CUDA(ctx, cudaMemsetAsync(dr, 0, n * sizeof(unsigned long long), ctx->stream));
        if (B.value_bytes == 4) {
            batch_reach_kernel<<<dim3(64, n), 256, 0, ctx->stream>>>(rows, vals, nvs, dr);
            SG_TRY_CUDA(ctx, cudaGetLastError());
        }
        std::vector<unsigned long long> hreach(n);
        SG_TRY_CUDA(ctx, cudaMemcpyAsync(hreach.data(), dr, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                         ctx->stream));
        SG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        for (auto x : hreach) reached += x;
    }
    SG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    SG_TRY_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    uint32_t bits = 0;
    std::vector<BatchResult> byq(n);
    for (uint32_t k = 0; k < n; ++k) {
        byq[B.order[k]] = res[k];
        bits |= res[k].error;
        if (B.bc) reached += 2 * res[k].reached;  // two traversals, as for a single BC query
    }
    if (stats) {
        std::memset(stats->rounds_by_variant, 0, sizeof stats->rounds_by_variant);
        stats->rounds = 0;
        stats->edges_processed = 0;
        stats->max_iteration_reached = 0;
        for (auto &r : byq) {
            stats->rounds = std::max(stats->rounds, r.rounds);
            for (int k = 0; k < 8; ++k) stats->rounds_by_variant[k] += r.rounds_by_variant[k];
            stats->edges_processed += r.edges_processed;
            stats->max_iteration_reached |= r.max_iteration_reached;
        }
        stats->time_total_ms = stats->time_kernel_ms = ms;
        stats->edges_reached = reached;
        stats->vertices_processed = n;  // queries in the batch
        stats->device_error = bits;
        stats->search_depth = B.n_teams;  // teams used
        stats->vertices_reached = B.team_blocks;
    }
    if (per_query_ms)
        for (uint32_t i = 0; i < n; ++i) per_query_ms[i] = (float)((byq[i].t_end - byq[i].t_start) * 1e-6);
    const sg_status dst = sgb::device_error_status(bits);
    if (dst != SG_OK) return sgb::set_error(ctx, dst, "batch device error bits 0x%x", bits);
    return SG_OK;
}

// Runs n queries of one functor type in one batched launch.  outs[i] receives
// query i's value array (host or device memory of nv_i elements).
template <typename App, typename TV, typename TB, typename TW>
sg_status run_batch(sg_ctx *ctx, std::vector<engine::BatchQuery<App, TV>> qs, const std::vector<sg_graph *> &graphs,
                    const std::vector<void *> &outs, const sg_options &o, engine::Params p, sg_stats *stats,
                    float *per_query_ms) {
    if (!ctx->batch_ws) ctx->batch_ws = new sgb::Workspace(&ctx->stream, sgb::device_pool(ctx->device));
    BatchBuild B;
    sg_status st = prepare_batch<App, TV, TB, TW>(ctx, *ctx->batch_ws, std::move(qs), graphs, outs, o, p, false, B);
    if (st != SG_OK) return st;
    SG_TRY_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    if ((st = enqueue_batch(ctx, B, ctx->stream)) != SG_OK) return st;
    SG_TRY_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    if (!o.blocking) return SG_OK;
    return finish_batch(ctx, *ctx->batch_ws, B, true, stats, per_query_ms);
}

engine::Params batch_params(const sg_options &o, int scheme) {
    engine::Params p;
    std::memset(&p, 0, sizeof p);
    p.scheme = scheme;
    p.forced = o.variant;
    if (o.alpha == 0) p.forced = engine::V_ASYNC_PUSH_DD;
    p.lb_push = o.lb_push >= 0 ? o.lb_push : engine::LB_FINE;
    p.lb_pull = o.lb_pull >= 0 ? o.lb_pull : engine::LB_FINE;
    p.collect = p.forced < 0 ? 1 : 0;
    p.has_csc = 1;
    p.max_iteration = o.max_iteration > 0 ? (uint32_t)o.max_iteration : 200u;
    p.heavy_threshold = o.heavy_degree > 0 ? (uint32_t)o.heavy_degree : 32u;
    p.chunk_edges = o.chunk_edges > 0 ? ((uint32_t)std::max(32, o.chunk_edges) + 3u) & ~3u : 256u;
    p.pull_warp_threshold = 32;
    p.local_depth = o.local_depth > 0 ? (uint32_t)o.local_depth : 0u;
    p.sample_cut = o.priority == SG_PRIORITY_SAMPLING && o.cut_threshold > 0 ? (float)std::min(o.cut_threshold, 1.0) : 0.f;
    p.bitmap_frontier = engine::use_bitmap_frontier(p.forced, p.lb_push, false, o.worklist);
    p.pull_coop = o.pull_scan == SG_PULL_SCAN_WARP;
    p.stage_chunks = o.hub_stage >= 0;
    p.alpha = o.alpha;
    p.beta = o.beta > 0 ? o.beta : 18;
    p.timeout_ns = (unsigned long long)((o.timeout_s > 0 ? o.timeout_s : 30.0) * 1e9);
    return p;
}

template <typename App>
engine::BatchQuery<App, uint32_t> make_query(App app, sg_graph *g) {
    engine::BatchQuery<App, uint32_t> bq{app, {}, {}, nullptr, nullptr, nullptr, 0ull};
    bq.csr.nnodes = g->nv;
    bq.csr.nedges = (uint32_t)g->ne;
    bq.csr.row_start = g->row;
    bq.csr.edge_dst = g->col;
    bq.csr.edge_weights = g->w;
    bq.csc.nnodes = g->nv;
    bq.csc.nedges = (uint32_t)g->ne;
    bq.csc.col_start = g->crow ? g->crow : g->row;
    bq.csc.edge_source = g->ccol ? g->ccol : g->col;
    bq.csc.edge_weights = g->cw;
    bq.csc.csr_row_start = g->row;
    bq.csr_w = g->w;
    bq.csc_w = g->cw;
    bq.value = nullptr;
    app.m_csr_graph = bq.csr;
    app.m_csc_graph = bq.csc;
    app.m_nnodes = g->nv;
    app.m_nedges = (uint32_t)g->ne;
    bq.app = app;
    return bq;
}

// The reference's delta heuristic, 32 * average weight / average degree
// (samples/hybrid_sssp/hybrid_sssp.cu:196-197), at least 1.
double default_sssp_delta(const sg_graph *g) {
    if (!g->ne) return 1.0;
    return std::max(1.0, std::floor(32.0 * (g->weight_sum / g->ne) / ((double)g->ne / g->nv)));
}

sg_status check_batch(sg_ctx *ctx, const sg_batch_query *q, uint32_t n) {
    if (!ctx || !q || n == 0) return SG_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < n; ++i) {
        if (!q[i].graph || q[i].graph->ctx->device != ctx->device || !q[i].out)
            return sgb::set_error(ctx, SG_ERR_INVALID_ARG, "query %u: graph on another device or null output", i);
        if (q[i].source >= q[i].graph->nv)
            return sgb::set_error(ctx, SG_ERR_INVALID_ARG, "query %u: source out of range", i);
    }
    return SG_OK;
}

struct DevGuard {
    int prev = -1, dev;
    explicit DevGuard(int d) : dev(d) {
        cudaGetDevice(&prev);
        if (prev != d) cudaSetDevice(d);
    }
    ~DevGuard() {
        if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    }
};

// Builds the functors and launch parameters of a batch of one algorithm
// (SG_QUERY_BFS / SSSP / BC) and hands them to `run`, whose
// go<App, TV, TB, TW>(queries, graphs, outputs, params) plans or runs them.
template <typename Run>
sg_status dispatch_batch(int algo, const sg_batch_query *q, uint32_t n, const sg_options &o, Run &run) {
    engine::Params p = batch_params(o, 0);
    std::vector<sg_graph *> graphs(n);
    std::vector<void *> outs(n);
    for (uint32_t i = 0; i < n; ++i) {
        graphs[i] = q[i].graph;
        outs[i] = q[i].out;
        if (!q[i].graph->has_csc && p.forced < 0) p.forced = engine::V_ASYNC_PUSH_DD;
    }
    auto build = [&](auto make_app, auto *tag) {
        using App = std::remove_pointer_t<decltype(tag)>;
        std::vector<engine::BatchQuery<App, uint32_t>> qs;
        qs.reserve(n);
        for (uint32_t i = 0; i < n; ++i) qs.push_back(make_query(make_app(q[i].source), q[i].graph));
        return qs;
    };
    if (algo == SG_QUERY_SSSP) {
        using App = apps::SSSP<uint32_t, uint32_t, uint32_t>;
        auto qs = build([](uint32_t s) { return App(s); }, (App *)nullptr);
        if (o.priority == SG_PRIORITY_LOW_HIGH) {
            // a given delta for every query, else the reference heuristic on each query's own graph
            p.priority = 1;
            if (o.priority_delta > 0)
                p.prio_init_raw = p.prio_step_raw = engine::to_raw<uint32_t>((uint32_t)o.priority_delta);
            for (uint32_t i = 0; i < n; ++i) {
                const sg_graph *g = graphs[i];
                const double delta = o.priority_delta > 0 ? o.priority_delta : default_sssp_delta(g);
                qs[i].prio_raw = engine::to_raw<uint32_t>((uint32_t)delta);
            }
            if (p.forced < 0) p.forced = engine::V_ASYNC_PUSH_DD;
            p.collect = 0;
        }
        return run.template go<App, uint32_t, uint32_t, uint32_t>(qs, graphs, outs, p);
    }
    if (algo == SG_QUERY_BFS) {
        using App = apps::BFS<uint32_t, uint32_t, graphs::NoWeight>;
        const bool non_atomic = o.non_atomic != 0 && o.local_depth <= 0;  // lookahead needs the atomic minimum
        auto qs = build([non_atomic](uint32_t s) { return App(s, non_atomic); }, (App *)nullptr);
        return run.template go<App, uint32_t, uint32_t, graphs::NoWeight>(qs, graphs, outs, p);
    }
    if (algo == SG_QUERY_BC) {
        // HybridBC forces FINE_GRAINED load balancing (hybrid_bc.cu:335-336)
        if (o.lb_push < 0) p.lb_push = engine::LB_FINE;
        if (o.lb_pull < 0) p.lb_pull = engine::LB_FINE;
        // team state (path counts, level stack) is bound on the device
        auto qs = build([](uint32_t s) { return BCApp(s, nullptr, nullptr, apps::LevelStack{}); }, (BCApp *)nullptr);
        return run.template go<BCApp, uint32_t, uint32_t, graphs::NoWeight>(qs, graphs, outs, p);
    }
    return SG_ERR_INVALID_ARG;
}

struct DirectRun {
    sg_ctx *ctx;
    const sg_options &o;
    sg_stats *stats;
    float *per_query_ms;
    template <typename App, typename TV, typename TB, typename TW>
    sg_status go(std::vector<engine::BatchQuery<App, TV>> &qs, const std::vector<sg_graph *> &graphs,
                 const std::vector<void *> &outs, engine::Params p) {
        return run_batch<App, TV, TB, TW>(ctx, std::move(qs), graphs, outs, o, p, stats, per_query_ms);
    }
};

sg_status batch_entry(int algo, sg_ctx *ctx, const sg_batch_query *q, uint32_t n, const sg_options *opt,
                      sg_stats *stats, float *per_query_ms) {
    sg_status st = check_batch(ctx, q, n);
    if (st != SG_OK) return st;
    DevGuard dg(ctx->device);
    sg_options o;
    if (opt)
        o = *opt;
    else
        sg_options_default(&o);
    DirectRun run{ctx, o, stats, per_query_ms};
    return dispatch_batch(algo, q, n, o, run);
}

}  // namespace

extern "C" sg_status sg_sssp_batch(sg_ctx *ctx, const sg_batch_query *q, uint32_t n, const sg_options *opt,
                                   sg_stats *stats, float *per_query_ms) {
    return batch_entry(SG_QUERY_SSSP, ctx, q, n, opt, stats, per_query_ms);
}

extern "C" sg_status sg_bfs_batch(sg_ctx *ctx, const sg_batch_query *q, uint32_t n, const sg_options *opt,
                                  sg_stats *stats, float *per_query_ms) {
    return batch_entry(SG_QUERY_BFS, ctx, q, n, opt, stats, per_query_ms);
}

extern "C" sg_status sg_bc_batch(sg_ctx *ctx, const sg_batch_query *q, uint32_t n, const sg_options *opt,
                                 sg_stats *stats, float *per_query_ms) {
    return batch_entry(SG_QUERY_BC, ctx, q, n, opt, stats, per_query_ms);
}

// ---------------------------------------------------------------- planned batches (CUDA graphs)
struct sg_batch_plan {
    sg_ctx *ctx = nullptr;
    sgb::Workspace ws;  // owned: a captured graph holds these addresses
    BatchBuild B;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool captured = false;
    bool launched = false;
};

namespace {

struct PlanRun {
    sg_batch_plan *plan;
    const sg_options &o;
    template <typename App, typename TV, typename TB, typename TW>
    sg_status go(std::vector<engine::BatchQuery<App, TV>> &qs, const std::vector<sg_graph *> &graphs,
                 const std::vector<void *> &outs, engine::Params p) {
        return prepare_batch<App, TV, TB, TW>(plan->ctx, plan->ws, std::move(qs), graphs, outs, o, p, true, plan->B);
    }
};

}  // namespace

extern "C" sg_status sg_batch_plan_create(sg_ctx *ctx, int algo, const sg_batch_query *q, uint32_t n,
                                          const sg_options *opt, sg_batch_plan **out) {
    if (!out || (algo != SG_QUERY_BFS && algo != SG_QUERY_SSSP && algo != SG_QUERY_BC)) return SG_ERR_INVALID_ARG;
    *out = nullptr;
    sg_status st = check_batch(ctx, q, n);
    if (st != SG_OK) return st;
    DevGuard dg(ctx->device);
    sg_options o;
    if (opt)
        o = *opt;
    else
        sg_options_default(&o);
    auto plan = std::make_unique<sg_batch_plan>();
    plan->ctx = ctx;
    PlanRun run{plan.get(), o};
    if ((st = dispatch_batch(algo, q, n, o, run)) != SG_OK) return st;
    SG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // descriptors are on the device
    // Capture memsets + the cooperative launch once; a driver that cannot
    // capture them leaves the plan on direct launches (same work, more calls).
    cudaStream_t s = ctx->stream;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const sg_status est = enqueue_batch(ctx, plan->B, s);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(s, &g);
        if (est == SG_OK && ce == cudaSuccess && g &&
            cudaGraphInstantiate(&plan->exec, g, 0) == cudaSuccess) {
            plan->graph = g;
            plan->captured = true;
        } else if (g) {
            cudaGraphDestroy(g);
        }
    }
    cudaGetLastError();  // a refused capture leaves no error behind
    ctx->last_error.clear();
    *out = plan.release();
    return SG_OK;
}

extern "C" sg_status sg_batch_plan_launch(sg_batch_plan *plan) {
    if (!plan) return SG_ERR_INVALID_ARG;
    sg_ctx *ctx = plan->ctx;
    DevGuard dg(ctx->device);
    SG_TRY_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    if (plan->captured) {
        SG_TRY_CUDA(ctx, cudaGraphLaunch(plan->exec, ctx->stream));
    } else {
        const sg_status st = enqueue_batch(ctx, plan->B, ctx->stream);
        if (st != SG_OK) return st;
    }
    SG_TRY_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    plan->launched = true;
    return SG_OK;
}

extern "C" sg_status sg_batch_plan_wait(sg_batch_plan *plan, sg_stats *stats, float *per_query_ms) {
    if (!plan || !plan->launched) return SG_ERR_INVALID_ARG;
    DevGuard dg(plan->ctx->device);
    return finish_batch(plan->ctx, plan->ws, plan->B, false, stats, per_query_ms);
}

extern "C" int sg_batch_plan_captured(const sg_batch_plan *plan) { return plan && plan->captured ? 1 : 0; }

extern "C" sg_status sg_batch_plan_destroy(sg_batch_plan *plan) {
    if (!plan) return SG_ERR_INVALID_ARG;
    DevGuard dg(plan->ctx->device);
    cudaStreamSynchronize(plan->ctx->stream);
    if (plan->exec) cudaGraphExecDestroy(plan->exec);
    if (plan->graph) cudaGraphDestroy(plan->graph);
    delete plan;
    return SG_OK;
}
