// Device-resident hybrid engine: one cooperative launch runs the whole round
// loop of the reference's Engine::Start (include/framework/framework.cuh:315-375)
// — PreComputation, ExecutePolicy, PostComputation and the PolicyDecisionMaker
// (include/framework/hybrid_policy.h:123-311) — with no host round trip per round.
//
// Per round the grid executes one variant:
//   ASYNC_PUSH_DD  frontier queue -> warp-cooperative, edge-balanced expansion
//                  (async_push_dd.cuh:24-147, push_functor.h:118-164); vertices
//                  above `heavy_threshold` out-edges are split into fixed-size
//                  chunks spread over all warps (the CTA tier of
//                  cta_scheduler_hybrid.cuh:59-277, but grid-wide).  Optional
//                  two-level priority (near/far piles, driver.cuh:605-685).
//   ASYNC_PULL_DD / SYNC_PULL_DD
//                  bottom-up: CombineValueBuffer over all vertices builds the
//                  "middle" list (variants/common.cuh:17-53), then each middle
//                  vertex scans its in-edges against the input frontier bitmap
//                  with early exit (async_pull_dd.cuh:26-136, pull_functor.h:138-188).
//   SYNC_PULL_TD   all-vertex pull from the tmp buffer (sync_pull_td.cuh:22-112).
//   ASYNC_PUSH_TD  all-vertex push (async_push_td.cuh:25-147).
// TD rounds end with RebuildArrayWorklist (algo_variants.cuh:58-76).
//
// Control: block 0 is the fixed leader.  At every grid barrier it waits for
// the other blocks, evaluates the policy from the round's atomic counters
// (every append to the next worklist also accumulates the appended vertex's
// out-degree — the "scout count" that SumOutDegreeQueue computes with a separate
// kernel and a D2H copy, driver.cuh:225-248), rotates worklists, records the
// trace and publishes a 64-byte round snapshot that every block reads with
// four vector loads.  Policy state (RunningInfo, hybrid_policy.h:36-120) stays
// in the leader thread's local memory for the whole launch.
//
// A per-vertex "queued" bitmap keeps each worklist free of duplicates, which
// bounds every worklist by |V| (the reference sizes them at 0.2*|E| and can
// overflow silently, graph_datum.cuh:90).
#pragma once
#include <cstdint>
#include <limits>
#include <cstring>
#include <type_traits>
#include <utility>

#include "../../include/sepgraph.h"
#include "sg_api.cuh"
#include "sg_device.cuh"

namespace sepgraph {
namespace engine {

constexpr int kBlockThreads = 256;
constexpr int kWarpsPerBlock = kBlockThreads / 32;

// Variant ids (AlgoVariant::Id): (model << 2) | (msg << 1) | sched
enum : int32_t {
    V_SYNC_PUSH_TD = 0,
    V_SYNC_PUSH_DD = 1,
    V_SYNC_PULL_TD = 2,
    V_SYNC_PULL_DD = 3,
    V_ASYNC_PUSH_TD = 4,
    V_ASYNC_PUSH_DD = 5,
    V_ASYNC_PULL_TD = 6,
    V_ASYNC_PULL_DD = 7
};
__host__ __device__ inline bool is_dd(int v) { return v & 1; }
__host__ __device__ inline bool is_pull(int v) { return (v >> 1) & 1; }
__host__ __device__ inline bool is_sync(int v) { return ((v >> 2) & 1) == 0; }
__host__ __device__ inline bool is_pull_dd(int v) { return v >= 0 && is_dd(v) && is_pull(v); }

enum : int32_t { LB_NONE = 0, LB_COARSE = 1, LB_FINE = 2, LB_HYBRID = 3 };

template <typename TBuffer>
struct HeavyItem {
    uint32_t src, beg, deg, chunk_base;
    TBuffer payload;
};

// Round snapshot: written by the leader, read by every block after a barrier.
struct alignas(16) RoundState {
    int32_t variant, last_variant;
    uint32_t round, done;
    uint32_t qin, qhi, qlo, bin;
    uint32_t bout, dirty, pile, F;
    uint32_t heavy_expected;  // heavy vertices forecast for this round (level-synchronous apps)
    uint32_t chunks;          // chunks registered by the previous push round, run at this round's start
    unsigned long long prio_raw;
};
static_assert(sizeof(RoundState) == 64, "snapshot is four 16-byte loads");

// Updated atomically by all blocks during a round.
struct Counters {
    uint32_t qcount[4];
    uint32_t heavy_enq[4];
    unsigned long long scout[4];
    uint32_t middle_count, error;
    uint32_t active_count;  // active vertices of a round whose worklist nobody reads (forced TD)
    uint32_t heavy_count[2], chunk_count[2];  // heavy-vertex tables, one set per round parity
    unsigned long long edges_processed;
    uint32_t popped;  // worklist items taken from a bitmap worklist this round
};

struct Ctrl {
    uint32_t bar_count, bar_gen, pad0, pad1;
    RoundState rs;
    Counters cnt;
    // results, written by the leader when the loop ends
    uint32_t round, max_iteration_reached, n_trace, error;
    uint32_t rounds_by_variant[8];
    unsigned long long edges_processed, vertices_processed;
    unsigned long long t_start, t_end;
};

struct Params {
    int32_t scheme;  // 0 = TRAVERSAL_SCHEME, 1 = ITERATIVE_SCHEME
    int32_t forced;  // variant id or -1
    int32_t lb_push, lb_pull;
    int32_t priority;  // 1 = two-level (LOW_HIGH)
    int32_t trace;
    int32_t collect;  // keep policy statistics (!forced || trace), framework.cuh:529
    int32_t has_csc;
    uint32_t max_iteration;
    uint32_t heavy_threshold;
    uint32_t chunk_edges;
    uint32_t pull_warp_threshold;
    uint32_t local_depth;  // levels a block follows its own discoveries inside a push round (0 = off)
    float sample_cut;      // sampling priority in ASYNC_PUSH_TD rounds (SetSampleBasedPriority), 0 = off
    // Bitmap worklists (forced ASYNC_PUSH_DD with load balancing, worklists
    // unsorted): a push sets the destination's bit in the output slot's queued
    // bitmap with a fire-and-forget reduction and appends nothing; the next
    // round takes its items from that bitmap (see push_phase_a).  The slot
    // counters then count pushes, not distinct vertices (zero iff empty).
    int32_t bitmap_frontier;
    // Hub chunks of min-relax functors staged by bulk copies (256-edge chunks).
    int32_t stage_chunks;
    // Data-driven pull into vertices of at most pull_warp_threshold in-edges:
    // 1 = a warp walks 32 vertices' in-edge lists together (pull_coop), 0 = a
    // thread per vertex with early exit (pull_serial).  Measured on B200 the
    // thread form is as fast or faster (8 BFS on symmetric RMAT-22: 9.33 vs
    // 9.74 ms; BC and grid BFS equal): in a pull round most vertices find a
    // frontier neighbour within their first in-edges, and the warp form loads
    // whole lists.
    int32_t pull_coop;
    double alpha, beta;
    long long total_workload0;
    unsigned long long prio_init_raw, prio_step_raw;
    unsigned long long timeout_ns;
};

// Bitmap worklists are used when every round is a forced ASYNC_PUSH_DD with
// load balancing and the worklists need not be sorted (--wl_sort builds a
// sorted queue instead).
// worklist: SG_WORKLIST_AUTO / _QUEUE / _BITMAP (sg_options.worklist).
inline bool use_bitmap_frontier(int forced, int lb_push, bool wl_sort, int worklist) {
    if (forced != V_ASYNC_PUSH_DD || lb_push == LB_NONE || wl_sort) return false;
    return worklist == SG_WORKLIST_BITMAP;
}

template <typename TValue, typename TBuffer, typename TWeight>
struct KArgs {
    graphs::dev::CSRGraph csr;
    graphs::dev::CSCGraph csc;
    const uint32_t *csr_w;
    const uint32_t *csc_w;
    TValue *value;
    TBuffer *buffer;
    TBuffer *tmp;
    uint32_t *queue[3];
    uint32_t queue_cap;
    uint32_t *bitmap[2];
    uint32_t *qflag[3];  // queued bitmap of each worklist slot
    uint32_t nwords;
    uint32_t *middle;
    HeavyItem<TBuffer> *heavy;  // 2 * heavy_cap items: set k starts at heavy + k * heavy_cap
    uint32_t heavy_cap;
    uint32_t *chunk_owner;      // 2 * chunk_cap entries, likewise
    uint32_t chunk_cap;
    Ctrl *ctrl;
    sg_round_trace *trace;
    uint32_t trace_cap;
    Params p;
    // --wl_sort: one count per block of the team; null = worklists are not sorted
    uint32_t *sort_counts = nullptr;
    // Edge-tiled topology-driven pull (functors with PullReduce, unweighted):
    // tile_row[t] = the in-edge row holding CSC edge t * kPullTileEdges
    // (ceil(E / kPullTileEdges) + 1 entries, the last = V - 1), filled at the
    // launch's start; null = the destination-per-lane pull is used instead.
    uint32_t *tile_row = nullptr;
};

// In-edges per warp tile of the edge-tiled pull: 8 per lane, two 16-byte loads.
constexpr uint32_t kPullTileEdges = 256;
// Rows a tile may span and still sum its rows in shared memory first.
constexpr uint32_t kPullTileRows = 64;

// Leader-only policy state (RunningInfo), lives in block 0 / thread 0.
struct PolicyState {
    RoundState rs;
    long long total_workload;
    uint32_t input_active, output_active;
    unsigned long long input_workload, output_workload;
    float policy_time[8];
    uint32_t policy_seen, inspect_next;
    float time_per_work;
    unsigned long long t_round_start, t_start;
    uint32_t rounds_by_variant[8];
    unsigned long long vertices_processed;
    uint32_t n_trace, max_iteration_reached;
};

template <typename TBuffer>
struct WarpLB {
    uint32_t excl[32];
    uint32_t beg[32];
    uint32_t src[32];
    TBuffer pay[32];
    // topology-driven pull: each lane's first and last (possibly shared) segment
    uint32_t partk[2][32];
    TBuffer part[2][32];
    // edge-tiled pull: per-row sums of one tile and the rows touched
    TBuffer rowsum[kPullTileRows];
    unsigned long long touched;
    // bitmap worklist: the 32 words a warp took and their exclusive popcount scan
    uint32_t scan_excl[32];
    uint32_t scan_bits[32];
};

// A block's own queue of vertices it discovered in a push round and may
// process before the round ends (local lookahead, reorder-safe functors only).
// Two buffers alternate between "being processed" and "being filled"; what
// does not fit, and what is left when the depth runs out, goes to the global
// worklist.
constexpr uint32_t kLocalCap = 1024;
struct LocalQ {
    uint32_t item[2][kLocalCap];
    uint32_t n[2];
    uint32_t out;  // buffer receiving discoveries
};

// Per-thread accumulators flushed once per phase.
struct Acc {
    unsigned long long scout_hi, scout_lo;
    uint32_t heavy_hi, heavy_lo;
    unsigned long long edges;
    __device__ void reset() {
        scout_hi = scout_lo = 0;
        heavy_hi = heavy_lo = 0;
        edges = 0;
    }
    __device__ __forceinline__ void count(bool hi, uint32_t deg, uint32_t heavy_threshold) {
        const uint32_t h = deg > heavy_threshold;
        if (hi) {
            scout_hi += deg;
            heavy_hi += h;
        } else {
            scout_lo += deg;
            heavy_lo += h;
        }
    }
};

template <typename T>
__host__ __device__ inline unsigned long long to_raw(T x) {
    unsigned long long r = 0;
    memcpy(&r, &x, sizeof(T));
    return r;
}
template <typename T>
__host__ __device__ inline T from_raw(unsigned long long r) {
    T x;
    memcpy(&x, &r, sizeof(T));
    return x;
}

// ---- optional PullReduce extension detection
template <typename App, typename TB, typename = void>
struct has_pull_reduce : std::false_type {};
template <typename App, typename TB>
struct has_pull_reduce<App, TB,
                       std::void_t<decltype(std::declval<const App &>().PullReduce(std::declval<TB>(),
                                                                                    std::declval<TB>()))>>
    : std::true_type {};

// Functors whose result does not depend on the order in which pushes are
// applied (atomic monotone label correction as in BFS/SSSP, residual
// accumulation as in PageRank) declare `bool ReorderSafe() const` returning
// true (BFS only when its accumulation is atomic: a plain store may lose a
// smaller level written concurrently by a push of another level).  For them,
// when every round is ASYNC_PUSH_DD (a forced variant), the chunks of heavy
// vertices found in a round run at the start of the next round instead of
// behind an extra barrier.  Under the hybrid policy the next round may be a
// pull round, whose frontier must already hold every vertex those chunks would
// reach, and level-synchronous functors (BC's path counting) need both halves
// of a round apart, so both keep the barrier.
// Local lookahead (Params::local_depth) also relies on this declaration, and
// adds one obligation: a block may combine a vertex it discovered while
// another block combines the same vertex (from its own lookahead queue or the
// round's worklist), so a reorder-safe functor's CombineValueBuffer must
// tolerate concurrent calls for one vertex while m_concurrent_combine is set
// (BFS/SSSP: atomic minimum on the value; PageRank: atomic exchange of the
// residual, atomic add to the value).
template <typename App, typename = void>
struct has_reorder_safe : std::false_type {};
template <typename App>
struct has_reorder_safe<App, std::void_t<decltype(std::declval<const App &>().ReorderSafe())>> : std::true_type {};
template <typename App>
__device__ __forceinline__ bool reorder_safe(const App &app) {
    if constexpr (has_reorder_safe<App>::value)
        return app.ReorderSafe();
    else
        return false;
}

// Optional functor extension (no reference counterpart): a functor whose
// weighted AccumulateBuffer is exactly a monotone minimum,
//   cand = RelaxCandidate(src, dst, weight, offered);
//   if (cand < *p_buffer) { atomicMin(p_buffer, cand); return SUCCESS_CONTINUE; }
//   return FAILURE_CONTINUE;
// over an unsigned integer buffer, declares
//   __device__ TBuffer RelaxCandidate(index_t src, index_t dst, TWeight w, TBuffer offered) const
// and the engine relaxes hub chunks eight edges per lane at a time: the eight
// current values are loaded together and only improving minima are issued.
// IsHighPriority of such a functor must hold for every value at or below one
// it holds for (a smaller buffer is never of lower priority): the engine then
// routes a push by its candidate instead of re-reading the destination.
template <typename App, typename TB, typename TW, typename = void>
struct has_min_relax : std::false_type {};
template <typename App, typename TB, typename TW>
struct has_min_relax<App, TB, TW,
                     std::void_t<decltype(std::declval<const App &>().RelaxCandidate(
                         std::declval<uint32_t>(), std::declval<uint32_t>(), std::declval<TW>(), std::declval<TB>()))>>
    : std::integral_constant<bool, std::is_same<TB, uint32_t>::value> {};

// Edge range of chunk k of a heavy vertex's list [beg, beg + deg): chunks are
// cut on the 4-edge grid (from beg rounded down to a multiple of 4) so that
// every chunk starts on a 16-byte boundary of the edge arrays, which lets a
// lane read its edges with 16-byte loads; the first chunk starts at beg.
__host__ __device__ __forceinline__ uint32_t chunk_count_of(uint32_t beg, uint32_t deg, uint32_t ce) {
    const uint32_t a0 = beg & ~3u;
    return (beg + deg - a0 + ce - 1) / ce;
}
__host__ __device__ __forceinline__ void chunk_span(uint32_t beg, uint32_t deg, uint32_t ce, uint32_t k,
                                                    uint32_t *lo, uint32_t *hi) {
    const uint32_t a0 = beg & ~3u;
    const uint32_t s = a0 + k * ce;
    *lo = s > beg ? s : beg;
    const uint32_t e = s + ce, end = beg + deg;
    *hi = e < end ? e : end;
}

// Dispatch to the weighted or unweighted AccumulateBuffer overload like
// PushFunctor/PullFunctor do (push_functor.h:123-138).  Unweighted graphs
// give weight 1 to weighted apps (EdgeInputDatum fallback, csr_graph.h:1786-1868).
template <typename App, typename TB, typename TW>
__device__ __forceinline__ int accumulate(App &app, const uint32_t *w, uint32_t src, uint32_t dst, uint32_t edge,
                                          TB *p, TB val) {
    if constexpr (std::is_same<TW, graphs::NoWeight>::value) {
        return app.App::AccumulateBuffer(src, dst, p, val);
    } else {
        TW wt = w ? (TW)__ldg(w + edge) : (TW)1;
        return app.App::AccumulateBuffer(src, dst, wt, p, val);
    }
}
__device__ __forceinline__ bool acc_success(int st) { return st < 2; }
__device__ __forceinline__ bool acc_continue(int st) { return st & 1; }

// A team is the set of blocks that run one query together: the whole grid for
// a single query, or one group of a batched launch.  Every block records its
// rank in the team and the team size before the first barrier.
__shared__ uint32_t g_team_rank, g_team_size;
// Generation of the team barrier this block passed last (kept by thread 0).
__shared__ uint32_t g_bar_gen;

constexpr uint32_t kGenMask = 0x7fffffffu;   // generation counter bits
constexpr uint32_t kGenAbort = 0x80000000u;  // set by a leader whose wait gave up

// Joins the team and reads the barrier generation; must run before this
// block's first arrival (no generation can pass without it).
__device__ __forceinline__ void set_team(uint32_t rank, uint32_t size, Ctrl *c) {
    if (threadIdx.x == 0) {
        g_team_rank = rank;
        g_team_size = size;
        g_bar_gen = dev::ld_acquire(&c->bar_gen);
    }
    __syncthreads();
}

// Bounded team barrier with team rank 0 as the fixed leader.  Every other block
// arrives with a release fence and a fire-and-forget add, then polls the
// generation word; block 0 waits for all arrivals, runs `leader()` on one
// thread and publishes the next generation with a release store.  Each block
// tracks the generation it expects, so an arrival costs no read.  A wait that
// exceeds timeout_ns raises kErrTimeout and returns false; a leader that gives
// up releases the others with the abort bit set, so they return false too.
template <typename Leader>
__device__ __forceinline__ bool grid_sync(Ctrl *c, unsigned long long timeout_ns, Leader &&leader) {
    __shared__ uint32_t s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t ok = 1;
        const uint32_t g = g_bar_gen;
        uint32_t next = g;
        if (g_team_rank == 0) {
            const uint32_t need = g_team_size - 1;
            const uint64_t t0 = dev::globaltimer_ns();
            uint32_t spins = 0;
            while (dev::ld_acquire(&c->bar_count) < need) {
                ++spins;
                if ((spins & 255u) == 0 && (dev::globaltimer_ns() - t0 > timeout_ns || spins > (1u << 28))) {
                    atomicOr(&c->cnt.error, dev::kErrTimeout);
                    ok = 0;
                    break;
                }
                __nanosleep(20);
            }
            dev::st_relaxed(&c->bar_count, 0u);  // ordered before the next arrivals by the release below
            if (ok) leader();
            next = ((g + 1) & kGenMask) | (ok ? 0u : kGenAbort);
            dev::st_release(&c->bar_gen, next);
        } else {
            dev::arrive_release(&c->bar_count);
            const uint64_t t0 = dev::globaltimer_ns();
            uint32_t spins = 0;
            for (;;) {
                next = dev::ld_acquire(&c->bar_gen);
                if (next != g) break;
                ++spins;
                if ((spins & 255u) == 0 && (dev::globaltimer_ns() - t0 > timeout_ns || spins > (1u << 28))) {
                    atomicOr(&c->cnt.error, dev::kErrTimeout);
                    ok = 0;
                    break;
                }
                __nanosleep(20);
            }
            if (next & kGenAbort) ok = 0;
        }
        g_bar_gen = next;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

template <typename App, typename TV, typename TB, typename TW>
struct EngineKernel {
    using Args = KArgs<TV, TB, TW>;
    using Snap = RoundState;

    static __device__ __forceinline__ uint32_t gthread() { return g_team_rank * blockDim.x + threadIdx.x; }
    static __device__ __forceinline__ uint32_t nthreads() { return g_team_size * blockDim.x; }
    static __device__ __forceinline__ uint32_t gwarp() { return gthread() >> 5; }
    static __device__ __forceinline__ uint32_t nwarps() { return nthreads() >> 5; }

    static __device__ __forceinline__ uint32_t out_degree(const Args &a, uint32_t v) {
        return a.csr.end_edge(v) - a.csr.begin_edge(v);
    }

    // Out-degree of an appended vertex feeds the policy (scout count) and the
    // heavy-vertex forecast; with a forced variant and no trace neither is
    // needed and the two dependent loads are skipped (the round then always
    // runs its chunk phase).
    static __device__ __forceinline__ void count_enq(const Args &a, Acc &acc, bool hi, uint32_t v) {
        if (a.p.collect) acc.count(hi, out_degree(a, v), a.p.heavy_threshold);
    }

    static __device__ void flush_acc(const Args &a, Acc &acc, uint32_t q_hi, uint32_t q_lo) {
        unsigned long long s0 = dev::warp_sum(acc.scout_hi), s1 = dev::warp_sum(acc.scout_lo);
        uint32_t h0 = dev::warp_sum(acc.heavy_hi), h1 = dev::warp_sum(acc.heavy_lo);
        unsigned long long ed = dev::warp_sum(acc.edges);
        if (dev::lane_id() == 0) {
            Counters *n = &a.ctrl->cnt;
            if (s0) atomicAdd(&n->scout[q_hi], s0);
            if (h0) atomicAdd(&n->heavy_enq[q_hi], h0);
            if (s1) atomicAdd(&n->scout[q_lo], s1);
            if (h1) atomicAdd(&n->heavy_enq[q_lo], h1);
            if (ed) atomicAdd(&n->edges_processed, ed);
        }
        acc.reset();
    }

    // Append dst to the next worklist(s) if `want`: dedupe through the output
    // slot's queued bitmap, route by IsHighPriority when two-level priority is
    // on, and count its out-degree for the policy.  Each worklist slot has its
    // own queued bitmap: pops clear bits of the input slot only and appends set
    // bits of an output slot only, so a vertex improved during a round always
    // reaches the next round's worklist (which reads it after the barrier) and
    // no fence is needed between the state update and the queued bit.
    // With a block queue `lq`, near (high-priority) vertices go there first.
    // All 32 lanes must call.
    static __device__ __forceinline__ void enqueue(App &app, const Args &a, const Snap &s, uint32_t dst, bool want,
                                                   Acc &acc, LocalQ *lq = nullptr, const TB *offered = nullptr) {
        Counters *n = &a.ctrl->cnt;
        bool hi = true;
        if (a.p.priority && want)
            hi = app.App::IsHighPriority(from_raw<TB>(s.prio_raw), offered ? *offered : dev::ld_l2(a.buffer + dst));
        if (lq) {
            bool loc = want && hi;
            const uint32_t m = __ballot_sync(dev::kFullMask, loc);
            if (m) {
                const uint32_t lane = dev::lane_id(), leader = __ffs(m) - 1, o = lq->out;
                uint32_t base = 0;
                if (lane == leader) base = atomicAdd(&lq->n[o], (uint32_t)__popc(m));
                base = __shfl_sync(dev::kFullMask, base, leader);
                if (loc) {
                    const uint32_t pos = base + __popc(m & dev::lanemask_lt());
                    if (pos < kLocalCap)
                        lq->item[o][pos] = dst;
                    else
                        loc = false;  // block queue full: global worklist
                }
            }
            want = want && !loc;
        }
        bool w_hi = want && hi, w_lo = want && !hi;
        if (a.p.bitmap_frontier) {
            // no dedupe round trip and no append: the bit is the worklist entry
            if (w_hi) dev::bitmap_set_nr(a.qflag[s.qhi], dst);
            if (w_lo) dev::bitmap_set_nr(a.qflag[s.qlo], dst);
            count_pushes(n, s, w_hi, w_lo);
            if (w_hi || w_lo) count_enq(a, acc, w_hi, dst);
            return;
        }
        if (w_hi) w_hi = dev::bitmap_set(a.qflag[s.qhi], dst);
        if (w_lo) w_lo = dev::bitmap_set(a.qflag[s.qlo], dst);
        dev::warp_append(a.queue[s.qhi], &n->qcount[s.qhi], a.queue_cap, w_hi, dst, &n->error);
        if (a.p.priority) dev::warp_append(a.queue[s.qlo], &n->qcount[s.qlo], a.queue_cap, w_lo, dst, &n->error);
        if (w_hi || w_lo) count_enq(a, acc, w_hi, dst);
    }

    // Bitmap worklists: one fire-and-forget add per warp and slot of the
    // number of pushes (the leader only needs to know whether a slot is empty).
    // All 32 lanes must call.
    static __device__ __forceinline__ void count_pushes(Counters *n, const Snap &s, bool w_hi, bool w_lo) {
        const uint32_t mh = __ballot_sync(dev::kFullMask, w_hi), ml = __ballot_sync(dev::kFullMask, w_lo);
        if (dev::lane_id() == 0) {
            if (mh) dev::red_add(&n->qcount[s.qhi], (uint32_t)__popc(mh));
            if (ml) dev::red_add(&n->qcount[s.qlo], (uint32_t)__popc(ml));
        }
    }

    // K pushes per lane at once, with the candidate values the pushes offer
    // (the priority routing uses them, see has_min_relax; null = read each
    // destination's buffer as enqueue() does).  Same effect as K
    // enqueue() calls, but the K queued-bit updates are issued together and
    // each slot gets one warp-wide reservation for all of them: two dependent
    // memory round trips per call instead of two per push.  All 32 lanes must
    // call.
    template <int K>
    static __device__ __forceinline__ void enqueue_batch(App &app, const Args &a, const Snap &s, const uint32_t *dst,
                                                         bool *want, const TB *offered, Acc &acc, LocalQ *lq) {
        Counters *n = &a.ctrl->cnt;
        const TB prio = from_raw<TB>(s.prio_raw);
        bool hi[K];
#pragma unroll
        for (int j = 0; j < K; ++j)
            hi[j] = !a.p.priority || !want[j] ||
                    app.App::IsHighPriority(prio, offered ? offered[j] : dev::ld_l2(a.buffer + dst[j]));
        if (lq) {  // near vertices go to the block's lookahead queue first
            const uint32_t lane = dev::lane_id();
#pragma unroll
            for (int j = 0; j < K; ++j) {
                bool loc = want[j] && hi[j];
                const uint32_t m = __ballot_sync(dev::kFullMask, loc);
                if (m) {
                    const uint32_t leader = __ffs(m) - 1, o = lq->out;
                    uint32_t base = 0;
                    if (lane == leader) base = atomicAdd(&lq->n[o], (uint32_t)__popc(m));
                    base = __shfl_sync(dev::kFullMask, base, leader);
                    if (loc) {
                        const uint32_t pos = base + __popc(m & dev::lanemask_lt());
                        if (pos < kLocalCap)
                            lq->item[o][pos] = dst[j];
                        else
                            loc = false;
                    }
                }
                want[j] = want[j] && !loc;
            }
        }
        if (a.p.bitmap_frontier) {
            uint32_t ch = 0, cl = 0;
#pragma unroll
            for (int j = 0; j < K; ++j) {
                if (want[j]) {
                    dev::bitmap_set_nr(a.qflag[hi[j] ? s.qhi : s.qlo], dst[j]);
                    count_enq(a, acc, hi[j], dst[j]);
                }
                ch += want[j] && hi[j];
                cl += want[j] && !hi[j];
            }
            ch = dev::warp_sum(ch);
            cl = dev::warp_sum(cl);
            if (dev::lane_id() == 0) {
                if (ch) dev::red_add(&n->qcount[s.qhi], ch);
                if (cl) dev::red_add(&n->qcount[s.qlo], cl);
            }
            return;
        }
        bool w[K];
#pragma unroll
        for (int j = 0; j < K; ++j) w[j] = want[j] ? dev::bitmap_set(a.qflag[hi[j] ? s.qhi : s.qlo], dst[j]) : false;
        uint32_t ch = 0, cl = 0;
#pragma unroll
        for (int j = 0; j < K; ++j) {
            ch += w[j] && hi[j];
            cl += w[j] && !hi[j];
        }
        const uint32_t ih = dev::warp_inclusive_scan(ch), il = dev::warp_inclusive_scan(cl);
        const uint32_t th = __shfl_sync(dev::kFullMask, ih, 31), tl = __shfl_sync(dev::kFullMask, il, 31);
        uint32_t bh = 0, bl = 0;
        if (dev::lane_id() == 0) {
            if (th) bh = atomicAdd(&n->qcount[s.qhi], th);
            if (tl) bl = atomicAdd(&n->qcount[s.qlo], tl);
        }
        bh = __shfl_sync(dev::kFullMask, bh, 0) + ih - ch;
        bl = __shfl_sync(dev::kFullMask, bl, 0) + il - cl;
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (!w[j]) continue;
            const uint32_t q = hi[j] ? s.qhi : s.qlo;
            const uint32_t pos = hi[j] ? bh++ : bl++;
            if (pos < a.queue_cap)
                a.queue[q][pos] = dst[j];
            else
                atomicOr(&n->error, dev::kErrCapacity);
            count_enq(a, acc, hi[j], dst[j]);
        }
    }

    // Single-thread enqueue (LB NONE paths run divergent per-thread loops).
    static __device__ __forceinline__ void enqueue_one(App &app, const Args &a, const Snap &s, uint32_t dst,
                                                       Acc &acc, LocalQ *lq = nullptr) {
        Counters *n = &a.ctrl->cnt;
        bool hi = true;
        if (a.p.priority) hi = app.App::IsHighPriority(from_raw<TB>(s.prio_raw), dev::ld_l2(a.buffer + dst));
        if (lq && hi) {
            const uint32_t o = lq->out;
            const uint32_t pos = atomicAdd(&lq->n[o], 1u);
            if (pos < kLocalCap) {
                lq->item[o][pos] = dst;
                return;
            }
        }
        const uint32_t q = hi ? s.qhi : s.qlo;
        if (!dev::bitmap_set(a.qflag[q], dst)) return;
        const uint32_t pos = atomicAdd(&n->qcount[q], 1u);
        if (pos < a.queue_cap)
            a.queue[q][pos] = dst;
        else
            atomicOr(&n->error, dev::kErrCapacity);
        count_enq(a, acc, hi, dst);
    }

    // Registers the lanes' heavy vertices as chunk lists (warp-aggregated: one
    // ballot, one scan, two atomics per warp).  All 32 lanes must call.
    static __device__ __forceinline__ void register_heavy(const Args &a, uint32_t set, bool heavy, uint32_t src,
                                                          uint32_t beg, uint32_t deg, TB payload) {
        const uint32_t m = __ballot_sync(dev::kFullMask, heavy);
        if (m == 0) return;
        Counters *n = &a.ctrl->cnt;
        const uint32_t lane = dev::lane_id();
        const uint32_t ce = a.p.chunk_edges;
        const uint32_t nch = heavy ? chunk_count_of(beg, deg, ce) : 0u;
        const uint32_t incl = dev::warp_inclusive_scan(nch);
        const uint32_t tot = __shfl_sync(dev::kFullMask, incl, 31);
        const uint32_t leader = __ffs(m) - 1;
        uint32_t hb = 0, cb = 0;
        if (lane == leader) {
            hb = atomicAdd(&n->heavy_count[set], (uint32_t)__popc(m));
            cb = atomicAdd(&n->chunk_count[set], tot);
        }
        hb = __shfl_sync(dev::kFullMask, hb, leader);
        cb = __shfl_sync(dev::kFullMask, cb, leader);
        if (!heavy) return;
        const uint32_t idx = hb + __popc(m & dev::lanemask_lt());
        const uint32_t c0 = cb + incl - nch;
        if (idx < a.heavy_cap && c0 <= a.chunk_cap && nch <= a.chunk_cap - c0) {
            HeavyItem<TB> h;
            h.src = src;
            h.beg = beg;
            h.deg = deg;
            h.chunk_base = c0;
            h.payload = payload;
            a.heavy[(size_t)set * a.heavy_cap + idx] = h;
            uint32_t *own = a.chunk_owner + (size_t)set * a.chunk_cap;
            for (uint32_t i = 0; i < nch; ++i) own[c0 + i] = idx;
        } else {
            atomicOr(&n->error, dev::kErrChunkCapacity);
        }
    }

    // Owner lane of edge e in a warp's concatenated edge lists: the largest k
    // with excl[k] <= e (binary search over the exclusive degree scan).
    static __device__ __forceinline__ uint32_t owner(const uint32_t *excl, uint32_t e) {
        uint32_t k = 0;
#pragma unroll
        for (uint32_t step = 16; step > 0; step >>= 1)
            if (excl[k + step] <= e) k += step;
        return k;
    }

    // Warp-cooperative expansion of up to 32 (src, beg, deg, payload) items:
    // the warp walks the concatenation of their edge lists 32 edges at a time.
    // All 32 lanes must call.
    static __device__ void expand_warp(App &app, const Args &a, const Snap &s, WarpLB<TB> &w, uint32_t src,
                                       uint32_t beg, uint32_t deg, TB payload, bool dd, Acc &acc,
                                       LocalQ *lq = nullptr) {
        const uint32_t lane = dev::lane_id();
        const uint32_t incl = dev::warp_inclusive_scan(deg);
        const uint32_t total = __shfl_sync(dev::kFullMask, incl, 31);
        if (total == 0) return;
        w.excl[lane] = incl - deg;
        w.beg[lane] = beg;
        w.src[lane] = src;
        w.pay[lane] = payload;
        __syncwarp();
        if constexpr (has_min_relax<App, TB, TW>::value) {
            // Min-relax functors: 4 edges per lane per step (edge eb + 32j + lane),
            // their 4 destination values loaded together, one batched push.
            for (uint32_t eb = 0; eb < total; eb += 128) {
                EdgeRef r[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) r[j] = locate(a, w, eb + 32u * j + lane, total);
                uint32_t d[4];
                TB cand[4], cur[4];
                bool want[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    d[j] = r[j].dst;
                    cand[j] = r[j].valid ? app.RelaxCandidate(r[j].src, r[j].dst, (TW)r[j].wt, r[j].pay)
                                         : std::numeric_limits<TB>::max();
                    cur[j] = r[j].valid ? dev::ld_l2(a.buffer + r[j].dst) : (TB)0;
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    want[j] = cand[j] < cur[j];
                    if (want[j]) atomicMin(a.buffer + d[j], cand[j]);
                    want[j] = want[j] && dd;
                }
                enqueue_batch<4>(app, a, s, d, want, cand, acc, lq);
            }
        } else {
            // 4 edges per lane per step (edge eb + 32j + lane): their owner lookups
            // and index/weight loads, then the 4 accumulations, then one batched
            // push, so a lane has 4 independent memory chains in flight.
            for (uint32_t eb = 0; eb < total; eb += 128) {
                EdgeRef r[4];
    #pragma unroll
                for (int j = 0; j < 4; ++j) r[j] = locate(a, w, eb + 32u * j + lane, total);
                uint32_t d[4];
                bool want[4];
    #pragma unroll
                for (int j = 0; j < 4; ++j) {
                    d[j] = r[j].dst;
                    want[j] = false;
                    if (r[j].valid) {
                        const int st = accumulate_w(app, r[j].src, r[j].dst, r[j].wt, a.buffer + r[j].dst, r[j].pay);
                        want[j] = dd && acc_success(st);
                    }
                }
                enqueue_batch<4>(app, a, s, d, want, nullptr, acc, lq);
            }
        }
        if (lane == 0) acc.edges += total;
        __syncwarp();
    }

    struct EdgeRef {
        uint32_t src, dst, wt;
        TB pay;
        bool valid;
    };

    // Edge e of the warp's concatenated edge lists: source, destination,
    // weight (1 when unweighted) and payload; the destination's state line is
    // prefetched into L2.
    static __device__ __forceinline__ EdgeRef locate(const Args &a, const WarpLB<TB> &w, uint32_t e, uint32_t total) {
        EdgeRef r;
        r.valid = e < total;
        r.src = 0;
        r.dst = 0;
        r.wt = 1;
        r.pay = TB{};
        if (r.valid) {
            const uint32_t k = owner(w.excl, e);
            const uint32_t edge = w.beg[k] + (e - w.excl[k]);
            r.src = w.src[k];
            r.pay = w.pay[k];
            const uint64_t pol = dev::stream_policy();
            r.dst = dev::ldg_stream(a.csr.edge_dst + edge, pol);
            if constexpr (!std::is_same<TW, graphs::NoWeight>::value)
                if (a.csr_w) r.wt = dev::ldg_stream(a.csr_w + edge, pol);
            asm volatile("prefetch.global.L2 [%0];" ::"l"(a.buffer + r.dst));
        }
        return r;
    }

    static __device__ __forceinline__ int accumulate_w(App &app, uint32_t src, uint32_t dst, uint32_t wt, TB *p,
                                                       TB val) {
        if constexpr (std::is_same<TW, graphs::NoWeight>::value) {
            return app.App::AccumulateBuffer(src, dst, p, val);
        } else {
            return app.App::AccumulateBuffer(src, dst, (TW)wt, p, val);
        }
    }

    // Thread-per-vertex sequential expansion honouring BREAK (LB NONE,
    // async_push_dd.cuh:24-77).
    static __device__ void expand_serial(App &app, const Args &a, const Snap &s, uint32_t src, uint32_t beg,
                                         uint32_t deg, TB payload, bool dd, Acc &acc, LocalQ *lq = nullptr) {
        uint32_t e = beg;
        for (; e < beg + deg; ++e) {
            const uint32_t dst = a.csr.edge_dest(e);
            const int st = accumulate<App, TB, TW>(app, a.csr_w, src, dst, e, a.buffer + dst, payload);
            if (dd && acc_success(st)) enqueue_one(app, a, s, dst, acc, lq);
            if (!acc_continue(st)) {
                ++e;
                break;
            }
        }
        acc.edges += e - beg;
    }

    // Chunks of the heavy vertices registered in table `set`, spread over all warps.
    static __device__ void heavy_phase(App &app, const Args &a, const Snap &s, uint32_t set, bool dd, Acc &acc) {
        if constexpr (has_min_relax<App, TB, TW>::value)
            heavy_phase_relax(app, a, s, set, dd, acc);
        else
            heavy_phase_generic(app, a, s, set, dd, acc);
    }

    static __device__ void heavy_phase_generic(App &app, const Args &a, const Snap &s, uint32_t set, bool dd,
                                               Acc &acc) {
        const uint32_t C = min(dev::ld_l2(&a.ctrl->cnt.chunk_count[set]), a.chunk_cap);
        const uint32_t H = min(dev::ld_l2(&a.ctrl->cnt.heavy_count[set]), a.heavy_cap);
        const uint32_t *own = a.chunk_owner + (size_t)set * a.chunk_cap;
        const HeavyItem<TB> *items = a.heavy + (size_t)set * a.heavy_cap;
        const uint32_t lane = dev::lane_id();
        const uint32_t ce = a.p.chunk_edges;
        for (uint32_t ch = gwarp(); ch < C; ch += nwarps()) {
            const uint32_t e = dev::ld_l2(own + ch);
            if (e >= H) continue;
            const HeavyItem<TB> h = items[e];
            if (ch < h.chunk_base) continue;
            uint32_t lo, hi;
            chunk_span(h.beg, h.deg, ce, ch - h.chunk_base, &lo, &hi);
            if (lo >= hi) continue;
            const uint32_t off = lo - h.beg;
            const uint32_t len = hi - lo;
            for (uint32_t k = 0; k < len; k += 128) {
                uint32_t d[4], wt[4];
                bool want[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const uint32_t i = k + 32u * j + lane;
                    d[j] = 0;
                    wt[j] = 1;
                    if (i < len) {
                        const uint32_t edge = h.beg + off + i;
                        d[j] = a.csr.edge_dest(edge);
                        if constexpr (!std::is_same<TW, graphs::NoWeight>::value)
                            if (a.csr_w) wt[j] = __ldg(a.csr_w + edge);
                    }
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    want[j] = false;
                    if (k + 32u * j + lane < len) {
                        const int st = accumulate_w(app, h.src, d[j], wt[j], a.buffer + d[j], h.payload);
                        want[j] = dd && acc_success(st);
                    }
                }
                enqueue_batch<4>(app, a, s, d, want, nullptr, acc, nullptr);
            }
            if (lane == 0) acc.edges += len;
        }
    }

    // The 8 edge slots [base, base + 8) of one window of a hub chunk, already in
    // registers (d, wt), relaxed by one lane: the 8 current destination values
    // are loaded together, the improving minima issued as reductions, the
    // improved destinations pushed in one batch.  All 32 lanes must call.
    static __device__ __forceinline__ void relax_slots(App &app, const Args &a, const Snap &s, uint32_t src,
                                                       TB payload, uint32_t lo, uint32_t hi, uint32_t base,
                                                       uint32_t (&d)[8], const uint32_t (&wt)[8], bool dd, Acc &acc) {
        if constexpr (has_min_relax<App, TB, TW>::value) {
            TB cand[8], cur[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint32_t i = base + j;
                const bool in = i >= lo && i < hi;
                cand[j] = in ? app.RelaxCandidate(src, d[j], (TW)wt[j], payload) : std::numeric_limits<TB>::max();
                cur[j] = in ? dev::ld_l2(a.buffer + d[j]) : (TB)0;
            }
            bool want[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                want[j] = cand[j] < cur[j];
                if (want[j]) atomicMin(a.buffer + d[j], cand[j]);
                want[j] = want[j] && dd;
            }
            enqueue_batch<8>(app, a, s, d, want, cand, acc, nullptr);
        }
    }

    // Hub chunks of a min-relax functor: lane l takes the 8 edge slots
    // [w + 8l, w + 8l + 8) of each 256-slot window w of the chunk (windows
    // start on the chunk grid's 16-byte boundaries) and relaxes them with
    // relax_slots.  With 256-edge chunks (one window each) and 16-byte aligned
    // edge arrays, a chunk's destinations and weights are staged by the TMA
    // engine: while the warp relaxes chunk k from registers, a bulk copy
    // (cp.async.bulk, completed on the warp's mbarrier) brings chunk k+1's
    // window into the warp's shared-memory stage, and lane 0 already fetches
    // the descriptor of chunk k+2, so the adjacency's HBM latency overlaps
    // the relaxations instead of preceding them.  Otherwise lanes load their
    // slots with two 16-byte loads per array.
    struct alignas(16) ChunkStage {
        uint32_t dst[256];
        uint32_t wt[256];
        unsigned long long bar;
        uint32_t src, lo, hi, w0, ncopy, pad;
        TB pay;
    };

    static __device__ void heavy_phase_relax(App &app, const Args &a, const Snap &s, uint32_t set, bool dd,
                                             Acc &acc) {
        if constexpr (has_min_relax<App, TB, TW>::value) {
            const uint32_t C = min(dev::ld_l2(&a.ctrl->cnt.chunk_count[set]), a.chunk_cap);
            const uint32_t H = min(dev::ld_l2(&a.ctrl->cnt.heavy_count[set]), a.heavy_cap);
            const uint32_t *own = a.chunk_owner + (size_t)set * a.chunk_cap;
            const HeavyItem<TB> *items = a.heavy + (size_t)set * a.heavy_cap;
            const uint32_t lane = dev::lane_id();
            const uint32_t ce = a.p.chunk_edges;
            const uint32_t E = a.csr.nedges;
            const uint32_t *col = a.csr.edge_dst;
            const uint32_t *wts = a.csr_w;
            const bool vec = (reinterpret_cast<uintptr_t>(col) & 15u) == 0 &&
                             (reinterpret_cast<uintptr_t>(wts) & 15u) == 0;
            const uint64_t pol = dev::stream_policy();
            const uint32_t nw = nwarps();
            if (vec && ce == 256u && a.p.stage_chunks) {
                heavy_phase_staged(app, a, s, dd, acc, C, H, own, items);
                return;
            }
            uint32_t ch = gwarp();
            uint32_t e_next = ch < C ? dev::ld_l2(own + ch) : 0xffffffffu;
            for (; ch < C; ch += nw) {
                const uint32_t e = e_next;
                e_next = ch + nw < C ? dev::ld_l2(own + ch + nw) : 0xffffffffu;
                if (e >= H) continue;
                const HeavyItem<TB> h = items[e];
                if (ch < h.chunk_base) continue;
                uint32_t lo, hi;
                chunk_span(h.beg, h.deg, ce, ch - h.chunk_base, &lo, &hi);
                if (lo >= hi) continue;
                for (uint32_t w0 = lo & ~3u; w0 < hi; w0 += 256u) {
                    const uint32_t base = w0 + lane * 8u;
                    uint32_t d[8], wt[8];
                    if (vec && base + 8u <= E) {
                        const uint4 x = dev::ldg_v4_stream(col + base, pol), y = dev::ldg_v4_stream(col + base + 4, pol);
                        d[0] = x.x, d[1] = x.y, d[2] = x.z, d[3] = x.w, d[4] = y.x, d[5] = y.y, d[6] = y.z, d[7] = y.w;
                        if (wts) {
                            const uint4 p = dev::ldg_v4_stream(wts + base, pol), q = dev::ldg_v4_stream(wts + base + 4, pol);
                            wt[0] = p.x, wt[1] = p.y, wt[2] = p.z, wt[3] = p.w, wt[4] = q.x, wt[5] = q.y, wt[6] = q.z,
                            wt[7] = q.w;
                        } else {
#pragma unroll
                            for (int j = 0; j < 8; ++j) wt[j] = 1u;
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const uint32_t i = base + j;
                            const bool in = i >= lo && i < hi;
                            d[j] = in ? dev::ldg_stream(col + i, pol) : 0u;
                            wt[j] = in && wts ? dev::ldg_stream(wts + i, pol) : 1u;
                        }
                    }
                    relax_slots(app, a, s, h.src, h.payload, lo, hi, base, d, wt, dd, acc);
                }
                if (lane == 0) acc.edges += hi - lo;
            }
        }
    }

    // The staged form of heavy_phase_relax (256-edge chunks, aligned arrays).
    static __device__ void heavy_phase_staged(App &app, const Args &a, const Snap &s, bool dd, Acc &acc,
                                              uint32_t C, uint32_t H, const uint32_t *own,
                                              const HeavyItem<TB> *items) {
        __shared__ ChunkStage stage[kWarpsPerBlock];
        ChunkStage &st = stage[dev::warp_id()];
        const uint32_t lane = dev::lane_id();
        const uint32_t E = a.csr.nedges;
        const uint32_t *col = a.csr.edge_dst;
        const uint32_t *wts = a.csr_w;
        const uint32_t nw = nwarps();
        uint32_t c = gwarp();
        if (c >= C) return;
        // Lane 0 only: stage chunk `ch` (descriptor h, from owner entry e) — the
        // window's metadata, then one arrival announcing the copy's bytes and the
        // bulk copies; a chunk with no edges completes the phase with 0 bytes.
        auto issue = [&](uint32_t ch, uint32_t e, const HeavyItem<TB> &h) {
            uint32_t lo = 0, hi = 0;
            if (e < H && ch >= h.chunk_base) chunk_span(h.beg, h.deg, 256u, ch - h.chunk_base, &lo, &hi);
            if (lo >= hi) lo = hi = 0;
            const uint32_t w0 = lo & ~3u;
            const uint32_t nc = hi > lo ? (min(256u, E - w0) & ~3u) : 0u;  // whole 16-byte groups inside the array
            st.src = h.src;
            st.pay = h.payload;
            st.lo = lo;
            st.hi = hi;
            st.w0 = w0;
            st.ncopy = nc;
            dev::fence_proxy_async_smem();
            dev::mbar_arrive_expect_tx(&st.bar, nc * 4u * (wts ? 2u : 1u));
            if (nc) {
                dev::bulk_copy_g2s(st.dst, col + w0, nc * 4u, &st.bar);
                if (wts) dev::bulk_copy_g2s(st.wt, wts + w0, nc * 4u, &st.bar);
            }
        };
        auto item = [&](uint32_t e) {
            HeavyItem<TB> h{};
            if (e < H) h = items[e];
            return h;
        };
        uint32_t e1 = 0xffffffffu, e2 = 0xffffffffu;
        HeavyItem<TB> h1{};
        if (lane == 0) {
            dev::mbar_init(&st.bar, 1);
            const uint32_t e0 = dev::ld_l2(own + c);
            issue(c, e0, item(e0));
            e1 = c + nw < C ? dev::ld_l2(own + c + nw) : 0xffffffffu;
            h1 = item(e1);
            e2 = c + 2 * nw < C ? dev::ld_l2(own + c + 2 * nw) : 0xffffffffu;
        }
        __syncwarp();
        uint32_t parity = 0;
        bool ok = true;
        for (; c < C; c += nw) {
            // every lane observes the copy's completion itself; the verdict is warp-uniform
            ok = __all_sync(dev::kFullMask, dev::mbar_wait_bounded(&st.bar, parity, a.p.timeout_ns));
            if (!ok) break;
            parity ^= 1u;
            __syncwarp();
            const uint32_t lo = st.lo, hi = st.hi, w0 = st.w0, nc = st.ncopy, src = st.src;
            const TB pay = st.pay;
            const uint32_t k0 = lane * 8u;
            uint32_t d[8], wt[8];
            if (k0 + 8u <= nc) {
                const uint4 x = *reinterpret_cast<const uint4 *>(st.dst + k0);
                const uint4 y = *reinterpret_cast<const uint4 *>(st.dst + k0 + 4);
                d[0] = x.x, d[1] = x.y, d[2] = x.z, d[3] = x.w, d[4] = y.x, d[5] = y.y, d[6] = y.z, d[7] = y.w;
                if (wts) {
                    const uint4 p = *reinterpret_cast<const uint4 *>(st.wt + k0);
                    const uint4 q = *reinterpret_cast<const uint4 *>(st.wt + k0 + 4);
                    wt[0] = p.x, wt[1] = p.y, wt[2] = p.z, wt[3] = p.w, wt[4] = q.x, wt[5] = q.y, wt[6] = q.z,
                    wt[7] = q.w;
                } else {
#pragma unroll
                    for (int j = 0; j < 8; ++j) wt[j] = 1u;
                }
            } else {  // slots past the staged groups: the array's last (< 4) edges, read directly
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const uint32_t slot = k0 + j, i = w0 + slot;
                    const bool in = i >= lo && i < hi;
                    d[j] = in ? (slot < nc ? st.dst[slot] : __ldg(col + i)) : 0u;
                    wt[j] = in && wts ? (slot < nc ? st.wt[slot] : __ldg(wts + i)) : 1u;
                }
            }
            __syncwarp();  // the stage is free: the next chunk's copy may overwrite it
            if (lane == 0 && c + nw < C) {
                issue(c + nw, e1, h1);
                e1 = e2;
                h1 = item(e1);  // arrives while this chunk relaxes
                e2 = c + 3 * nw < C ? dev::ld_l2(own + c + 3 * nw) : 0xffffffffu;
            }
            if (lo < hi) {
                relax_slots(app, a, s, src, pay, lo, hi, w0 + k0, d, wt, dd, acc);
                if (lane == 0) acc.edges += hi - lo;
            }
        }
        if (!ok) {
            // a copy that never completed: report, and give it one more bounded
            // wait before the stage can be reused or the block exits
            if (lane == 0) atomicOr(&a.ctrl->cnt.error, dev::kErrTimeout);
            dev::mbar_wait_bounded(&st.bar, parity, a.p.timeout_ns);
            return;
        }
        __syncwarp();
        if (lane == 0) dev::mbar_inval(&st.bar);
        __syncwarp();
    }

    static __device__ void clear_dirty(const Args &a, const Snap &s) {
        if (!s.dirty) return;
        for (uint32_t w = gthread(); w < a.nwords; w += nthreads()) {
            if (s.dirty & 1u) a.bitmap[0][w] = 0;
            if (s.dirty & 2u) a.bitmap[1][w] = 0;
        }
    }

    // Worklist items that a round consumes without popping lose their queued bit.
    static __device__ void release_input_flags(const Args &a, const Snap &s, bool to_bitmap) {
        const uint32_t *Q = a.queue[s.qin];
        for (uint32_t i = gthread(); i < s.F; i += nthreads()) {
            const uint32_t v = dev::ld_l2(Q + i);
            dev::bitmap_clear(a.qflag[s.qin], v);
            if (to_bitmap) dev::bitmap_set(a.bitmap[s.bin], v);  // Queue2Bitmap (driver.cuh:119-129)
        }
    }

    // ---------------------------------------------------------------- --wl_sort
    // The reference sorts the worklist of every data-driven push round by
    // vertex id (thrust::sort, framework.cuh:488-496).  Here the input slot's
    // queued bitmap already holds exactly the worklist's vertices when a round
    // starts (every bit set comes with an append to that slot, and bits are
    // cleared only while the slot is the input), so the sort is a pass over
    // that bitmap in two barrier-separated phases: each block counts the bits
    // of its contiguous word range; each block writes its range's vertices in
    // ascending order at the sum of the counts before it.

    // Block-wide exclusive scan of x; *total = the block's sum.  All threads call.
    static __device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t *total) {
        __shared__ uint32_t part[kWarpsPerBlock];
        const uint32_t lane = dev::lane_id(), wid = threadIdx.x >> 5;
        const uint32_t incl = dev::warp_inclusive_scan(x);
        if (lane == 31) part[wid] = incl;
        __syncthreads();
        uint32_t before = 0, sum = 0;
#pragma unroll
        for (uint32_t k = 0; k < kWarpsPerBlock; ++k) {
            const uint32_t p = part[k];
            if (k < wid) before += p;
            sum += p;
        }
        __syncthreads();  // part[] is free for the next call
        *total = sum;
        return before + incl - x;
    }

    static __device__ __forceinline__ void sort_range(const Args &a, uint32_t &w0, uint32_t &w1) {
        const uint32_t per = (a.nwords + g_team_size - 1) / g_team_size;
        w0 = min(a.nwords, g_team_rank * per);
        w1 = min(a.nwords, w0 + per);
    }

    static __device__ void sort_count(const Args &a, const Snap &s) {
        uint32_t w0, w1, total;
        sort_range(a, w0, w1);
        const uint32_t *bits = a.qflag[s.qin];
        uint32_t cnt = 0;
        for (uint32_t w = w0 + threadIdx.x; w < w1; w += blockDim.x) cnt += __popc(dev::ld_l2(bits + w));
        block_exclusive_scan(cnt, &total);
        if (threadIdx.x == 0) __stcg(a.sort_counts + g_team_rank, total);
    }

    static __device__ void sort_emit(const Args &a, const Snap &s) {
        uint32_t w0, w1, total;
        sort_range(a, w0, w1);
        uint32_t before = 0;
        for (uint32_t b = threadIdx.x; b < g_team_rank; b += blockDim.x) before += dev::ld_l2(a.sort_counts + b);
        block_exclusive_scan(before, &total);
        uint32_t off = total;
        const uint32_t *bits = a.qflag[s.qin];
        uint32_t *Q = a.queue[s.qin];
        for (uint32_t base = w0; base < w1; base += blockDim.x) {  // block-uniform trip count
            const uint32_t w = base + threadIdx.x;
            uint32_t x = w < w1 ? dev::ld_l2(bits + w) : 0u;
            const uint32_t c = __popc(x);
            uint32_t pos = off + block_exclusive_scan(c, &total);
            while (x) {
                __stcg(Q + pos++, w * 32u + (uint32_t)(__ffs(x) - 1));
                x &= x - 1;
            }
            off += total;
        }
    }

    // ---------------------------------------------------------------- push
    // Phase A of a push round over worklist items (DD) or all vertices (TD).
    // Sampling priority threshold (GetPriorityThreshold, algo_variants.cuh:98-131):
    // the buffers of 1000 vertices drawn at random are sorted and the value at
    // index 1000 * (1 - cut) becomes the round's threshold.  The reference draws
    // with the unseeded std::rand; here a counter-based hash of (round, index).
    // Run by one block (all its threads) in `scratch` (1024 buffer values of
    // shared memory that topology-driven rounds leave unused), which publishes
    // the threshold in the control block's prio_raw.
    static __device__ void sample_threshold(const Args &a, const Snap &s, TB *vals) {
        constexpr uint32_t kSample = 1000, kPad = 1024;
        const uint32_t nn = a.csr.nnodes;
        const uint32_t n = min(kSample, nn);
        for (uint32_t i = threadIdx.x; i < kPad; i += blockDim.x) {
            TB x = std::numeric_limits<TB>::max();
            if (i < n) {
                unsigned long long h = ((unsigned long long)s.round << 32) ^ i ^ 0x9E3779B97F4A7C15ull;
                h = (h ^ (h >> 30)) * 0xBF58476D1CE4E5B9ull;
                h = (h ^ (h >> 27)) * 0x94D049BB133111EBull;
                h ^= h >> 31;
                x = dev::ld_l2(a.buffer + (uint32_t)(h % nn));
            }
            vals[i] = x;
        }
        __syncthreads();
        for (uint32_t k = 2; k <= kPad; k <<= 1)
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < kPad / 2; i += blockDim.x) {
                    const uint32_t lo = ((i & ~(j - 1)) << 1) | (i & (j - 1)), hi = lo + j;
                    const TB x = vals[lo], y = vals[hi];
                    if ((x > y) == ((lo & k) == 0)) {
                        vals[lo] = y;
                        vals[hi] = x;
                    }
                }
                __syncthreads();
            }
        if (threadIdx.x == 0) {
            uint32_t idx = (uint32_t)((float)n * (1.0f - a.p.sample_cut));
            if (idx >= n) idx = n - 1;
            __stcg(&a.ctrl->rs.prio_raw, to_raw<TB>(vals[idx]));
        }
        __syncthreads();
    }

    // The r-th (from 0) set bit of x; r < popc(x).
    static __device__ __forceinline__ uint32_t nth_set_bit(uint32_t x, uint32_t r) {
        uint32_t pos = 0;
#pragma unroll
        for (uint32_t w = 16; w > 0; w >>= 1) {
            const uint32_t lo = __popc(x & ((1u << w) - 1u));
            if (r >= lo) {
                r -= lo;
                x >>= w;
                pos += w;
            } else {
                x &= (1u << w) - 1u;
            }
        }
        return pos;
    }

    static __device__ void push_phase_a(App &app, const Args &a, const Snap &s, WarpLB<TB> &wlb, bool dd,
                                        int lb, Acc &acc, LocalQ *lq = nullptr) {
        const uint32_t lane = dev::lane_id();
        const uint32_t N = dd ? s.F : a.csr.nnodes;
        const uint32_t *Q = a.queue[s.qin];
        if (dd && a.p.bitmap_frontier) {
            // The worklist is the input slot's bitmap.  A warp takes 32 words
            // spread evenly over the vertex range (word gw + k * nwarps for lane
            // k), so every warp samples every region of the id space (RMAT
            // graphs put their dense rows at low ids); it clears the words it
            // took (no other writer touches the input slot this round), ranks
            // their set bits with one warp scan and processes them 32 at a time
            // exactly like queue items.
            uint32_t *bits = a.qflag[s.qin];
            const uint32_t W = a.nwords, nw = nwarps();
            uint32_t popped = 0;
            for (uint32_t b = gwarp(); b < W; b += 32u * nw) {
                const uint32_t wi = b + lane * nw;
                uint32_t x = 0;
                if (wi < W) {
                    x = dev::ld_l2(bits + wi);
                    if (x) bits[wi] = 0u;
                }
                const uint32_t c = __popc(x);
                const uint32_t incl = dev::warp_inclusive_scan(c);
                const uint32_t total = __shfl_sync(dev::kFullMask, incl, 31);
                popped += c;
                if (total == 0) continue;
                wlb.scan_excl[lane] = incl - c;
                wlb.scan_bits[lane] = x;
                __syncwarp();
                for (uint32_t g0 = 0; g0 < total; g0 += 32) {
                    const uint32_t r = g0 + lane;
                    const bool valid = r < total;
                    uint32_t v = 0;
                    if (valid) {
                        const uint32_t k = owner(wlb.scan_excl, r);
                        v = (b + k * nw) * 32u + nth_set_bit(wlb.scan_bits[k], r - wlb.scan_excl[k]);
                    }
                    push_item(app, a, s, wlb, true, lb, acc, lq, v, valid, false);
                }
                __syncwarp();
            }
            popped = dev::warp_sum(popped);
            if (lane == 0 && popped) dev::red_add(&a.ctrl->cnt.popped, popped);
        } else {
            for (uint32_t base = gwarp() * 32; base < N; base += nwarps() * 32) {
                const uint32_t i = base + lane;
                const bool valid = i < N;
                uint32_t v = 0;
                if (valid) v = dd ? dev::ld_l2(Q + i) : i;
                push_item(app, a, s, wlb, dd, lb, acc, lq, v, valid, dd);
            }
        }
        if (lq) local_levels(app, a, s, wlb, lb, acc, lq);
    }

    // One worklist item per lane (valid lanes): pop (queue worklists), far-pile
    // check, combine, heavy registration and the warp's expansion.  All 32
    // lanes must call.
    static __device__ __forceinline__ void push_item(App &app, const Args &a, const Snap &s, WarpLB<TB> &wlb,
                                                     bool dd, int lb, Acc &acc, LocalQ *lq, uint32_t v, bool valid,
                                                     bool pop) {
        const TB prio = from_raw<TB>(s.prio_raw);
        Counters *n = &a.ctrl->cnt;
        {
            bool proceed = valid;
            bool keep = false;
            if (valid) {
                // sampling priority: a topology-driven round takes only the
                // vertices above this round's sampled threshold (driver.cuh:362-383)
                if (!dd && a.p.sample_cut > 0.f) proceed = app.App::IsHighPriority(prio, dev::ld_l2(a.buffer + v));
                if (dd) {
                    if (pop) dev::bitmap_clear(a.qflag[s.qin], v);  // pop
                    if (s.pile && !app.App::IsHighPriority(prio, dev::ld_l2(a.buffer + v))) {
                        // far pile: vertices still outside the priority window move to the new pile
                        if (a.p.bitmap_frontier) {
                            dev::bitmap_set_nr(a.qflag[s.qlo], v);
                            keep = true;
                        } else {
                            keep = dev::bitmap_set(a.qflag[s.qlo], v);
                        }
                        proceed = false;
                    }
                }
            }
            if (dd && s.pile) {
                if (a.p.bitmap_frontier)
                    count_pushes(n, s, false, keep);
                else
                    dev::warp_append(a.queue[s.qlo], &n->qcount[s.qlo], a.queue_cap, keep, v, &n->error);
                if (keep) count_enq(a, acc, false, v);
            }
            // the row offsets are read-only: load them alongside the combine's
            // loads instead of after it (one dependent memory trip less per round)
            uint32_t beg = 0, end = 0;
            if (proceed) {
                beg = a.csr.begin_edge(v);
                end = a.csr.end_edge(v);
            }
            TB payload{};
            bool sched = false;
            if (proceed) {
                auto pr = app.App::CombineValueBuffer(v, a.value + v, a.buffer + v);
                payload = pr.first;
                sched = pr.second;
            }
            uint32_t deg = sched ? end - beg : 0u;
            if (lb == LB_NONE) {
                if (deg) expand_serial(app, a, s, v, beg, deg, payload, dd, acc, lq);
                return;
            }
            const bool heavy = deg > a.p.heavy_threshold;
            register_heavy(a, s.round & 1u, heavy, v, beg, deg, payload);
            if (heavy) deg = 0;
            expand_warp(app, a, s, wlb, v, beg, deg, payload, dd, acc, lq);
        }
    }

    // Local lookahead: the block processes the vertices it discovered itself,
    // up to local_depth levels deep, without waiting for the round's barrier
    // (reorder-safe functors: any order of pushes reaches the same result).
    // Only under a forced ASYNC_PUSH_DD: the worklist it leaves mixes levels,
    // and a pull round that takes the first frontier neighbour's offer and
    // stops (BFS, pull_functor.h:138-188) would keep a level that is too high.
    // Heavy vertices are left to the worklist uncombined, so that a later round
    // splits them into chunks; whatever is still queued at the end goes to the
    // worklist too.  Every thread of the block must call.
    static __device__ void local_levels(App &app, const Args &a, const Snap &s, WarpLB<TB> &wlb, int lb, Acc &acc,
                                        LocalQ *lq) {
        const uint32_t lane = dev::lane_id(), warp = dev::warp_id();
        for (uint32_t d = 0; d < a.p.local_depth; ++d) {
            __syncthreads();
            const uint32_t in = lq->out;
            const uint32_t cnt = min(lq->n[in], kLocalCap);
            __syncthreads();
            if (cnt == 0) return;  // the same values in every thread
            if (threadIdx.x == 0) {
                lq->out = in ^ 1u;
                lq->n[in ^ 1u] = 0;
            }
            __syncthreads();
            for (uint32_t base = warp * 32; base < cnt; base += kWarpsPerBlock * 32) {
                const uint32_t i = base + lane;
                const bool valid = i < cnt;
                const uint32_t v = valid ? lq->item[in][i] : 0u;
                uint32_t beg = 0, end = 0;
                if (valid) {
                    beg = a.csr.begin_edge(v);
                    end = a.csr.end_edge(v);
                }
                const bool heavy = valid && lb != LB_NONE && end - beg > a.p.heavy_threshold;
                enqueue(app, a, s, v, heavy, acc);
                TB payload{};
                bool sched = false;
                if (valid && !heavy) {
                    auto pr = app.App::CombineValueBuffer(v, a.value + v, a.buffer + v);
                    payload = pr.first;
                    sched = pr.second;
                }
                const uint32_t deg = sched ? end - beg : 0u;
                if (lb == LB_NONE) {
                    if (deg) expand_serial(app, a, s, v, beg, deg, payload, true, acc, lq);
                    continue;
                }
                expand_warp(app, a, s, wlb, v, beg, deg, payload, true, acc, lq);
            }
        }
        __syncthreads();
        const uint32_t in = lq->out;
        const uint32_t cnt = min(lq->n[in], kLocalCap);
        for (uint32_t base = warp * 32; base < cnt; base += kWarpsPerBlock * 32) {
            const uint32_t i = base + lane;
            const bool valid = i < cnt;
            enqueue(app, a, s, valid ? lq->item[in][i] : 0u, valid, acc);
        }
    }

    // ---------------------------------------------------------------- pull
    // CombineValueBuffer over every vertex; scheduled vertices form the middle
    // list (variants/common.cuh:17-84).  `sync` writes the combined buffer to
    // tmp (SYNC_PULL_*), else back into buffer (ASYNC_PULL_DD, algo_variants.cuh:842-849).
    static __device__ void combine_all(App &app, const Args &a, bool sync, bool build_middle = true) {
        const uint32_t lane = dev::lane_id();
        const uint32_t N = a.csr.nnodes;
        Counters *n = &a.ctrl->cnt;
        for (uint32_t base = gwarp() * 32; base < N; base += nwarps() * 32) {
            const uint32_t v = base + lane;
            bool want = false;
            if (v < N) {
                auto pr = app.App::CombineValueBuffer(v, a.value + v, a.buffer + v);
                if (sync)
                    a.tmp[v] = pr.first;
                else
                    a.buffer[v] = pr.first;
                want = pr.second;
            }
            if (build_middle) dev::warp_append(a.middle, &n->middle_count, a.csr.nnodes, want, v, &n->error);
        }
    }

    // Pull into one destination, sequentially over its in-edges (early exit on BREAK).
    static __device__ bool pull_serial(App &app, const Args &a, const Snap &s, uint32_t v, uint32_t beg,
                                       uint32_t deg, bool dd, bool sync, Acc &acc) {
        const TB *srcbuf = sync ? a.tmp : a.buffer;
        const uint32_t *bin = a.bitmap[s.bin];
        bool hit = false;
        uint32_t e = beg;
        for (; e < beg + deg; ++e) {
            const uint32_t u = a.csc.edge_src(e);
            if (dd && !dev::bitmap_test(bin, u)) continue;
            const int st = accumulate<App, TB, TW>(app, a.csc_w, u, v, e, a.buffer + v, dev::ld_l2(srcbuf + u));
            hit |= acc_success(st);
            if (!acc_continue(st)) {
                ++e;
                break;
            }
        }
        acc.edges += e - beg;
        return hit;
    }

    // Warp-cooperative data-driven pull into up to 32 destinations of at most
    // pull_warp_threshold in-edges each (one per lane; deg 0 = none): the warp
    // walks their concatenated in-edge lists 32 edges at a time, so one
    // coalesced load of sources and one batch of frontier-bit tests cover
    // several destinations at once.  Per destination the frontier sources are
    // taken in edge order, as the serial scan takes them (async_pull_dd.cuh:
    // 34-136): the lowest pending lane of each destination calls
    // AccumulateBuffer, a BREAK retires the destination (no further calls,
    // later batches skip its edges), otherwise its next frontier source
    // follows.  Returns whether some call succeeded for the lane's own
    // destination.  All 32 lanes must call.
    static __device__ bool pull_coop(App &app, const Args &a, const Snap &s, WarpLB<TB> &w, uint32_t v,
                                     uint32_t beg, uint32_t deg, bool sync, Acc &acc) {
        const uint32_t lane = dev::lane_id();
        const TB *srcbuf = sync ? a.tmp : a.buffer;
        const uint32_t *bin = a.bitmap[s.bin];
        const uint32_t incl = dev::warp_inclusive_scan(deg);
        const uint32_t total = __shfl_sync(dev::kFullMask, incl, 31);
        if (total == 0) return false;
        w.excl[lane] = incl - deg;
        w.beg[lane] = beg;
        w.src[lane] = v;
        __syncwarp();
        const uint32_t has = __ballot_sync(dev::kFullMask, deg > 0);
        uint32_t done = 0, hitm = 0, scanned = 0;
        for (uint32_t eb = 0; eb < total; eb += 32) {
            const uint32_t e = eb + lane;
            const bool valid = e < total;
            const uint32_t k = valid ? owner(w.excl, e) : 0u;
            const bool live = valid && !((done >> k) & 1u);
            bool cand = false;
            uint32_t u = 0, edge = 0;
            if (live) {
                edge = w.beg[k] + (e - w.excl[k]);
                u = dev::ldg_stream(a.csc.edge_source + edge, dev::stream_policy());
                cand = dev::bitmap_test_l1(bin, u);  // the input frontier is read-only this round
            }
            scanned += __popc(__ballot_sync(dev::kFullMask, live));
            // first lane of this lane's destination inside the batch
            const uint32_t first = valid ? (w.excl[k] > eb ? w.excl[k] - eb : 0u) : lane;
            const uint32_t below = ((1u << lane) - 1u) & ~((1u << first) - 1u);
            uint32_t P = __ballot_sync(dev::kFullMask, cand);
            while (P) {
                const bool elected = ((P >> lane) & 1u) && !(P & below);
                bool ok = false, brk = false;
                if (elected) {
                    const uint32_t dst = w.src[k];
                    const int st =
                        accumulate<App, TB, TW>(app, a.csc_w, u, dst, edge, a.buffer + dst, dev::ld_l2(srcbuf + u));
                    ok = acc_success(st);
                    brk = !acc_continue(st);
                }
                hitm |= __reduce_or_sync(dev::kFullMask, ok ? (1u << k) : 0u);
                done |= __reduce_or_sync(dev::kFullMask, brk ? (1u << k) : 0u);
                P &= ~__ballot_sync(dev::kFullMask, elected || (valid && ((done >> k) & 1u)));
            }
            if ((done & has) == has) break;  // every destination retired
        }
        if (lane == 0) acc.edges += scanned;
        __syncwarp();
        return (hitm >> lane) & 1u;
    }

    // The whole warp pulls into one high in-degree destination, 32 in-edges per step.
    static __device__ bool pull_warp(App &app, const Args &a, const Snap &s, uint32_t v, uint32_t beg, uint32_t deg,
                                     bool dd, bool sync, Acc &acc) {
        const uint32_t lane = dev::lane_id();
        const TB *srcbuf = sync ? a.tmp : a.buffer;
        const uint32_t *bin = a.bitmap[s.bin];
        bool hit = false;
        uint32_t scanned = 0;
        for (uint32_t off = 0; off < deg; off += 32) {
            const uint32_t k = off + lane;
            bool brk = false;
            if (k < deg) {
                const uint32_t e = beg + k;
                const uint32_t u = a.csc.edge_src(e);
                if (!dd || dev::bitmap_test(bin, u)) {
                    const int st = accumulate<App, TB, TW>(app, a.csc_w, u, v, e, a.buffer + v, dev::ld_l2(srcbuf + u));
                    hit |= acc_success(st);
                    brk = !acc_continue(st);
                }
            }
            scanned = min(deg, off + 32);
            if (__any_sync(dev::kFullMask, brk)) break;
        }
        if (lane == 0) acc.edges += scanned;
        return __any_sync(dev::kFullMask, hit);
    }

    static __device__ void pull_phase(App &app, const Args &a, const Snap &s, WarpLB<TB> &wlb, bool dd, bool sync,
                                      int lb, Acc &acc) {
        const uint32_t lane = dev::lane_id();
        const uint32_t M = min(dev::ld_l2(&a.ctrl->cnt.middle_count), a.csr.nnodes);
        const bool natural = (M == a.csr.nnodes);  // every vertex scheduled: keep CSC order
        Counters *n = &a.ctrl->cnt;
        for (uint32_t base = gwarp() * 32; base < M; base += nwarps() * 32) {
            const uint32_t i = base + lane;
            const bool valid = i < M;
            uint32_t v = 0, beg = 0, deg = 0;
            if (valid) {
                v = natural ? i : dev::ld_l2(a.middle + i);
                beg = a.csc.begin_edge(v);
                deg = a.csc.end_edge(v) - beg;
            }
            const bool big = valid && lb != LB_NONE && deg > a.p.pull_warp_threshold;
            bool hit = false;
            if (dd && lb != LB_NONE && a.p.pull_coop)
                hit = pull_coop(app, a, s, wlb, v, beg, valid && !big ? deg : 0u, sync, acc);
            else if (valid && !big)
                hit = pull_serial(app, a, s, v, beg, deg, dd, sync, acc);
            uint32_t bigmask = __ballot_sync(dev::kFullMask, big);
            while (bigmask) {
                const uint32_t j = __ffs(bigmask) - 1;
                bigmask &= bigmask - 1;
                const uint32_t vj = __shfl_sync(dev::kFullMask, v, j);
                const uint32_t bj = __shfl_sync(dev::kFullMask, beg, j);
                const uint32_t dj = __shfl_sync(dev::kFullMask, deg, j);
                const bool h = pull_warp(app, a, s, vj, bj, dj, dd, sync, acc);
                if (lane == j) hit = h;
            }
            if (dd) {
                bool want = valid && hit;
                if (want) {
                    dev::bitmap_set(a.bitmap[s.bout], v);
                    want = dev::bitmap_set(a.qflag[s.qhi], v);
                }
                dev::warp_append(a.queue[s.qhi], &n->qcount[s.qhi], a.queue_cap, want, v, &n->error);
                if (want) count_enq(a, acc, true, v);
            }
        }
    }

    // Topology-driven pull for functors with PullReduce: the warp walks the
    // concatenated in-edge lists of 32 destinations (edge-balanced), folds the
    // pulled values per destination in shared memory and issues one
    // AccumulateBuffer per destination.  Destinations above heavy_threshold
    // in-edges are split into chunks handled by pull_reduce_chunks.
    static __device__ void pull_reduce_td(App &app, const Args &a, const Snap &s, WarpLB<TB> &w, Acc &acc) {
        if constexpr (has_pull_reduce<App, TB>::value && std::is_same<TW, graphs::NoWeight>::value) {
            const uint32_t lane = dev::lane_id();
            const uint32_t N = a.csr.nnodes;
            const TB *srcbuf = a.tmp;
            for (uint32_t base = gwarp() * 32; base < N; base += nwarps() * 32) {
                const uint32_t v = base + lane;
                uint32_t beg = 0, deg = 0;
                if (v < N) {
                    beg = a.csc.begin_edge(v);
                    deg = a.csc.end_edge(v) - beg;
                }
                const bool heavy = deg > a.p.heavy_threshold;
                register_heavy(a, s.round & 1u, heavy, v, beg, deg, app.PullIdentity());
                if (heavy) deg = 0;
                const uint32_t incl = dev::warp_inclusive_scan(deg);
                const uint32_t total = __shfl_sync(dev::kFullMask, incl, 31);
                w.excl[lane] = incl - deg;
                w.beg[lane] = beg;
                w.pay[lane] = app.PullIdentity();
                __syncwarp();
                // Each lane reduces one contiguous 1/32 of the warp's concatenated
                // in-edge lists, four independent gathers at a time, with one owner
                // search at its start; a destination wholly inside one lane's range
                // is written by that lane, the (at most two) segments a lane shares
                // with neighbouring lanes are combined afterwards.
                const uint32_t per = (total + 31) / 32;
                const uint32_t lo = min(total, lane * per), hi = min(total, lo + per);
                w.partk[0][lane] = w.partk[1][lane] = 0xffffffffu;
                if (lo < hi) {
                    uint32_t k = owner(w.excl, lo);
                    uint32_t e = lo;
                    bool first = true;
                    while (e < hi) {
                        const uint32_t seg_lo = w.excl[k];
                        uint32_t seg_hi = total;  // next lane with a larger start
                        for (uint32_t j = k + 1; j < 32; ++j)
                            if (w.excl[j] > seg_lo) {
                                seg_hi = w.excl[j];
                                break;
                            }
                        const uint32_t end = min(hi, seg_hi);
                        const uint32_t *src = a.csc.edge_source;
                        const uint32_t off = w.beg[k] - seg_lo;  // CSC edge of e is off + e (mod 2^32)
                        TB r = app.PullIdentity();
                        for (; e + 4 <= end; e += 4) {
                            const uint32_t s0 = __ldg(src + (off + e)), s1 = __ldg(src + (off + e + 1));
                            const uint32_t s2 = __ldg(src + (off + e + 2)), s3 = __ldg(src + (off + e + 3));
                            const TB g0 = dev::ld_l2(srcbuf + s0), g1 = dev::ld_l2(srcbuf + s1);
                            const TB g2 = dev::ld_l2(srcbuf + s2), g3 = dev::ld_l2(srcbuf + s3);
                            r = app.PullReduce(r, app.PullReduce(app.PullReduce(g0, g1), app.PullReduce(g2, g3)));
                        }
                        for (; e < end; ++e) r = app.PullReduce(r, dev::ld_l2(srcbuf + __ldg(src + (off + e))));
                        const bool shared = seg_lo < lo || seg_hi > hi;  // other lanes hold part of k
                        if (!shared) {
                            w.pay[k] = r;
                        } else {
                            const int slot = first ? 0 : 1;
                            w.partk[slot][lane] = k;
                            w.part[slot][lane] = r;
                        }
                        first = false;
                        // next destination with edges
                        while (k < 31 && w.excl[k + 1] <= e) ++k;
                    }
                }
                __syncwarp();
                {
                    TB r = w.pay[lane];
                    for (uint32_t j = 0; j < 32; ++j) {
                        if (w.partk[0][j] == lane) r = app.PullReduce(r, w.part[0][j]);
                        if (w.partk[1][j] == lane) r = app.PullReduce(r, w.part[1][j]);
                    }
                    w.pay[lane] = r;
                }
                __syncwarp();
                if (v < N && deg > 0) accumulate<App, TB, TW>(app, a.csc_w, v, v, beg, a.buffer + v, w.pay[lane]);
                if (lane == 0) acc.edges += total;
                __syncwarp();
            }
        }
    }

    // Largest row r in [lo, hi] with col_start[r] <= e: the in-edge row that
    // holds CSC edge e (empty rows share their start with the next row, so the
    // largest such r is the non-empty one).
    static __device__ __forceinline__ uint32_t row_of(const uint32_t *crow, uint32_t lo, uint32_t hi, uint32_t e) {
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo + 1) / 2;
            if (__ldg(crow + mid) <= e)
                lo = mid;
            else
                hi = mid - 1;
        }
        return lo;
    }

    // tile_row[] of the edge-tiled pull, once per launch (all threads of the team).
    static __device__ void compute_tile_rows(const Args &a) {
        const uint32_t V = a.csc.nnodes, E = a.csc.nedges;
        const uint32_t T = (E + kPullTileEdges - 1) / kPullTileEdges;
        for (uint32_t t = gthread(); t <= T; t += nthreads())
            a.tile_row[t] = (t == T || V == 0) ? (V ? V - 1 : 0) : row_of(a.csc.col_start, 0, V - 1, t * kPullTileEdges);
    }

    // Topology-driven pull for functors with PullReduce, tiled over the in-edge
    // array instead of over destinations: a warp takes 256 consecutive CSC
    // edges (8 per lane, two 16-byte index loads, 8 independent gathers of
    // the sources' pulled values in flight per lane), finds each edge's
    // destination row from the tile's row range, folds runs of one row in
    // registers, sums the tile's rows in shared memory and issues one
    // AccumulateBuffer per (row, tile).  Rows of any in-degree need no
    // separate chunk phase: a long row is simply spread over many tiles.
    // The pulled values were written by the combine phase of this round
    // (before a grid barrier), so they are read through L1, where the
    // contributions of high out-degree sources stay resident.
    static __device__ void pull_tiles(App &app, const Args &a, WarpLB<TB> &w, Acc &acc) {
        if constexpr (has_pull_reduce<App, TB>::value && std::is_same<TW, graphs::NoWeight>::value) {
            const uint32_t lane = dev::lane_id();
            const uint32_t V = a.csc.nnodes, E = a.csc.nedges;
            const uint32_t T = (E + kPullTileEdges - 1) / kPullTileEdges;
            const uint32_t *crow = a.csc.col_start;
            const uint32_t *srcs = a.csc.edge_source;
            const bool aligned = (reinterpret_cast<uintptr_t>(srcs) & 15u) == 0;
            const uint64_t pol = dev::stream_policy();
            const TB *vals = a.tmp;
            const TB idn = app.PullIdentity();
            for (uint32_t t = gwarp(); t < T; t += nwarps()) {
                const uint32_t e0 = t * kPullTileEdges + lane * 8u;
                uint32_t s[8];
                if (aligned && e0 + 8u <= E) {
                    const uint4 x = dev::ldg_v4_stream(srcs + e0, pol), y = dev::ldg_v4_stream(srcs + e0 + 4, pol);
                    s[0] = x.x, s[1] = x.y, s[2] = x.z, s[3] = x.w, s[4] = y.x, s[5] = y.y, s[6] = y.z, s[7] = y.w;
                } else {
#pragma unroll
                    for (int j = 0; j < 8; ++j) s[j] = e0 + j < E ? dev::ldg_stream(srcs + e0 + j, pol) : 0u;
                }
                TB g[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) g[j] = e0 + j < E ? dev::ld_l1(vals + s[j]) : idn;
                const uint32_t rlo = __ldg(a.tile_row + t), rhi = __ldg(a.tile_row + t + 1);
                const bool in_smem = rhi - rlo < kPullTileRows;
                if (in_smem) {
                    for (uint32_t k = lane; k <= rhi - rlo; k += 32) w.rowsum[k] = idn;
                    if (lane == 0) w.touched = 0ull;
                    __syncwarp();
                }
                auto flush = [&](uint32_t r, TB v) {
                    if (in_smem) {
                        atomicAdd(&w.rowsum[r - rlo], v);  // shared-memory reduction of the tile's rows
                        atomicOr(&w.touched, 1ull << (r - rlo));
                    } else {
                        accumulate<App, TB, TW>(app, a.csc_w, r, r, 0, a.buffer + r, v);
                    }
                };
                if (e0 < E) {
                    uint32_t r = row_of(crow, rlo, rhi, e0);
                    uint32_t next = r + 1 < V ? __ldg(crow + r + 1) : E;
                    TB run = idn;
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const uint32_t e = e0 + j;
                        if (e < E) {
                            if (e >= next) {
                                flush(r, run);
                                run = idn;
                                r = row_of(crow, r + 1, rhi, e);
                                next = r + 1 < V ? __ldg(crow + r + 1) : E;
                            }
                            run = app.PullReduce(run, g[j]);
                        }
                    }
                    flush(r, run);
                }
                if (in_smem) {
                    __syncwarp();
                    const unsigned long long m = w.touched;
                    for (uint32_t k = lane; k <= rhi - rlo; k += 32)
                        if ((m >> k) & 1ull) accumulate<App, TB, TW>(app, a.csc_w, rlo + k, rlo + k, 0, a.buffer + rlo + k,
                                                                    w.rowsum[k]);
                    __syncwarp();
                }
                if (lane == 0) acc.edges += min(kPullTileEdges, E - t * kPullTileEdges);
            }
        }
    }

    static __device__ void pull_reduce_chunks(App &app, const Args &a, uint32_t set, Acc &acc) {
        if constexpr (has_pull_reduce<App, TB>::value && std::is_same<TW, graphs::NoWeight>::value) {
            const uint32_t C = min(dev::ld_l2(&a.ctrl->cnt.chunk_count[set]), a.chunk_cap);
            const uint32_t H = min(dev::ld_l2(&a.ctrl->cnt.heavy_count[set]), a.heavy_cap);
            const uint32_t *own = a.chunk_owner + (size_t)set * a.chunk_cap;
            const HeavyItem<TB> *items = a.heavy + (size_t)set * a.heavy_cap;
            const uint32_t lane = dev::lane_id();
            const uint32_t ce = a.p.chunk_edges;
            for (uint32_t ch = gwarp(); ch < C; ch += nwarps()) {
                const uint32_t e = dev::ld_l2(own + ch);
                if (e >= H) continue;
                const HeavyItem<TB> h = items[e];
                if (ch < h.chunk_base) continue;
                uint32_t lo, hi;
                chunk_span(h.beg, h.deg, ce, ch - h.chunk_base, &lo, &hi);
                if (lo >= hi) continue;
                const uint32_t len = hi - lo;
                TB r = app.PullIdentity();
                for (uint32_t k = lane; k < len; k += 32)
                    r = app.PullReduce(r, dev::ld_l2(a.tmp + a.csc.edge_src(lo + k)));
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) r = app.PullReduce(r, __shfl_xor_sync(dev::kFullMask, r, d));
                if (lane == 0) {
                    accumulate<App, TB, TW>(app, a.csc_w, h.src, h.src, h.beg, a.buffer + h.src, r);
                    acc.edges += len;
                }
            }
        }
    }

    // RebuildWorklist (driver.cuh:162-178): active vertices -> worklist `slot`.
    // Under a forced topology-driven variant every round scans all vertices and
    // no round reads the worklist, so only the active vertices are counted (for
    // termination and the trace), without queued bits or appends.
    static __device__ __forceinline__ bool count_only(const Args &a) {
        return a.p.forced == V_SYNC_PULL_TD || a.p.forced == V_ASYNC_PUSH_TD;
    }

    static __device__ void rebuild(App &app, const Args &a, uint32_t slot, Acc &acc) {
        const uint32_t lane = dev::lane_id();
        const uint32_t N = a.csr.nnodes;
        Counters *n = &a.ctrl->cnt;
        if (count_only(a)) {
            uint32_t cnt = 0;
            for (uint32_t v = gthread(); v < N; v += nthreads()) cnt += app.App::IsActiveNode(v, dev::ld_l2(a.buffer + v));
            cnt = dev::warp_sum(cnt);
            if (lane == 0 && cnt) atomicAdd(&n->active_count, cnt);
            return;
        }
        for (uint32_t base = gwarp() * 32; base < N; base += nwarps() * 32) {
            const uint32_t v = base + lane;
            bool act = false;
            if (v < N) act = app.App::IsActiveNode(v, dev::ld_l2(a.buffer + v));
            if (act) act = dev::bitmap_set(a.qflag[slot], v);
            dev::warp_append(a.queue[slot], &n->qcount[slot], a.queue_cap, act, v, &n->error);
            if (act) count_enq(a, acc, true, v);
        }
    }

    // ---------------------------------------------------------------- leader (block 0, thread 0)
    // Heavy-vertex chunks of a round run at the start of the next one (see reorder_safe).
    static __device__ __forceinline__ bool defer_chunks(const App &app, const Args &a) {
        return a.p.forced == V_ASYNC_PUSH_DD && a.p.lb_push != LB_NONE && reorder_safe(app);
    }

    static __device__ bool supported(const Args &a, int v) {
        if (v == V_SYNC_PUSH_TD || v == V_SYNC_PUSH_DD || v == V_ASYNC_PULL_TD) return false;
        if (is_pull(v) && !a.p.has_csc) return false;
        return true;
    }

    // PreComputation's statistics for the round about to run (framework.cuh:528-568).
    static __device__ void pre_bookkeeping(const Args &a, PolicyState &ps, uint32_t qin_count,
                                           unsigned long long qin_scout) {
        const int var = ps.rs.variant;
        if (!a.p.collect) return;
        if (is_dd(var)) {
            ps.input_active = qin_count;
            ps.input_workload = is_pull(var) ? 0ull : qin_scout;
            ps.total_workload -= (long long)ps.input_workload;
            if (ps.total_workload < 0) ps.total_workload = 0;
        } else {
            ps.input_workload = a.csr.nedges;
            ps.input_active = a.csr.nnodes;
        }
    }

    static __device__ void publish(const Args &a, const PolicyState &ps) {
        const uint4 *src = reinterpret_cast<const uint4 *>(&ps.rs);
        uint4 *dst = reinterpret_cast<uint4 *>(&a.ctrl->rs);
#pragma unroll
        for (int k = 0; k < 4; ++k) __stcg(dst + k, src[k]);
    }

    static __device__ void finish(const Args &a, PolicyState &ps, unsigned long long now) {
        Ctrl *c = a.ctrl;
        ps.rs.done = 1;
        c->round = ps.rs.round;
        c->max_iteration_reached = ps.max_iteration_reached;
        c->n_trace = ps.n_trace;
        for (int k = 0; k < 8; ++k) c->rounds_by_variant[k] = ps.rounds_by_variant[k];
        c->vertices_processed = ps.vertices_processed;
        c->t_start = ps.t_start;
        c->t_end = now;
    }

    static __device__ void leader_start(const Args &a, PolicyState &ps) {
        Counters *n = &a.ctrl->cnt;
        memset(&ps, 0, sizeof ps);
        RoundState &rs = ps.rs;
        rs.round = 1;
        rs.last_variant = -1;
        rs.variant = a.p.forced >= 0 ? a.p.forced : (a.p.scheme == 0 ? V_ASYNC_PUSH_DD : V_SYNC_PULL_TD);
        ps.inspect_next = 1;
        rs.qin = 0;
        rs.qhi = 1;
        rs.qlo = 2;
        rs.bin = 0;
        rs.bout = 1;
        rs.F = min(dev::ld_l2(&n->qcount[0]), a.queue_cap);
        rs.heavy_expected = a.p.collect ? dev::ld_l2(&n->heavy_enq[0]) : (rs.F > 0);
        rs.prio_raw = a.p.prio_init_raw;
        ps.total_workload = a.p.total_workload0;
        pre_bookkeeping(a, ps, rs.F, dev::ld_l2(&n->scout[0]));
        ps.t_start = ps.t_round_start = dev::globaltimer_ns();
        if (!supported(a, rs.variant)) {
            atomicOr(&n->error, dev::kErrUnsupported);
            finish(a, ps, ps.t_start);
        }
        publish(a, ps);
    }

    static __device__ int traversal_policy(const Args &a, const PolicyState &ps, int var) {
        // GetNextPolicy, TRAVERSAL_SCHEME (hybrid_policy.h:265-288)
        if (is_pull(var) && (double)ps.output_active > (double)a.csr.nnodes / a.p.beta) return V_ASYNC_PULL_DD;
        if ((double)ps.output_workload > (double)ps.total_workload / a.p.alpha) return V_ASYNC_PULL_DD;
        return V_ASYNC_PUSH_DD;
    }

    static __device__ int iterative_policy(PolicyState &ps, int var) {
        // Inspect SYNC_PULL_TD, ASYNC_PUSH_TD, ASYNC_PUSH_DD once each (std::set order,
        // hybrid_policy.h:180-195), then pick the smallest predicted time (130-169, 242-263).
        const int order[3] = {V_SYNC_PULL_TD, V_ASYNC_PUSH_TD, V_ASYNC_PUSH_DD};
        if (ps.inspect_next < 3) return order[ps.inspect_next++];
        if (is_dd(var) && ps.input_workload > 0) ps.time_per_work = ps.policy_time[var] / (float)ps.input_workload;
        int best = -1;
        float bt = 0.f;
        for (int k = 0; k < 3; ++k) {
            const int v = order[k];
            if (!(ps.policy_seen & (1u << v))) continue;
            const float t = is_dd(v) ? ps.time_per_work * (float)ps.output_workload : ps.policy_time[v];
            if (best < 0 || t < bt) {
                best = v;
                bt = t;
            }
        }
        return best < 0 ? var : best;
    }

    static __device__ void leader_end_round(App &app, const Args &a, PolicyState &ps) {
        Counters *n = &a.ctrl->cnt;
        RoundState &rs = ps.rs;
        const int var = rs.variant;
        // counters of this round (independent loads)
        uint32_t qc[3], he[3];
        unsigned long long sc[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            qc[k] = dev::ld_l2(&n->qcount[k]);
            he[k] = dev::ld_l2(&n->heavy_enq[k]);
            sc[k] = dev::ld_l2(&n->scout[k]);
        }
        const uint32_t err = dev::ld_l2(&n->error);
        // chunks of this round's heavy vertices left for the next round's start
        const uint32_t cur = rs.round & 1u;
        const bool deferred = defer_chunks(app, a);
        const uint32_t pend = deferred ? min(dev::ld_l2(&n->chunk_count[cur]), a.chunk_cap) : 0u;
        app.App::PostComputation();
        ps.rounds_by_variant[var & 7]++;
        const unsigned long long now = dev::globaltimer_ns();
        const float round_ms = (float)(now - ps.t_round_start) * 1e-6f;
        ps.vertices_processed += !is_dd(var) ? a.csr.nnodes
                                 : (a.p.bitmap_frontier && var == V_ASYNC_PUSH_DD) ? dev::ld_l2(&n->popped) : rs.F;
        const bool prio_push = a.p.priority && var == V_ASYNC_PUSH_DD;
        const uint32_t out_hi = count_only(a) ? dev::ld_l2(&n->active_count) : qc[rs.qhi];
        const uint32_t out_lo = prio_push ? qc[rs.qlo] : 0;
        ps.output_active = out_hi + out_lo;
        if (a.p.collect) {
            if (!is_pull_dd(var))
                ps.output_workload = sc[rs.qhi] + (prio_push ? sc[rs.qlo] : 0ull);
            else
                ps.output_workload = 1;  // framework.cuh:790
        }
        ps.policy_time[var & 7] = round_ms;
        ps.policy_seen |= 1u << (var & 7);
        if (a.p.trace && a.trace && ps.n_trace < a.trace_cap) {
            sg_round_trace t;
            t.round = rs.round;
            t.variant = var;
            t.in_nodes = ps.input_active;
            t.out_nodes = ps.output_active;
            t.in_workload = ps.input_workload;
            t.out_workload = ps.output_workload;
            t.total_workload = ps.total_workload;
            t.time_ms = round_ms;
            t.pad = 0;
            a.trace[ps.n_trace++] = t;
        }
        int next = var;
        if (a.p.forced < 0) next = a.p.scheme == 0 ? traversal_policy(a, ps, var) : iterative_policy(ps, var);
        const bool fatal = (err & (dev::kErrTimeout | dev::kErrCapacity | dev::kErrChunkCapacity |
                                   dev::kErrUnsupported | dev::kErrOverflow)) != 0;
        const bool work_left = ps.output_active != 0 || pend != 0;
        if (!work_left || rs.round >= a.p.max_iteration || fatal) {
            ps.max_iteration_reached = work_left && rs.round >= a.p.max_iteration;
            finish(a, ps, now);
            publish(a, ps);
            return;
        }
        // rotate worklists
        uint32_t reset_q;
        if (prio_push && out_hi == 0 && pend == 0) {
            // near pile drained: open the next priority window over the far pile (driver.cuh:668-675)
            rs.prio_raw = to_raw<TB>((TB)(from_raw<TB>(rs.prio_raw) + from_raw<TB>(a.p.prio_step_raw)));
            const uint32_t t = rs.qin;
            rs.qin = rs.qlo;
            rs.qlo = t;
            reset_q = rs.qlo;
            rs.pile = 1;
        } else {
            const uint32_t t = rs.qin;
            rs.qin = rs.qhi;
            rs.qhi = t;
            reset_q = rs.qhi;
            rs.pile = 0;
        }
        n->qcount[reset_q] = 0;
        n->scout[reset_q] = 0;
        n->heavy_enq[reset_q] = 0;
        if (is_pull_dd(var)) {
            const uint32_t t = rs.bin;
            rs.bin = rs.bout;
            rs.bout = t;
            rs.dirty = is_pull_dd(next) ? (1u << rs.bout) : 3u;
        } else {
            rs.dirty = 0;
        }
        if (!supported(a, next)) {
            atomicOr(&n->error, dev::kErrUnsupported);
            finish(a, ps, now);
            publish(a, ps);
            return;
        }
        rs.last_variant = var;
        rs.variant = next;
        rs.round++;
        rs.F = min(qc[rs.qin], a.queue_cap);
        rs.heavy_expected = a.p.collect ? he[rs.qin] : (rs.F > 0);
        rs.chunks = pend;
        n->middle_count = 0;
        n->active_count = 0;
        n->popped = 0;
        // the previous round's deferred set ran at the start of this round; this
        // round's set either ran inside the round or is now pending
        n->heavy_count[cur ^ 1u] = 0;
        n->chunk_count[cur ^ 1u] = 0;
        if (!pend) {
            n->heavy_count[cur] = 0;
            n->chunk_count[cur] = 0;
        }
        pre_bookkeeping(a, ps, rs.F, sc[rs.qin]);
        publish(a, ps);
        ps.t_round_start = dev::globaltimer_ns();
    }

    static __device__ void load_snap(const Args &a, Snap &s) {
        if (threadIdx.x < 4) {
            const uint4 *src = reinterpret_cast<const uint4 *>(&a.ctrl->rs);
            reinterpret_cast<uint4 *>(&s)[threadIdx.x] = __ldcg(src + threadIdx.x);
        }
        __syncthreads();
    }

    static __device__ void set_app_variant(App &app, int v) {
        app.m_model = (common::Model)((v >> 2) & 1);
        app.m_msg_passing = (common::MsgPassing)((v >> 1) & 1);
        app.m_scheduling = (common::Scheduling)(v & 1);
    }
};

// The whole round loop of one query, run by the calling team (set_team).
// Returns false when a bounded wait gave up (the team must stop).
template <typename App, typename TV, typename TB, typename TW>
__device__ bool run_instance(const App &app_in, const KArgs<TV, TB, TW> &a) {
    using K = EngineKernel<App, TV, TB, TW>;
    __shared__ RoundState s;
    __shared__ WarpLB<TB> wlb[kWarpsPerBlock];
    __shared__ LocalQ lq_block;
    App app = app_in;
    Ctrl *c = a.ctrl;
    const unsigned long long tmo = a.p.timeout_ns;
    Acc acc;
    acc.reset();
    PolicyState ps;  // meaningful in block 0 / thread 0 only
    auto nop = [] {};

    // InitGraph (driver.cuh:68-92) and all frontier state cleared.
    for (uint32_t v = K::gthread(); v < a.csr.nnodes; v += K::nthreads()) {
        const TB b = app.App::GetInitBuffer(v);
        a.value[v] = app.App::GetInitValue(v);
        a.buffer[v] = b;
        a.tmp[v] = b;
    }
    for (uint32_t w = K::gthread(); w < a.nwords; w += K::nthreads()) {
        a.bitmap[0][w] = 0;
        a.bitmap[1][w] = 0;
        a.qflag[0][w] = 0;
        a.qflag[1][w] = 0;
        a.qflag[2][w] = 0;
    }
    if (a.tile_row) K::compute_tile_rows(a);
    if (!grid_sync(c, tmo, nop)) return false;
    K::rebuild(app, a, 0, acc);
    K::flush_acc(a, acc, 0, 2);
    if (!grid_sync(c, tmo, [&] { K::leader_start(a, ps); })) return false;

    WarpLB<TB> &my_lb = wlb[dev::warp_id()];
    const int lb_push = a.p.lb_push, lb_pull = a.p.lb_pull;
    for (;;) {
        K::load_snap(a, s);
        if (s.done) break;
        const int var = s.variant;
        const uint32_t set = s.round & 1u;  // heavy-vertex table this round registers into
        K::set_app_variant(app, var);
        app.m_concurrent_combine =
            var == V_ASYNC_PUSH_DD && a.p.local_depth > 0 && a.p.forced == V_ASYNC_PUSH_DD && reorder_safe(app);
        if (var == V_ASYNC_PUSH_DD && a.sort_counts && s.F > 1) {  // --wl_sort
            K::sort_count(a, s);
            if (!grid_sync(c, tmo, nop)) return false;
            K::sort_emit(a, s);
            if (!grid_sync(c, tmo, nop)) return false;
        }
        if (s.chunks) {
            // chunks of the heavy vertices the previous push round found (reorder-safe functors only)
            K::heavy_phase(app, a, s, set ^ 1u, true, acc);
            if (var != V_ASYNC_PUSH_DD) {  // not reached while chunks are deferred only under forced push DD
                K::flush_acc(a, acc, s.qhi, s.qlo);
                if (!grid_sync(c, tmo, nop)) return false;
            }
        }
        switch (var) {
            case V_ASYNC_PUSH_DD: {
                K::clear_dirty(a, s);
                LocalQ *lq = nullptr;
                if (a.p.local_depth > 0 && a.p.forced == V_ASYNC_PUSH_DD && reorder_safe(app)) {
                    if (threadIdx.x == 0) {
                        lq_block.out = 0;
                        lq_block.n[0] = lq_block.n[1] = 0;
                    }
                    __syncthreads();
                    lq = &lq_block;
                }
                K::push_phase_a(app, a, s, my_lb, true, lb_push, acc, lq);
                if (!K::defer_chunks(app, a) && s.heavy_expected > 0 && lb_push != LB_NONE) {
                    K::flush_acc(a, acc, s.qhi, s.qlo);
                    if (!grid_sync(c, tmo, nop)) return false;
                    K::heavy_phase(app, a, s, set, true, acc);
                }
                K::flush_acc(a, acc, s.qhi, s.qlo);
                break;
            }
            case V_ASYNC_PUSH_TD: {
                if (a.p.sample_cut > 0.f) {  // this round's threshold, from the team's first block
                    static_assert(sizeof(LocalQ::item) >= 1024 * sizeof(TB), "sample scratch");
                    if (g_team_rank == 0) K::sample_threshold(a, s, reinterpret_cast<TB *>(&lq_block.item[0][0]));
                    if (!grid_sync(c, tmo, nop)) return false;
                    if (threadIdx.x == 0) s.prio_raw = __ldcg(&a.ctrl->rs.prio_raw);
                    __syncthreads();
                }
                K::clear_dirty(a, s);
                K::release_input_flags(a, s, false);
                K::push_phase_a(app, a, s, my_lb, false, lb_push, acc);
                K::flush_acc(a, acc, s.qhi, s.qlo);
                if (!grid_sync(c, tmo, nop)) return false;
                if (lb_push != LB_NONE) {
                    K::heavy_phase(app, a, s, set, false, acc);
                    K::flush_acc(a, acc, s.qhi, s.qlo);
                    if (!grid_sync(c, tmo, nop)) return false;
                }
                K::rebuild(app, a, s.qhi, acc);
                K::flush_acc(a, acc, s.qhi, s.qlo);
                break;
            }
            case V_ASYNC_PULL_DD:
            case V_SYNC_PULL_DD:
            case V_SYNC_PULL_TD: {
                const bool dd = is_dd(var);
                const bool sync = is_sync(var);
                const bool convert = dd && !is_pull_dd(s.last_variant);
                constexpr bool reduce = has_pull_reduce<App, TB>::value && std::is_same<TW, graphs::NoWeight>::value;
                K::clear_dirty(a, s);
                K::release_input_flags(a, s, convert);
                const bool reduce_td = reduce && !dd && lb_pull != LB_NONE;  // scans every vertex, no middle list
                K::combine_all(app, a, sync, !reduce_td);
                if (!grid_sync(c, tmo, nop)) return false;
                if (reduce_td && a.tile_row) {
                    K::pull_tiles(app, a, my_lb, acc);
                } else if (reduce_td) {
                    K::pull_reduce_td(app, a, s, my_lb, acc);
                    K::flush_acc(a, acc, s.qhi, s.qlo);
                    if (!grid_sync(c, tmo, nop)) return false;
                    K::pull_reduce_chunks(app, a, set, acc);
                } else {
                    K::pull_phase(app, a, s, my_lb, dd, sync, lb_pull, acc);
                }
                K::flush_acc(a, acc, s.qhi, s.qlo);
                if (!dd) {
                    if (!grid_sync(c, tmo, nop)) return false;
                    K::rebuild(app, a, s.qhi, acc);
                    K::flush_acc(a, acc, s.qhi, s.qlo);
                }
                break;
            }
            default:
                break;  // unsupported variants never start a round (leader_start / leader_end_round)
        }
        if (!grid_sync(c, tmo, [&] { K::leader_end_round(app, a, ps); })) return false;
    }
    if (g_team_rank == 0 && threadIdx.x == 0) {
        c->edges_processed = dev::ld_l2(&c->cnt.edges_processed);
        c->error = dev::ld_l2(&c->cnt.error);
    }
    return true;
}

// One query: the whole cooperative grid is the team.
template <typename App, typename TV, typename TB, typename TW>
__global__ void __launch_bounds__(kBlockThreads) hybrid_engine_kernel(const App app_in, KArgs<TV, TB, TW> a) {
    set_team(blockIdx.x, gridDim.x, a.ctrl);
    run_instance<App, TV, TB, TW>(app_in, a);
}

// ---------------------------------------------------------------- batched queries
// One query of a batch: its functor (source etc.), graph views and output.
template <typename App, typename TV>
struct BatchQuery {
    App app;
    graphs::dev::CSRGraph csr;
    graphs::dev::CSCGraph csc;
    const uint32_t *csr_w, *csc_w;
    TV *value;
    unsigned long long prio_raw;  // this query's two-level priority step (0 = the batch's)
};

// Per-team workspace of a batched launch, sized for the largest graph of the
// batch; every query a team runs reuses it.
template <typename TB>
struct TeamSpace {
    TB *buffer, *tmp;
    uint32_t *queue[3], *bitmap[2], *qflag[3], *middle, *chunk_owner;
    HeavyItem<TB> *heavy;
    Ctrl *ctrl;
    sg_round_trace *trace;
    uint32_t cap_v, heavy_cap, chunk_cap, trace_cap;
};

// Per-query result record written when the query finishes.
struct BatchResult {
    uint32_t rounds, error, max_iteration_reached, team;
    uint32_t rounds_by_variant[8];
    unsigned long long edges_processed, t_start, t_end;
    unsigned long long reached;  // edges of the reached component, where the kernel counts it
};

// Leader-side record of a finished query (every field but `reached`).
__device__ __forceinline__ void write_result(BatchResult *r, const Ctrl *c, uint32_t team, uint32_t extra_err,
                                             unsigned long long t_end) {
    r->rounds = c->round;
    r->error = dev::ld_l2(&c->cnt.error) | extra_err;
    r->max_iteration_reached = c->max_iteration_reached;
    r->team = team;
    for (int k = 0; k < 8; ++k) r->rounds_by_variant[k] = c->rounds_by_variant[k];
    r->edges_processed = dev::ld_l2(&c->cnt.edges_processed);
    r->t_start = c->t_start;
    r->t_end = t_end;
}

// Batched engine: the cooperative grid is split into teams of team_blocks
// blocks; each team takes the next query from a device counter (queries are
// ordered largest first by the host), runs its whole round loop with a
// team-local barrier, records its result and moves on.  Per-query frontiers
// and state never leave the device; the batch is one launch (capturable in a
// CUDA graph).
template <typename App, typename TV, typename TB, typename TW>
__global__ void __launch_bounds__(kBlockThreads)
    batched_engine_kernel(const BatchQuery<App, TV> *queries, uint32_t nq, const TeamSpace<TB> *spaces,
                          uint32_t team_blocks, uint32_t *next_query, BatchResult *results, Params p) {
    const uint32_t team = blockIdx.x / team_blocks;
    const TeamSpace<TB> &sp = spaces[team];
    Ctrl *c = sp.ctrl;
    set_team(blockIdx.x % team_blocks, team_blocks, c);
    __shared__ uint32_t s_q;
    for (;;) {
        // the team leader claims the next query; zero its control state (barrier words excluded)
        auto claim = [&] {
            const uint32_t q = atomicAdd(next_query, 1u);
            unsigned char *z = reinterpret_cast<unsigned char *>(&c->rs);
            memset(z, 0, sizeof(Ctrl) - offsetof(Ctrl, rs));
            c->pad0 = q;
        };
        if (!grid_sync(c, p.timeout_ns, claim)) return;
        if (threadIdx.x == 0) s_q = dev::ld_l2(&c->pad0);
        __syncthreads();
        const uint32_t q = s_q;
        if (q >= nq) return;
        const BatchQuery<App, TV> &bq = queries[q];
        KArgs<TV, TB, TW> a;
        a.csr = bq.csr;
        a.csc = bq.csc;
        a.csr_w = bq.csr_w;
        a.csc_w = bq.csc_w;
        a.value = bq.value;
        a.buffer = sp.buffer;
        a.tmp = sp.tmp;
        for (int k = 0; k < 3; ++k) {
            a.queue[k] = sp.queue[k];
            a.qflag[k] = sp.qflag[k];
        }
        a.bitmap[0] = sp.bitmap[0];
        a.bitmap[1] = sp.bitmap[1];
        a.queue_cap = bq.csr.nnodes;
        a.nwords = bq.csr.nnodes / 32 + 1;
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
        if (bq.prio_raw) a.p.prio_init_raw = a.p.prio_step_raw = bq.prio_raw;
        App app = bq.app;
        app.m_p_current_round = &c->rs.round;
        if (!run_instance<App, TV, TB, TW>(app, a)) return;
        if (g_team_rank == 0 && threadIdx.x == 0) write_result(results + q, c, team, 0u, c->t_end);
    }
}

}  // namespace engine
}  // namespace sepgraph
