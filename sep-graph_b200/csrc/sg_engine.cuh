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
// Frontier bookkeeping lives on the device: every append to the next worklist
// also accumulates the appended vertex's out-degree (the "scout count" that
// SumOutDegreeQueue computes with a separate kernel and a D2H copy,
// driver.cuh:225-248), so the policy needs no extra pass.  The last block to
// reach each grid barrier evaluates the policy, rotates worklists and records
// the trace.  A per-vertex "queued" bitmap keeps each worklist free of
// duplicates, which bounds every worklist by |V| (the reference sizes them at
// 0.2*|E| and can overflow silently, graph_datum.cuh:90).
#pragma once
#include <cstdint>
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

enum : int32_t { LB_NONE = 0, LB_COARSE = 1, LB_FINE = 2, LB_HYBRID = 3 };

template <typename TBuffer>
struct HeavyItem {
    uint32_t src, beg, deg, chunk_base;
    TBuffer payload;
};

// Engine control block (device memory).  Field roles mirror RunningInfo
// (hybrid_policy.h:36-120) plus the worklist slot assignment.
struct Ctrl {
    uint32_t bar_count, bar_gen, error, done;
    uint32_t round, max_iteration_reached;
    int32_t variant, last_variant;
    uint32_t qin, qhi, qlo, bin, bout, dirty, pile, in_flag;
    uint32_t qcount[3];
    uint32_t heavy_enq[3];
    unsigned long long scout[3];
    uint32_t middle_count, heavy_count, chunk_count, inspect_next;
    long long total_workload;
    uint32_t input_active, output_active;
    unsigned long long input_workload, output_workload;
    unsigned long long prio_raw;
    float policy_time[8];
    uint32_t policy_seen;
    float time_per_work;
    unsigned long long t_round_start, t_start, t_end;
    uint32_t rounds_by_variant[8];
    unsigned long long edges_processed, vertices_processed;
    uint32_t n_trace;
    uint32_t pad;
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
    double alpha, beta;
    long long total_workload0;
    unsigned long long prio_init_raw, prio_step_raw;
    unsigned long long timeout_ns;
};

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
    uint32_t *qflag[2];
    uint32_t nwords;
    uint32_t *middle;
    HeavyItem<TBuffer> *heavy;
    uint32_t heavy_cap;
    uint32_t *chunk_owner;
    uint32_t chunk_cap;
    Ctrl *ctrl;
    sg_round_trace *trace;
    uint32_t trace_cap;
    Params p;
};

// Round snapshot broadcast through shared memory after every barrier.
struct Snap {
    int32_t variant, last_variant;
    uint32_t round, qin, qhi, qlo, bin, bout, dirty, pile, in_flag, F, heavy_expected, done;
    unsigned long long prio_raw;
};

template <typename TBuffer>
struct WarpLB {
    uint32_t excl[32];
    uint32_t beg[32];
    uint32_t src[32];
    TBuffer pay[32];
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

template <typename App, typename TV, typename TB, typename TW>
struct EngineKernel {
    using Args = KArgs<TV, TB, TW>;

    static __device__ __forceinline__ uint32_t gthread() { return blockIdx.x * blockDim.x + threadIdx.x; }
    static __device__ __forceinline__ uint32_t nthreads() { return gridDim.x * blockDim.x; }
    static __device__ __forceinline__ uint32_t gwarp() { return gthread() >> 5; }
    static __device__ __forceinline__ uint32_t nwarps() { return nthreads() >> 5; }

    static __device__ __forceinline__ uint32_t out_degree(const Args &a, uint32_t v) {
        return a.csr.end_edge(v) - a.csr.begin_edge(v);
    }

    static __device__ void flush_acc(const Args &a, Acc &acc, uint32_t q_hi, uint32_t q_lo) {
        unsigned long long s0 = dev::warp_sum(acc.scout_hi), s1 = dev::warp_sum(acc.scout_lo);
        uint32_t h0 = dev::warp_sum(acc.heavy_hi), h1 = dev::warp_sum(acc.heavy_lo);
        unsigned long long ed = dev::warp_sum(acc.edges);
        if (dev::lane_id() == 0) {
            if (s0) atomicAdd(&a.ctrl->scout[q_hi], s0);
            if (h0) atomicAdd(&a.ctrl->heavy_enq[q_hi], h0);
            if (s1) atomicAdd(&a.ctrl->scout[q_lo], s1);
            if (h1) atomicAdd(&a.ctrl->heavy_enq[q_lo], h1);
            if (ed) atomicAdd(&a.ctrl->edges_processed, ed);
        }
        acc.reset();
    }

    // Append dst to the next worklist(s) if `want`: dedupe through the queued
    // bitmap, route by IsHighPriority when two-level priority is on, and count
    // its out-degree for the policy.  All 32 lanes must call.
    static __device__ __forceinline__ void enqueue(App &app, const Args &a, const Snap &s, uint32_t dst, bool want,
                                                   Acc &acc) {
        bool hi = true;
        if (a.p.priority && want) hi = app.App::IsHighPriority(from_raw<TB>(s.prio_raw), dev::ld_l2(a.buffer + dst));
        bool w_hi = want && hi, w_lo = want && !hi;
        if (want) __threadfence();  // order the buffer update before publishing the queued bit
        if (w_hi) w_hi = dev::bitmap_set(a.qflag[0], dst);
        if (w_lo) w_lo = dev::bitmap_set(a.qflag[1], dst);
        dev::warp_append(a.queue[s.qhi], &a.ctrl->qcount[s.qhi], a.queue_cap, w_hi, dst, &a.ctrl->error);
        if (a.p.priority) dev::warp_append(a.queue[s.qlo], &a.ctrl->qcount[s.qlo], a.queue_cap, w_lo, dst,
                                           &a.ctrl->error);
        if (w_hi || w_lo) acc.count(w_hi, out_degree(a, dst), a.p.heavy_threshold);
    }

    // Single-thread enqueue (LB NONE paths run divergent per-thread loops).
    static __device__ __forceinline__ void enqueue_one(App &app, const Args &a, const Snap &s, uint32_t dst,
                                                       Acc &acc) {
        bool hi = true;
        if (a.p.priority) hi = app.App::IsHighPriority(from_raw<TB>(s.prio_raw), dev::ld_l2(a.buffer + dst));
        __threadfence();
        const int k = hi ? 0 : 1;
        if (!dev::bitmap_set(a.qflag[k], dst)) return;
        const uint32_t q = hi ? s.qhi : s.qlo;
        const uint32_t pos = atomicAdd(&a.ctrl->qcount[q], 1u);
        if (pos < a.queue_cap)
            a.queue[q][pos] = dst;
        else
            atomicOr(&a.ctrl->error, dev::kErrCapacity);
        acc.count(hi, out_degree(a, dst), a.p.heavy_threshold);
    }

    static __device__ __forceinline__ void register_heavy(const Args &a, uint32_t src, uint32_t beg, uint32_t deg,
                                                          TB payload) {
        const uint32_t ce = a.p.chunk_edges;
        const uint32_t nch = (deg + ce - 1) / ce;
        const uint32_t idx = atomicAdd(&a.ctrl->heavy_count, 1u);
        const uint32_t cb = atomicAdd(&a.ctrl->chunk_count, nch);
        if (idx < a.heavy_cap && cb <= a.chunk_cap && nch <= a.chunk_cap - cb) {
            HeavyItem<TB> h;
            h.src = src;
            h.beg = beg;
            h.deg = deg;
            h.chunk_base = cb;
            h.payload = payload;
            a.heavy[idx] = h;
            for (uint32_t i = 0; i < nch; ++i) a.chunk_owner[cb + i] = idx;
        } else {
            atomicOr(&a.ctrl->error, dev::kErrChunkCapacity);
        }
    }

    // Warp-cooperative expansion of up to 32 (src, beg, deg, payload) items:
    // the warp walks the concatenation of their edge lists 32 edges at a time,
    // each lane locating its source by binary search over the warp's exclusive
    // degree scan (shared memory).  All 32 lanes must call.
    static __device__ void expand_warp(App &app, const Args &a, const Snap &s, WarpLB<TB> &w, uint32_t src,
                                       uint32_t beg, uint32_t deg, TB payload, bool dd, Acc &acc) {
        const uint32_t lane = dev::lane_id();
        const uint32_t incl = dev::warp_inclusive_scan(deg);
        const uint32_t total = __shfl_sync(dev::kFullMask, incl, 31);
        if (total == 0) return;
        w.excl[lane] = incl - deg;
        w.beg[lane] = beg;
        w.src[lane] = src;
        w.pay[lane] = payload;
        __syncwarp();
        for (uint32_t eb = 0; eb < total; eb += 32) {
            const uint32_t e = eb + lane;
            bool want = false;
            uint32_t dst = 0;
            if (e < total) {
                uint32_t k = 0;
#pragma unroll
                for (uint32_t step = 16; step > 0; step >>= 1)
                    if (w.excl[k + step] <= e) k += step;
                const uint32_t edge = w.beg[k] + (e - w.excl[k]);
                dst = a.csr.edge_dest(edge);
                const int st = accumulate<App, TB, TW>(app, a.csr_w, w.src[k], dst, edge, a.buffer + dst, w.pay[k]);
                want = dd && acc_success(st);
            }
            enqueue(app, a, s, dst, want, acc);
        }
        if (lane == 0) acc.edges += total;
        __syncwarp();
    }

    // Thread-per-vertex sequential expansion honouring BREAK (LB NONE,
    // async_push_dd.cuh:24-77).
    static __device__ void expand_serial(App &app, const Args &a, const Snap &s, uint32_t src, uint32_t beg,
                                         uint32_t deg, TB payload, bool dd, Acc &acc) {
        uint32_t e = beg;
        for (; e < beg + deg; ++e) {
            const uint32_t dst = a.csr.edge_dest(e);
            const int st = accumulate<App, TB, TW>(app, a.csr_w, src, dst, e, a.buffer + dst, payload);
            if (dd && acc_success(st)) enqueue_one(app, a, s, dst, acc);
            if (!acc_continue(st)) {
                ++e;
                break;
            }
        }
        acc.edges += e - beg;
    }

    // Chunks of heavy vertices registered in phase A, spread over all warps.
    static __device__ void heavy_phase(App &app, const Args &a, const Snap &s, bool dd, Acc &acc) {
        const uint32_t C = min(dev::ld_l2(&a.ctrl->chunk_count), a.chunk_cap);
        const uint32_t H = min(dev::ld_l2(&a.ctrl->heavy_count), a.heavy_cap);
        const uint32_t lane = dev::lane_id();
        const uint32_t ce = a.p.chunk_edges;
        for (uint32_t ch = gwarp(); ch < C; ch += nwarps()) {
            const uint32_t e = dev::ld_l2(a.chunk_owner + ch);
            if (e >= H) continue;
            const HeavyItem<TB> h = a.heavy[e];
            if (ch < h.chunk_base) continue;
            const uint32_t off = (ch - h.chunk_base) * ce;
            if (off >= h.deg) continue;
            const uint32_t len = min(ce, h.deg - off);
            for (uint32_t k = 0; k < len; k += 32) {
                const uint32_t i = k + lane;
                bool want = false;
                uint32_t dst = 0;
                if (i < len) {
                    const uint32_t edge = h.beg + off + i;
                    dst = a.csr.edge_dest(edge);
                    const int st = accumulate<App, TB, TW>(app, a.csr_w, h.src, dst, edge, a.buffer + dst, h.payload);
                    want = dd && acc_success(st);
                }
                enqueue(app, a, s, dst, want, acc);
            }
            if (lane == 0) acc.edges += len;
        }
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
            dev::bitmap_clear(a.qflag[0], v);
            if (to_bitmap) dev::bitmap_set(a.bitmap[s.bin], v);  // Queue2Bitmap (driver.cuh:119-129)
        }
    }

    // ---------------------------------------------------------------- push
    // Phase A of a push round over worklist items (DD) or all vertices (TD).
    static __device__ void push_phase_a(App &app, const Args &a, const Snap &s, WarpLB<TB> &wlb, bool dd,
                                        int lb, Acc &acc) {
        const uint32_t lane = dev::lane_id();
        const uint32_t N = dd ? s.F : a.csr.nnodes;
        const uint32_t *Q = a.queue[s.qin];
        const TB prio = from_raw<TB>(s.prio_raw);
        for (uint32_t base = gwarp() * 32; base < N; base += nwarps() * 32) {
            const uint32_t i = base + lane;
            const bool valid = i < N;
            uint32_t v = 0;
            bool proceed = valid;
            bool keep = false;
            if (valid) {
                v = dd ? dev::ld_l2(Q + i) : i;
                if (dd) {
                    if (s.pile) {
                        // far pile: vertices still below the priority window stay in the pile
                        if (!app.App::IsHighPriority(prio, dev::ld_l2(a.buffer + v))) {
                            keep = true;
                            proceed = false;
                        } else {
                            dev::bitmap_clear(a.qflag[1], v);
                        }
                    } else {
                        dev::bitmap_clear(a.qflag[0], v);
                    }
                }
            }
            if (dd) {
                __threadfence();  // pop (queued bit cleared) before reading the vertex state
                if (s.pile) dev::warp_append(a.queue[s.qlo], &a.ctrl->qcount[s.qlo], a.queue_cap, keep, v,
                                             &a.ctrl->error);
                if (keep) acc.count(false, out_degree(a, v), a.p.heavy_threshold);
            }
            TB payload{};
            bool sched = false;
            if (proceed) {
                auto pr = app.App::CombineValueBuffer(v, a.value + v, a.buffer + v);
                payload = pr.first;
                sched = pr.second;
            }
            uint32_t beg = 0, deg = 0;
            if (sched) {
                beg = a.csr.begin_edge(v);
                deg = a.csr.end_edge(v) - beg;
            }
            if (lb == LB_NONE) {
                if (deg) expand_serial(app, a, s, v, beg, deg, payload, dd, acc);
                continue;
            }
            if (deg > a.p.heavy_threshold) {
                register_heavy(a, v, beg, deg, payload);
                deg = 0;
            }
            expand_warp(app, a, s, wlb, v, beg, deg, payload, dd, acc);
        }
    }

    // ---------------------------------------------------------------- pull
    // CombineValueBuffer over every vertex; scheduled vertices form the middle
    // list (variants/common.cuh:17-84).  `sync` writes the combined buffer to
    // tmp (SYNC_PULL_*), else back into buffer (ASYNC_PULL_DD, algo_variants.cuh:842-849).
    static __device__ void combine_all(App &app, const Args &a, bool sync) {
        const uint32_t lane = dev::lane_id();
        const uint32_t N = a.csr.nnodes;
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
            dev::warp_append(a.middle, &a.ctrl->middle_count, a.csr.nnodes, want, v, &a.ctrl->error);
        }
    }

    // Pull into one destination, sequentially over its in-edges (early exit on BREAK).
    static __device__ bool pull_serial(App &app, const Args &a, const Snap &s, uint32_t v, uint32_t beg,
                                       uint32_t deg, bool dd, bool sync, Acc &acc) {
        const TB *srcbuf = sync ? a.tmp : a.buffer;
        const uint32_t *bin = a.bitmap[s.bin];
        bool hit = false;
        if constexpr (has_pull_reduce<App, TB>::value && std::is_same<TW, graphs::NoWeight>::value) {
            if (!dd) {
                TB r = app.PullIdentity();
                for (uint32_t e = beg; e < beg + deg; ++e) r = app.PullReduce(r, dev::ld_l2(srcbuf + a.csc.edge_src(e)));
                acc.edges += deg;
                if (deg) hit = acc_success(accumulate<App, TB, TW>(app, a.csc_w, v, v, beg, a.buffer + v, r));
                return hit;
            }
        }
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

    // The whole warp pulls into one high in-degree destination, 32 in-edges per step.
    static __device__ bool pull_warp(App &app, const Args &a, const Snap &s, uint32_t v, uint32_t beg, uint32_t deg,
                                     bool dd, bool sync, Acc &acc) {
        const uint32_t lane = dev::lane_id();
        const TB *srcbuf = sync ? a.tmp : a.buffer;
        const uint32_t *bin = a.bitmap[s.bin];
        if constexpr (has_pull_reduce<App, TB>::value && std::is_same<TW, graphs::NoWeight>::value) {
            if (!dd) {
                TB r = app.PullIdentity();
                for (uint32_t k = lane; k < deg; k += 32) r = app.PullReduce(r, dev::ld_l2(srcbuf + a.csc.edge_src(beg + k)));
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) r = app.PullReduce(r, __shfl_xor_sync(dev::kFullMask, r, d));
                bool hit = false;
                if (lane == 0) {
                    hit = acc_success(accumulate<App, TB, TW>(app, a.csc_w, v, v, beg, a.buffer + v, r));
                    acc.edges += deg;
                }
                return __shfl_sync(dev::kFullMask, hit, 0);
            }
        }
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

    static __device__ void pull_phase(App &app, const Args &a, const Snap &s, bool dd, bool sync, int lb,
                                      Acc &acc) {
        const uint32_t lane = dev::lane_id();
        const uint32_t M = min(dev::ld_l2(&a.ctrl->middle_count), a.csr.nnodes);
        const bool natural = (M == a.csr.nnodes);  // every vertex scheduled: keep CSC order
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
            if (valid && !big) hit = pull_serial(app, a, s, v, beg, deg, dd, sync, acc);
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
                    __threadfence();
                    dev::bitmap_set(a.bitmap[s.bout], v);
                    want = dev::bitmap_set(a.qflag[0], v);
                }
                dev::warp_append(a.queue[s.qhi], &a.ctrl->qcount[s.qhi], a.queue_cap, want, v, &a.ctrl->error);
                if (want) acc.count(true, out_degree(a, v), a.p.heavy_threshold);
            }
        }
    }

    // RebuildWorklist (driver.cuh:162-178): active vertices -> worklist `slot`.
    static __device__ void rebuild(App &app, const Args &a, uint32_t slot, Acc &acc) {
        const uint32_t lane = dev::lane_id();
        const uint32_t N = a.csr.nnodes;
        for (uint32_t base = gwarp() * 32; base < N; base += nwarps() * 32) {
            const uint32_t v = base + lane;
            bool act = false;
            if (v < N) act = app.App::IsActiveNode(v, dev::ld_l2(a.buffer + v));
            if (act) act = dev::bitmap_set(a.qflag[0], v);
            dev::warp_append(a.queue[slot], &a.ctrl->qcount[slot], a.queue_cap, act, v, &a.ctrl->error);
            if (act) acc.count(true, out_degree(a, v), a.p.heavy_threshold);
        }
    }

    // ---------------------------------------------------------------- leader work
    static __device__ void pre_bookkeeping(const Args &a, Ctrl *c, int var) {
        if (!a.p.collect) return;
        if (is_dd(var)) {
            c->input_active = c->qcount[c->qin];
            c->input_workload = is_pull(var) ? 0ull : c->scout[c->qin];
            c->total_workload -= (long long)c->input_workload;
            if (c->total_workload < 0) c->total_workload = 0;
        } else {
            c->input_workload = a.csr.nedges;
            c->input_active = a.csr.nnodes;
        }
    }

    static __device__ void reset_slot(Ctrl *c, uint32_t q) {
        c->qcount[q] = 0;
        c->scout[q] = 0;
        c->heavy_enq[q] = 0;
    }

    static __device__ bool supported(const Args &a, int v) {
        if (v == V_SYNC_PUSH_TD || v == V_SYNC_PUSH_DD || v == V_ASYNC_PULL_TD) return false;
        if (is_pull(v) && !a.p.has_csc) return false;
        return true;
    }

    static __device__ void leader_start(App &app, const Args &a) {
        Ctrl *c = a.ctrl;
        c->round = 1;
        c->last_variant = -1;
        int v = a.p.forced >= 0 ? a.p.forced : (a.p.scheme == 0 ? V_ASYNC_PUSH_DD : V_SYNC_PULL_TD);
        c->inspect_next = 1;
        c->variant = v;
        c->qin = 0;
        c->qhi = 1;
        c->qlo = 2;
        c->bin = 0;
        c->bout = 1;
        c->dirty = 0;
        c->pile = 0;
        c->in_flag = 0;
        c->total_workload = a.p.total_workload0;
        c->prio_raw = a.p.prio_init_raw;
        pre_bookkeeping(a, c, v);
        if (!supported(a, v)) {
            c->error |= dev::kErrUnsupported;
            c->done = 1;
        }
        c->t_start = c->t_round_start = dev::globaltimer_ns();
    }

    static __device__ int traversal_policy(const Args &a, const Ctrl *c, int var) {
        // GetNextPolicy, TRAVERSAL_SCHEME (hybrid_policy.h:265-288)
        if (is_pull(var) && (double)c->output_active > (double)a.csr.nnodes / a.p.beta) return V_ASYNC_PULL_DD;
        if ((double)c->output_workload > (double)c->total_workload / a.p.alpha) return V_ASYNC_PULL_DD;
        return V_ASYNC_PUSH_DD;
    }

    static __device__ int iterative_policy(const Args &a, Ctrl *c, int var) {
        // Inspect SYNC_PULL_TD, ASYNC_PUSH_TD, ASYNC_PUSH_DD once each (std::set order,
        // hybrid_policy.h:180-195), then pick the smallest predicted time (130-169, 242-263).
        const int order[3] = {V_SYNC_PULL_TD, V_ASYNC_PUSH_TD, V_ASYNC_PUSH_DD};
        if (c->inspect_next < 3) return order[c->inspect_next++];
        if (is_dd(var) && c->input_workload > 0) c->time_per_work = c->policy_time[var] / (float)c->input_workload;
        int best = -1;
        float bt = 0.f;
        for (int k = 0; k < 3; ++k) {
            const int v = order[k];
            if (!(c->policy_seen & (1u << v))) continue;
            const float t = is_dd(v) ? c->time_per_work * (float)c->output_workload : c->policy_time[v];
            if (best < 0 || t < bt) {
                best = v;
                bt = t;
            }
        }
        return best < 0 ? var : best;
    }

    static __device__ void leader_end_round(App &app, const Args &a) {
        Ctrl *c = a.ctrl;
        const int var = c->variant;
        app.App::PostComputation();
        c->rounds_by_variant[var & 7]++;
        const unsigned long long now = dev::globaltimer_ns();
        const float round_ms = (float)(now - c->t_round_start) * 1e-6f;
        c->vertices_processed += is_dd(var) ? c->qcount[c->qin] : a.csr.nnodes;
        const bool prio_push = a.p.priority && var == V_ASYNC_PUSH_DD;
        const uint32_t out_hi = c->qcount[c->qhi];
        const uint32_t out_lo = prio_push ? c->qcount[c->qlo] : 0;
        c->output_active = out_hi + out_lo;
        if (a.p.collect) {
            if (!is_dd(var) || !is_pull(var))
                c->output_workload = c->scout[c->qhi] + (prio_push ? c->scout[c->qlo] : 0ull);
            else
                c->output_workload = 1;  // framework.cuh:790
        }
        c->policy_time[var & 7] = round_ms;
        c->policy_seen |= 1u << (var & 7);
        if (a.p.trace && a.trace && c->n_trace < a.trace_cap) {
            sg_round_trace t;
            t.round = c->round;
            t.variant = var;
            t.in_nodes = c->input_active;
            t.out_nodes = c->output_active;
            t.in_workload = c->input_workload;
            t.out_workload = c->output_workload;
            t.total_workload = c->total_workload;
            t.time_ms = round_ms;
            t.pad = 0;
            a.trace[c->n_trace] = t;
            c->n_trace++;
        }
        int next = var;
        if (a.p.forced < 0) next = a.p.scheme == 0 ? traversal_policy(a, c, var) : iterative_policy(a, c, var);
        const bool fatal = (c->error & (dev::kErrTimeout | dev::kErrCapacity | dev::kErrChunkCapacity |
                                        dev::kErrUnsupported | dev::kErrOverflow)) != 0;
        if (c->output_active == 0 || c->round >= a.p.max_iteration || fatal) {
            c->max_iteration_reached = c->output_active != 0 && c->round >= a.p.max_iteration;
            c->done = 1;
            c->t_end = now;
            return;
        }
        // rotate worklists
        if (prio_push && out_hi == 0) {
            // near pile drained: open the next priority window over the far pile (driver.cuh:668-675)
            c->prio_raw = to_raw<TB>((TB)(from_raw<TB>(c->prio_raw) + from_raw<TB>(a.p.prio_step_raw)));
            const uint32_t t = c->qin;
            c->qin = c->qlo;
            c->qlo = t;
            reset_slot(c, c->qlo);
            c->pile = 1;
            c->in_flag = 1;
        } else {
            const uint32_t t = c->qin;
            c->qin = c->qhi;
            c->qhi = t;
            reset_slot(c, c->qhi);
            c->pile = 0;
            c->in_flag = 0;
        }
        if (is_dd(var) && is_pull(var)) {
            const uint32_t t = c->bin;
            c->bin = c->bout;
            c->bout = t;
            c->dirty = (is_dd(next) && is_pull(next)) ? (1u << c->bout) : 3u;
        } else {
            c->dirty = 0;
        }
        if (!supported(a, next)) {
            c->error |= dev::kErrUnsupported;
            c->done = 1;
            c->t_end = now;
            return;
        }
        c->last_variant = var;
        c->variant = next;
        c->round++;
        c->middle_count = 0;
        c->heavy_count = 0;
        c->chunk_count = 0;
        pre_bookkeeping(a, c, next);
        c->t_round_start = dev::globaltimer_ns();
    }

    static __device__ void load_snap(const Args &a, Snap &s) {
        if (threadIdx.x == 0) {
            const Ctrl *c = a.ctrl;
            s.variant = dev::ld_l2(&c->variant);
            s.last_variant = dev::ld_l2(&c->last_variant);
            s.round = dev::ld_l2(&c->round);
            s.qin = dev::ld_l2(&c->qin);
            s.qhi = dev::ld_l2(&c->qhi);
            s.qlo = dev::ld_l2(&c->qlo);
            s.bin = dev::ld_l2(&c->bin);
            s.bout = dev::ld_l2(&c->bout);
            s.dirty = dev::ld_l2(&c->dirty);
            s.pile = dev::ld_l2(&c->pile);
            s.in_flag = dev::ld_l2(&c->in_flag);
            s.F = min(dev::ld_l2(&c->qcount[s.qin]), a.queue_cap);
            s.heavy_expected = dev::ld_l2(&c->heavy_enq[s.qin]);
            s.done = dev::ld_l2(&c->done);
            s.prio_raw = dev::ld_l2(&c->prio_raw);
        }
        __syncthreads();
    }

    static __device__ void set_app_variant(App &app, int v) {
        app.m_model = (common::Model)((v >> 2) & 1);
        app.m_msg_passing = (common::MsgPassing)((v >> 1) & 1);
        app.m_scheduling = (common::Scheduling)(v & 1);
    }
};

template <typename App, typename TV, typename TB, typename TW>
__global__ void __launch_bounds__(kBlockThreads) hybrid_engine_kernel(const App app_in, KArgs<TV, TB, TW> a) {
    using K = EngineKernel<App, TV, TB, TW>;
    __shared__ Snap s;
    __shared__ WarpLB<TB> wlb[kWarpsPerBlock];
    App app = app_in;
    Ctrl *c = a.ctrl;
    const uint64_t tmo = a.p.timeout_ns;
    Acc acc;
    acc.reset();
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
    }
    if (!dev::grid_barrier(&c->bar_count, &c->bar_gen, &c->error, tmo, nop)) return;
    K::rebuild(app, a, 0, acc);
    K::flush_acc(a, acc, 0, 2);
    if (!dev::grid_barrier(&c->bar_count, &c->bar_gen, &c->error, tmo, [&] { K::leader_start(app, a); })) return;

    WarpLB<TB> &my_lb = wlb[dev::warp_id()];
    for (;;) {
        K::load_snap(a, s);
        if (s.done) break;
        const int var = s.variant;
        K::set_app_variant(app, var);
        const int lb_push = a.p.lb_push, lb_pull = a.p.lb_pull;
        switch (var) {
            case V_ASYNC_PUSH_DD: {
                K::clear_dirty(a, s);
                K::push_phase_a(app, a, s, my_lb, true, lb_push, acc);
                if (s.heavy_expected > 0 && lb_push != LB_NONE) {
                    K::flush_acc(a, acc, s.qhi, s.qlo);
                    if (!dev::grid_barrier(&c->bar_count, &c->bar_gen, &c->error, tmo, nop)) return;
                    K::heavy_phase(app, a, s, true, acc);
                }
                K::flush_acc(a, acc, s.qhi, s.qlo);
                break;
            }
            case V_ASYNC_PUSH_TD: {
                K::clear_dirty(a, s);
                K::release_input_flags(a, s, false);
                K::push_phase_a(app, a, s, my_lb, false, lb_push, acc);
                K::flush_acc(a, acc, s.qhi, s.qlo);
                if (!dev::grid_barrier(&c->bar_count, &c->bar_gen, &c->error, tmo, nop)) return;
                if (lb_push != LB_NONE) {
                    K::heavy_phase(app, a, s, false, acc);
                    K::flush_acc(a, acc, s.qhi, s.qlo);
                    if (!dev::grid_barrier(&c->bar_count, &c->bar_gen, &c->error, tmo, nop)) return;
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
                const bool convert = dd && !(s.last_variant >= 0 && is_dd(s.last_variant) && is_pull(s.last_variant));
                K::clear_dirty(a, s);
                K::release_input_flags(a, s, convert);
                K::combine_all(app, a, sync);
                if (!dev::grid_barrier(&c->bar_count, &c->bar_gen, &c->error, tmo, nop)) return;
                K::pull_phase(app, a, s, dd, sync, lb_pull, acc);
                K::flush_acc(a, acc, s.qhi, s.qlo);
                if (!dd) {
                    if (!dev::grid_barrier(&c->bar_count, &c->bar_gen, &c->error, tmo, nop)) return;
                    K::rebuild(app, a, s.qhi, acc);
                    K::flush_acc(a, acc, s.qhi, s.qlo);
                }
                break;
            }
            default:
                break;  // unsupported variants never start a round (leader_start / leader_end_round)
        }
        if (!dev::grid_barrier(&c->bar_count, &c->bar_gen, &c->error, tmo, [&] { K::leader_end_round(app, a); }))
            return;
    }
}

}  // namespace engine
}  // namespace sepgraph
