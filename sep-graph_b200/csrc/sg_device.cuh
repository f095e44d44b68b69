// Device primitives of the B200 hybrid engine: a bounded grid barrier whose
// last arriving block runs a single-thread callback, warp-aggregated worklist
// appends, bitmap frontier helpers and small warp collectives.
//
// Reference counterparts: cub::GridBarrier (unbounded spin, used by the fused
// kernels in include/framework/variants/driver.cuh:533-685), dev::Queue::append
// (one atomicAdd per item, include/groute/device/queue.cuh:84-88; its
// warp-aggregated append_warp at 90-116 is unused), and CompressedBitmap
// (64-bit words, CAS set_bit_atomic, include/groute/device/compressed_bitmap.cuh:35-48).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sepgraph {
namespace dev {

constexpr uint32_t kFullMask = 0xffffffffu;

// Device error bits (reported through sg_stats.device_error and mapped to sg_status).
enum : uint32_t {
    kErrTimeout = 1u,        // a bounded wait gave up
    kErrCapacity = 2u,       // a worklist reservation exceeded its capacity (nothing written past it)
    kErrOverflow = 4u,       // uint64 path-count overflow (BC)
    kErrUnsupported = 8u,    // variant not implemented (same set as the reference's assert(false))
    kErrChunkCapacity = 16u  // heavy-vertex chunk table overflow
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t warp_id() { return threadIdx.x >> 5; }
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t *p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(uint32_t *p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Barrier arrival: a release fence (this block's prior writes, ordered by the
// preceding __syncthreads, become visible first) and a fire-and-forget add
// whose result the arriving thread does not wait for.
__device__ __forceinline__ void arrive_release(uint32_t *p) {
    asm volatile("fence.acq_rel.gpu;\n\tred.relaxed.gpu.global.add.u32 [%0], 1;" ::"l"(p) : "memory");
}
// Loads of state that other blocks modify inside the same launch go through L2.
template <typename T>
__device__ __forceinline__ T ld_l2(const T *p) {
    return __ldcg(p);
}

// 16-byte read-only load (ld.global.nc.v4); p must be 16-byte aligned.
__device__ __forceinline__ uint4 ldg_v4(const uint32_t *p) { return __ldg(reinterpret_cast<const uint4 *>(p)); }

// Streamed graph arrays (edge destinations, weights, in-edge sources) are read
// with an L2 evict-first cache policy: a traversal streams hundreds of MB of
// them through L2 once, and without the hint they push out the vertex state
// (tentative values, frontier bitmaps, pulled values) that every round reads
// at random.
__device__ __forceinline__ uint64_t stream_policy() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ uint32_t ldg_stream(const uint32_t *p, uint64_t pol) {
    uint32_t r;
    asm("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(r) : "l"(p), "l"(pol));
    return r;
}
// 16-byte form; p must be 16-byte aligned.
__device__ __forceinline__ uint4 ldg_v4_stream(const uint32_t *p, uint64_t pol) {
    uint4 r;
    asm("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
        : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
        : "l"(p), "l"(pol));
    return r;
}
// ---- bulk copies (TMA engine, no tensor map) into shared memory, completed on
// an mbarrier.  The source is always this GPU's own global memory and the
// destination this CTA's own shared memory.
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the bulk-copy (async) proxy
    asm volatile("fence.mbarrier_init.release.cluster;\n\tfence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_inval(unsigned long long *bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}
// Orders this thread's earlier generic-proxy shared-memory accesses (reads of
// a staging buffer) before bulk copies it issues next into that buffer.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// One arrival that also announces `bytes` of bulk-copy data for the phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// dst (shared) and src (global) 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the barrier's phase of the given parity to complete, giving up
// after timeout_ns (false).
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, uint32_t parity,
                                                  unsigned long long timeout_ns) {
    uint64_t t0 = 0;
    for (uint32_t n = 1;; ++n) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((n & 63u) == 0) {
            const uint64_t t = globaltimer_ns();
            if (t0 == 0)
                t0 = t;
            else if (t - t0 > timeout_ns)
                return false;
        }
    }
}

// Load through L1 of data written earlier in the same launch by other blocks:
// valid after a grid barrier, whose acquire (thread 0) and __syncthreads order
// this SM's later loads after every block's earlier writes.
template <typename T>
__device__ __forceinline__ T ld_l1(const T *p) {
    return __ldca(p);
}

__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t x) {
    const uint32_t lane = lane_id();
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t y = __shfl_up_sync(kFullMask, x, d);
        if (lane >= (uint32_t)d) x += y;
    }
    return x;
}
template <typename T>
__device__ __forceinline__ T warp_sum(T x) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) x += __shfl_xor_sync(kFullMask, x, d);
    return x;
}

// Warp-aggregated append: one atomicAdd per warp, items packed in lane order.
// Must be called by all 32 lanes.  A reservation past `cap` writes nothing and
// raises kErrCapacity instead of the reference's silent out-of-bounds write
// (queue.cuh:86 asserts only in debug builds).
__device__ __forceinline__ uint32_t warp_append(uint32_t *queue, uint32_t *count, uint32_t cap, bool want,
                                                uint32_t item, uint32_t *err) {
    const uint32_t m = __ballot_sync(kFullMask, want);
    if (m == 0) return 0;
    const uint32_t leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(count, (uint32_t)__popc(m));
    base = __shfl_sync(kFullMask, base, leader);
    if (want) {
        const uint32_t pos = base + __popc(m & lanemask_lt());
        if (pos < cap)
            queue[pos] = item;
        else
            atomicOr(err, kErrCapacity);
    }
    return m;
}

// Appends, for every lane, items[k] for each set bit k (< 4) of `which`, with
// one atomic per warp on `count`; all 32 lanes must call it.
__device__ __forceinline__ void warp_append4(uint32_t *queue, uint32_t *count, uint32_t cap, uint32_t which,
                                             const uint32_t (&items)[4], uint32_t *err) {
    const uint32_t c = __popc(which);
    uint32_t incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(kFullMask, incl, d);
        if (lane_id() >= (uint32_t)d) incl += y;
    }
    const uint32_t total = __shfl_sync(kFullMask, incl, 31);
    if (total == 0) return;
    uint32_t base = 0;
    if (lane_id() == 31) base = atomicAdd(count, total);
    base = __shfl_sync(kFullMask, base, 31);
    uint32_t pos = base + incl - c;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if ((which >> k) & 1u) {
            if (pos < cap)
                queue[pos] = items[k];
            else
                atomicOr(err, kErrCapacity);
            ++pos;
        }
}

__device__ __forceinline__ bool bitmap_test(const uint32_t *bm, uint32_t v) {
    return (ld_l2(bm + (v >> 5)) >> (v & 31u)) & 1u;
}
// For a bitmap no block writes during the current phase (read through L1).
__device__ __forceinline__ bool bitmap_test_l1(const uint32_t *bm, uint32_t v) {
    return (ld_l1(bm + (v >> 5)) >> (v & 31u)) & 1u;
}
// Returns true if this call set the bit.
__device__ __forceinline__ bool bitmap_set(uint32_t *bm, uint32_t v) {
    const uint32_t bit = 1u << (v & 31u);
    return (atomicOr(bm + (v >> 5), bit) & bit) == 0;
}
__device__ __forceinline__ void bitmap_clear(uint32_t *bm, uint32_t v) { atomicAnd(bm + (v >> 5), ~(1u << (v & 31u))); }
// Sets the bit without returning the old word: a fire-and-forget reduction
// the issuing thread never waits for.
__device__ __forceinline__ void bitmap_set_nr(uint32_t *bm, uint32_t v) {
    asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(bm + (v >> 5)), "r"(1u << (v & 31u)) : "memory");
}
__device__ __forceinline__ void red_add(uint32_t *p, uint32_t v) {
    asm volatile("red.relaxed.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bounded grid barrier for a cooperative launch (all blocks co-resident).
// The last block to arrive runs `leader()` on one thread with every block's
// prior writes visible, then releases the others; its writes are visible to
// all blocks after the barrier.  A waiter that exceeds timeout_ns raises
// kErrTimeout and returns false instead of spinning forever; every block then
// leaves the kernel at its next barrier or status check.
template <typename Leader>
__device__ __forceinline__ bool grid_barrier(uint32_t *bar_count, uint32_t *bar_gen, uint32_t *err,
                                             uint64_t timeout_ns, Leader &&leader) {
    __shared__ uint32_t s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t ok = 1;
        const uint32_t g = ld_acquire(bar_gen);
        __threadfence();
        const uint32_t arrived = atomicAdd(bar_count, 1u);
        if (arrived == gridDim.x - 1) {
            __threadfence();
            *bar_count = 0;
            leader();
            __threadfence();
            st_release(bar_gen, g + 1);
        } else {
            const uint64_t t0 = globaltimer_ns();
            uint32_t spins = 0;
            while (ld_acquire(bar_gen) == g) {
                ++spins;
                if ((spins & 255u) == 0 && (globaltimer_ns() - t0 > timeout_ns || spins > (1u << 28))) {
                    atomicOr(err, kErrTimeout);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        if (ld_l2(err) & kErrTimeout) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace dev
}  // namespace sepgraph
