// BC backward pass shared by the single-query kernel and the batched one.
//
// Dependency accumulation of Brandes' algorithm over the forward level stack,
// deepest level first, one barrier per phase (StageTwoDD{,CTA}Fused,
// samples/hybrid_bc/hybrid_bc.cu:134-225; host form hybrid_bc_host.cpp:66-80):
//   delta[v] = sum over out-edges v->w with level[w] == level[v]+1 of
//              sigma[v]/sigma[w] * (1 + delta[w])
// Each vertex is owned by one thread (small out-degree) or one warp; vertices
// above kBcBigDegree out-edges are split into chunks whose partial sums are
// added atomically after a barrier.  The source (depth 0) keeps delta 0, and
// the result is delta * 0.5 (hybrid_bc.cu:374-376).
#pragma once
#include <cstdint>

#include "sg_device.cuh"

namespace sepgraph {
namespace bc {

constexpr uint32_t kBcBigDegree = 256;
constexpr uint32_t kBcChunk = 256;

struct BCBackArgs {
    const uint32_t *row, *col;
    const uint32_t *level;
    const unsigned long long *sigma;
    float *delta;
    float *bc_out;  // delta * 0.5
    const uint32_t *stack, *ends;
    uint32_t nlevels, max_depth, nv;
    uint4 *chunks;  // (v, begin, len, -)
    uint32_t chunk_cap;
    uint32_t *chunk_count;  // [max_depth + 1], zero on entry
    uint32_t *bar;          // count, gen (single-query kernel)
    uint32_t *err;
    unsigned long long timeout_ns;
};

__device__ __forceinline__ float bc_term(const BCBackArgs &a, unsigned long long sv, uint32_t w, uint32_t d) {
    if (__ldcg(a.level + w) != d + 1) return 0.f;
    const float ratio = (float)((double)sv / (double)__ldcg(a.sigma + w));
    return ratio * (1.0f + __ldcg(a.delta + w));
}

// The whole backward pass for one query, run by `nt` threads numbered from
// `gt` (warps gw of nw); `sync()` is a barrier over exactly those threads and
// returns false when a bounded wait gave up.
template <typename Sync>
__device__ bool backward(const BCBackArgs &a, uint32_t gt, uint32_t nt, Sync &&sync) {
    const uint32_t lane = dev::lane_id();
    const uint32_t gw = gt >> 5, nw = nt >> 5;
    for (uint32_t d = a.max_depth; d >= 1; --d) {
        const uint32_t b = __ldcg(a.ends + d - 1), e = __ldcg(a.ends + d);
        for (uint32_t base = b + gw * 32; base < e; base += nw * 32) {
            const uint32_t i = base + lane;
            const bool valid = i < e;
            uint32_t v = 0, beg = 0, deg = 0;
            unsigned long long sv = 0;
            if (valid) {
                v = __ldcg(a.stack + i);
                beg = __ldg(a.row + v);
                deg = __ldg(a.row + v + 1) - beg;
                sv = __ldcg(a.sigma + v);
            }
            const bool big = valid && deg > kBcBigDegree;
            const bool mid = valid && !big && deg > 32;
            if (valid && !big && !mid) {
                float s = 0.f;
                for (uint32_t k = beg; k < beg + deg; ++k) s += bc_term(a, sv, __ldg(a.col + k), d);
                a.delta[v] = s;
            }
            if (big) {
                const uint32_t nch = (deg + kBcChunk - 1) / kBcChunk;
                const uint32_t c0 = atomicAdd(a.chunk_count + d, nch);
                for (uint32_t c = 0; c < nch; ++c) {
                    if (c0 + c < a.chunk_cap)
                        a.chunks[c0 + c] = make_uint4(v, beg + c * kBcChunk, min(kBcChunk, deg - c * kBcChunk), 0);
                    else
                        atomicOr(a.err, dev::kErrChunkCapacity);
                }
            }
            uint32_t m = __ballot_sync(dev::kFullMask, mid);
            while (m) {
                const uint32_t j = __ffs(m) - 1;
                m &= m - 1;
                const uint32_t vj = __shfl_sync(dev::kFullMask, v, j);
                const uint32_t bj = __shfl_sync(dev::kFullMask, beg, j);
                const uint32_t dj = __shfl_sync(dev::kFullMask, deg, j);
                const unsigned long long sj = __shfl_sync(dev::kFullMask, sv, j);
                float s = 0.f;
                for (uint32_t k = lane; k < dj; k += 32) s += bc_term(a, sj, __ldg(a.col + bj + k), d);
                s = dev::warp_sum(s);
                if (lane == 0) a.delta[vj] = s;
            }
        }
        if (!sync()) return false;
        const uint32_t nc = min(__ldcg(a.chunk_count + d), a.chunk_cap);
        if (nc) {
            for (uint32_t c = gw; c < nc; c += nw) {
                const uint4 ch = a.chunks[c];
                const unsigned long long sv = __ldcg(a.sigma + ch.x);
                float s = 0.f;
                for (uint32_t k = lane; k < ch.z; k += 32) s += bc_term(a, sv, __ldg(a.col + ch.y + k), d);
                s = dev::warp_sum(s);
                if (lane == 0) atomicAdd(a.delta + ch.x, s);
            }
            if (!sync()) return false;
        }
    }
    for (uint32_t v = gt; v < a.nv; v += nt) a.bc_out[v] = __ldcg(a.delta + v) * 0.5f;
    return true;
}

}  // namespace bc
}  // namespace sepgraph
