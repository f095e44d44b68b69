// The four algorithm functors of the reference samples, written against
// sepgraph::api::AppBase.  Each keeps the reference functor's semantics
// (initial values, combine/accumulate return codes, activity and priority
// predicates); differences are noted per method.
#pragma once
#include <cstdint>

#include "sg_api.cuh"
#include "sg_device.cuh"

namespace sepgraph {
namespace apps {

using api::AppBase;
using common::MsgPassing;

constexpr uint32_t kInf = 0xffffffffu;  // IDENTITY_ELEMENT of BFS/SSSP/BC (UINT32_MAX)

// ---------------------------------------------------------------- BFS
// samples/hybrid_bfs/hybrid_bfs.cu:29-170.  value = level, buffer = level
// offered to the vertex; `non_atomic` selects the plain read-compare-store
// minimum (the sample's --non_atomic default, main.cpp:37) or atomicMin.
template <typename TValue, typename TBuffer, typename TWeight, typename... Unused>
struct BFS : AppBase<TValue, TBuffer, TWeight> {
    using AppBase<TValue, TBuffer, TWeight>::AccumulateBuffer;
    index_t m_source_node;
    bool m_non_atomic;

    BFS(index_t source, bool non_atomic) : m_source_node(source), m_non_atomic(non_atomic) {}

    __forceinline__ __device__ TValue GetInitValue(index_t) const override { return (TValue)kInf; }
    __forceinline__ __device__ TBuffer GetInitBuffer(index_t node) const override {
        return node == m_source_node ? (TBuffer)0 : (TBuffer)kInf;
    }
    __forceinline__ __host__ __device__ TBuffer GetIdentityElement() const override { return kInf; }

    __forceinline__ __device__ utils::pair<TBuffer, bool> CombineValueBuffer(index_t, TValue *p_value,
                                                                            TBuffer *p_buffer) override {
        TBuffer buf = *p_buffer;
        const bool improved = *p_value > buf;
        if (improved) {
            // under local lookahead two blocks may combine one vertex at once:
            // the value then only moves down (a reduction, no read-back; a
            // combine that saw a stale value expands once more, harmlessly)
            if (this->m_concurrent_combine) atomicMin(p_value, buf);
            else *p_value = buf;
            buf += 1;  // level offered to the neighbours
        }
        bool schedule;
        if (this->m_msg_passing == MsgPassing::PUSH) {
            schedule = improved;
        } else {
            // pull: a vertex pulls only while it has no level and was not just reached
            schedule = !improved && *p_buffer == kInf;
        }
        return utils::pair<TBuffer, bool>(buf, schedule);
    }

    __forceinline__ __device__ int AccumulateBuffer(index_t, index_t, TBuffer *p_buffer, TBuffer buffer) override {
        TBuffer prev;
        if (m_non_atomic) {
            prev = *p_buffer;
            if (prev > buffer) *p_buffer = buffer;
        } else {
            prev = atomicMin(p_buffer, buffer);
        }
        if (buffer < prev)
            return this->m_msg_passing == MsgPassing::PUSH ? this->ACCUMULATE_SUCCESS_CONTINUE
                                                           : this->ACCUMULATE_SUCCESS_BREAK;
        return this->ACCUMULATE_FAILURE_CONTINUE;
    }

    __forceinline__ __device__ bool IsActiveNode(index_t, TBuffer buffer) const override { return buffer != kInf; }
    // Levels are a monotone minimum only when the accumulation is atomic: a
    // plain store may overwrite a smaller level pushed concurrently by a round
    // of another depth (all pushes of one BFS round carry the same level).
    __forceinline__ __device__ bool ReorderSafe() const { return !m_non_atomic; }
};

// ---------------------------------------------------------------- SSSP
// samples/hybrid_sssp/hybrid_sssp.cu:28-141.  Relaxation is atomicMin on the
// uint32 distance offered to dst.  A plain read first skips the atomic when
// it cannot lower the distance (distances only decrease, so the skipped
// atomicMin would have returned FAILURE as well).
template <typename TValue, typename TBuffer, typename TWeight, typename... Unused>
struct SSSP : AppBase<TValue, TBuffer, TWeight> {
    using AppBase<TValue, TBuffer, TWeight>::AccumulateBuffer;
    index_t m_source_node;

    explicit SSSP(index_t source) : m_source_node(source) {}

    __forceinline__ __device__ TValue GetInitValue(index_t) const override { return (TValue)kInf; }
    __forceinline__ __device__ TBuffer GetInitBuffer(index_t node) const override {
        return node == m_source_node ? (TBuffer)0 : (TBuffer)kInf;
    }
    __forceinline__ __host__ __device__ TBuffer GetIdentityElement() const override { return kInf; }

    __forceinline__ __device__ utils::pair<TBuffer, bool> CombineValueBuffer(index_t, TValue *p_value,
                                                                            TBuffer *p_buffer) override {
        const TBuffer buf = *p_buffer;
        const bool improved = *p_value > buf;
        if (improved) {
            // concurrent combines of one vertex (local lookahead) keep the
            // smallest distance: a reduction without read-back
            if (this->m_concurrent_combine) atomicMin(p_value, buf);
            else *p_value = buf;
        }
        const bool schedule = this->m_msg_passing == MsgPassing::PUSH ? improved : true;
        return utils::pair<TBuffer, bool>(buf, schedule);
    }

    __forceinline__ __device__ int AccumulateBuffer(index_t, index_t, TWeight weight, TBuffer *p_buffer,
                                                    TBuffer buffer) override {
        if (buffer == kInf) return this->ACCUMULATE_FAILURE_CONTINUE;
        const TBuffer cand = buffer + weight;
        if (cand >= *p_buffer) return this->ACCUMULATE_FAILURE_CONTINUE;
        // The buffer only moves down, so a minimum reduction without read-back
        // is enough: the load above saw a larger value, hence the destination
        // has to be (re)scheduled.  A concurrent smaller candidate makes this a
        // redundant schedule of an already scheduled vertex, never a missed one.
        atomicMin(p_buffer, cand);
        return this->ACCUMULATE_SUCCESS_CONTINUE;
    }

    __forceinline__ __device__ bool IsActiveNode(index_t, TBuffer buffer) const override { return buffer != kInf; }
    __forceinline__ __device__ bool IsHighPriority(TBuffer current_priority, TBuffer buffer) const override {
        return current_priority > buffer;
    }
    __forceinline__ __device__ bool ReorderSafe() const { return true; }  // atomic monotone minimum
    // AccumulateBuffer above is the monotone minimum of this candidate (an
    // unreached source offers nothing: kInf never lowers a distance)
    __forceinline__ __device__ TBuffer RelaxCandidate(index_t, index_t, TWeight weight, TBuffer buffer) const {
        return buffer == kInf ? kInf : buffer + weight;
    }
};

// ---------------------------------------------------------------- PageRank
// samples/hybrid_pr/hybrid_pr.cu:24-126 with ALPHA = 0.85 (hybrid_pr_common.h:39).
// value = rank, buffer = residual.  Combine takes the whole residual
// (atomicExch), adds it to the rank and offers ALPHA*residual/outdeg.
// PullReduce/PullIdentity opt in to per-destination pre-summing in
// topology-driven pull rounds (one atomicAdd per vertex instead of per edge).
template <typename TValue, typename TBuffer, typename TWeight, typename... Unused>
struct PageRank : AppBase<TValue, TBuffer, TWeight> {
    using AppBase<TValue, TBuffer, TWeight>::AccumulateBuffer;
    double m_error;

    explicit PageRank(double error) : m_error(error) {}

    __forceinline__ __device__ TValue GetInitValue(index_t) const override { return (TValue)0.0f; }
    __forceinline__ __device__ TBuffer GetInitBuffer(index_t) const override { return (TBuffer)(1.0 - 0.85); }
    __forceinline__ __host__ __device__ TBuffer GetIdentityElement() const override { return (TBuffer)0.0f; }

    __forceinline__ __device__ utils::pair<TBuffer, bool> CombineValueBuffer(index_t node, TValue *p_value,
                                                                            TBuffer *p_buffer) override {
        TBuffer res = atomicExch(p_buffer, (TBuffer)0.0f);
        if (res > 0) {
            // two blocks may combine one vertex at once (local lookahead)
            if (this->m_concurrent_combine) atomicAdd(p_value, res);
            else *p_value += res;
            const index_t deg = this->m_msg_passing == MsgPassing::PUSH
                                    ? this->m_csr_graph.end_edge(node) - this->m_csr_graph.begin_edge(node)
                                    : this->m_csc_graph.out_degree(node);
            res = (TBuffer)(0.85 * (double)res / (double)deg);
        }
        return utils::pair<TBuffer, bool>(res, true);
    }

    __forceinline__ __device__ int AccumulateBuffer(index_t, index_t, TBuffer *p_buffer, TBuffer buffer) override {
        const TBuffer prev = atomicAdd(p_buffer, buffer);
        const bool crossed = prev < m_error && prev + buffer > m_error;
        return crossed ? this->ACCUMULATE_SUCCESS_CONTINUE : this->ACCUMULATE_FAILURE_CONTINUE;
    }

    __forceinline__ __device__ bool IsActiveNode(index_t, TBuffer buffer) const override { return buffer > m_error; }
    __forceinline__ __device__ bool IsHighPriority(TBuffer current_priority, TBuffer buffer) const override {
        return current_priority <= buffer;
    }

    __forceinline__ __device__ TBuffer PullReduce(TBuffer a, TBuffer b) const { return a + b; }
    __forceinline__ __device__ TBuffer PullIdentity() const { return (TBuffer)0.0f; }
    // residual pushes are atomic additions: any order reaches the same fixed point within the threshold
    __forceinline__ __device__ bool ReorderSafe() const { return true; }
};

// ---------------------------------------------------------------- BC
// Level stack of the forward pass (sepgraph::dev::WorklistStack,
// include/groute/device/worklist_stack.cuh:16-111): vertices are appended in
// the round their level is fixed and PostComputation closes one segment per
// round, so segment d holds exactly the vertices at depth d.
struct LevelStack {
    uint32_t *data;     // nnodes
    uint32_t *count;    // items appended so far
    uint32_t *ends;     // ends[d] = end of segment d
    uint32_t *nlevels;  // segments closed so far
    uint32_t capacity;
    uint32_t max_levels;
    uint32_t *err;

    __device__ __forceinline__ void append(uint32_t v) const {
        const uint32_t p = atomicAdd(count, 1u);
        if (p < capacity)
            data[p] = v;
        else
            atomicOr(err, dev::kErrCapacity);
    }
    __device__ __forceinline__ void push() const {
        const uint32_t n = *nlevels;
        if (n < max_levels) {
            ends[n] = min(*count, capacity);
            *nlevels = n + 1;
        }
    }
};

// samples/hybrid_bc/hybrid_bc.cu:22-131 (Stage1).  Path counts are uint64
// (the reference uses float); an add that wraps raises kErrOverflow.
template <typename TValue, typename TBuffer, typename TWeight, typename... Unused>
struct BCForward : AppBase<TValue, TBuffer, TWeight> {
    using AppBase<TValue, TBuffer, TWeight>::AccumulateBuffer;
    index_t m_source_node;
    unsigned long long *m_sigmas;
    uint32_t *m_p_search_depth;
    LevelStack m_stack;

    BCForward(index_t source, unsigned long long *sigmas, uint32_t *search_depth, LevelStack stack)
        : m_source_node(source), m_sigmas(sigmas), m_p_search_depth(search_depth), m_stack(stack) {}

    __forceinline__ __device__ TValue GetInitValue(index_t) const override { return (TValue)kInf; }
    __forceinline__ __device__ TBuffer GetInitBuffer(index_t node) const override {
        return node == m_source_node ? (TBuffer)0 : (TBuffer)kInf;
    }
    __forceinline__ __host__ __device__ TBuffer GetIdentityElement() const override { return kInf; }

    __forceinline__ __device__ utils::pair<TBuffer, bool> CombineValueBuffer(index_t node, TValue *p_value,
                                                                            TBuffer *p_buffer) override {
        TBuffer buf = *p_buffer;
        const bool improved = *p_value > buf;
        if (improved) {
            *p_value = buf;
            buf += 1;
            m_stack.append(node);
        }
        const bool schedule =
            this->m_msg_passing == MsgPassing::PUSH ? improved : (!improved && *p_buffer == kInf);
        return utils::pair<TBuffer, bool>(buf, schedule);
    }

    __forceinline__ __device__ void add_sigma(index_t dst, index_t src) const {
        const unsigned long long s = dev::ld_l2(m_sigmas + src);
        const unsigned long long old = atomicAdd(m_sigmas + dst, s);
        if (old + s < old) atomicOr(m_stack.err, dev::kErrOverflow);
    }

    __forceinline__ __device__ int AccumulateBuffer(index_t src, index_t dst, TBuffer *p_buffer,
                                                    TBuffer buffer) override {
        const TBuffer prev = atomicMin(p_buffer, buffer);
        if (prev == kInf) {
            add_sigma(dst, src);
            atomicMax(m_p_search_depth, buffer);
        } else if (dev::ld_l2(p_buffer) == buffer) {
            add_sigma(dst, src);
        }
        return buffer < prev ? this->ACCUMULATE_SUCCESS_CONTINUE : this->ACCUMULATE_FAILURE_CONTINUE;
    }

    __forceinline__ __device__ bool IsActiveNode(index_t, TBuffer buffer) const override { return buffer != kInf; }
    __forceinline__ __device__ void PostComputation() override { m_stack.push(); }
};

}  // namespace apps
}  // namespace sepgraph
