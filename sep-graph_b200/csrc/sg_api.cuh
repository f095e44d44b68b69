// Algorithm-functor API of the B200 hybrid engine.
//
// AppBase keeps the reference's plugin contract (include/framework/variants/api.cuh:22-120):
// the same member names, argument meanings and the four ACCUMULATE_* return
// codes, so an application functor written for the reference compiles here.
// Differences, all invisible to a functor:
//  - the device views (CSRGraph/CSCGraph/GraphDatum) are this library's own
//    (read-only graph arrays are loaded through the non-coherent path);
//  - the engine calls functor methods with qualified names (app.App::Method),
//    so the virtual declarations kept for `override` compatibility never cause
//    a device-side virtual dispatch on a host-constructed object;
//  - AccumulateBuffer's default bodies return ACCUMULATE_FAILURE_CONTINUE
//    instead of assert(false).
// Optional extension (not in the reference): a functor may define
//   __device__ TBuffer PullReduce(TBuffer a, TBuffer b) const and
//   __device__ TBuffer PullIdentity() const
// to declare that AccumulateBuffer over the values pulled into one destination
// may be pre-combined with PullReduce; the engine then issues one
// AccumulateBuffer per destination in topology-driven pull rounds.
#pragma once
#include <cstdint>
#include <type_traits>

#include "sg_common.h"

typedef uint32_t index_t;  // include/groute/graphs/common.h:36

namespace utils {
// include/utils/cuda_utils.h:64-71
template <typename T1, typename T2>
struct __align__(8) pair {
    T1 first;
    T2 second;
    __forceinline__ __host__ __device__ pair(const T1 _first, const T2 _second) : first(_first), second(_second) {}
};
}  // namespace utils

namespace sepgraph {
namespace graphs {

struct NoWeight {};  // groute::graphs::NoWeight

namespace dev {

// Out-edge view (groute::graphs::dev::CSRGraph, csr_graph.h:745-800).
struct CSRGraph {
    index_t nnodes = 0;
    index_t nedges = 0;
    const index_t *row_start = nullptr;
    const index_t *edge_dst = nullptr;
    const index_t *edge_weights = nullptr;

    __device__ __forceinline__ index_t begin_edge(index_t node) const { return __ldg(row_start + node); }
    __device__ __forceinline__ index_t end_edge(index_t node) const { return __ldg(row_start + node + 1); }
    __device__ __forceinline__ index_t edge_dest(index_t edge) const { return __ldg(edge_dst + edge); }
    __host__ __device__ __forceinline__ bool owns(index_t node) const { return node < nnodes; }
    __host__ __device__ __forceinline__ index_t owned_start_node() const { return 0; }
    __host__ __device__ __forceinline__ index_t owned_nnodes() const { return nnodes; }
    __host__ __device__ __forceinline__ index_t global_nnodes() const { return nnodes; }
};

// In-edge view (groute::graphs::dev::CSCGraph, csr_graph.h:800-871). out_degree
// is derived from the CSR row offsets instead of a separate array.
struct CSCGraph {
    index_t nnodes = 0;
    index_t nedges = 0;
    const index_t *col_start = nullptr;
    const index_t *edge_source = nullptr;
    const index_t *edge_weights = nullptr;
    const index_t *csr_row_start = nullptr;

    __device__ __forceinline__ index_t begin_edge(index_t node) const { return __ldg(col_start + node); }
    __device__ __forceinline__ index_t end_edge(index_t node) const { return __ldg(col_start + node + 1); }
    __device__ __forceinline__ index_t edge_src(index_t edge) const { return __ldg(edge_source + edge); }
    __device__ __forceinline__ index_t out_degree(index_t node) const {
        return __ldg(csr_row_start + node + 1) - __ldg(csr_row_start + node);
    }
    __host__ __device__ __forceinline__ bool owns(index_t node) const { return node < nnodes; }
    __host__ __device__ __forceinline__ index_t owned_nnodes() const { return nnodes; }
    __host__ __device__ __forceinline__ index_t global_nnodes() const { return nnodes; }
};

// Per-vertex or per-edge device array (groute::graphs::dev::GraphDatum).
template <typename T>
struct GraphDatum {
    T *data_ptr = nullptr;
    index_t size = 0;
    GraphDatum() = default;
    __host__ __device__ GraphDatum(T *p, index_t n) : data_ptr(p), size(n) {}
    __device__ __forceinline__ T get_item(index_t idx) const { return data_ptr[idx]; }
    __device__ __forceinline__ T &operator[](index_t idx) const { return data_ptr[idx]; }
    __device__ __forceinline__ T *get_item_ptr(index_t idx) const { return data_ptr + idx; }
    __device__ __forceinline__ void set_item(index_t idx, const T &item) const { data_ptr[idx] = item; }
};

}  // namespace dev
}  // namespace graphs

namespace api {

template <typename TValue, typename TBuffer, typename TWeight>
struct AppBase {
    // [ACCUMULATE] [CONTINUE/BREAK] (api.cuh:25-29)
    static constexpr int ACCUMULATE_SUCCESS_BREAK = 0;
    static constexpr int ACCUMULATE_SUCCESS_CONTINUE = 1;
    static constexpr int ACCUMULATE_FAILURE_BREAK = 2;
    static constexpr int ACCUMULATE_FAILURE_CONTINUE = 3;

    graphs::dev::CSRGraph m_csr_graph;
    graphs::dev::CSCGraph m_csc_graph;
    uint32_t m_nnodes = 0;
    uint32_t m_nedges = 0;
    common::Model m_model = common::Model::ASYNC;
    common::MsgPassing m_msg_passing = common::MsgPassing::PUSH;
    common::Scheduling m_scheduling = common::Scheduling::DATA_DRIVEN;
    uint32_t *m_p_current_round = nullptr;
    // Extension (no reference counterpart): set by the engine while local
    // lookahead runs, when CombineValueBuffer may be called for one vertex by
    // two blocks at once; reorder-safe functors then combine atomically.
    bool m_concurrent_combine = false;

    __forceinline__ __device__ virtual TValue GetInitValue(index_t node) const = 0;
    __forceinline__ __device__ virtual TBuffer GetInitBuffer(index_t node) const = 0;
    __forceinline__ __host__ __device__ virtual TBuffer GetIdentityElement() const = 0;
    __forceinline__ __device__ virtual utils::pair<TBuffer, bool> CombineValueBuffer(index_t node, TValue *p_value,
                                                                                    TBuffer *p_buffer) = 0;
    __forceinline__ __device__ virtual int AccumulateBuffer(index_t src, index_t dst, TBuffer *p_buffer,
                                                            TBuffer buffer) {
        return ACCUMULATE_FAILURE_CONTINUE;
    }
    __forceinline__ __device__ virtual int AccumulateBuffer(index_t src, index_t dst, TWeight weight,
                                                            TBuffer *p_buffer, TBuffer buffer) {
        return ACCUMULATE_FAILURE_CONTINUE;
    }
    __forceinline__ __device__ virtual bool IsActiveNode(index_t node, TBuffer buffer) const { return false; }
    __forceinline__ __device__ virtual void PostComputation() {}
    __forceinline__ __device__ virtual bool IsHighPriority(TBuffer current_priority, TBuffer buffer) const {
        return true;
    }

    __host__ void SetVariant(common::Model model, common::MsgPassing msg_passing, common::Scheduling scheduling) {
        m_model = model;
        m_msg_passing = msg_passing;
        m_scheduling = scheduling;
    }
    __host__ void SetVariant(common::AlgoVariant v) {
        m_model = v.m_model;
        m_msg_passing = v.m_msg_passing;
        m_scheduling = v.m_scheduling;
    }
};

}  // namespace api
}  // namespace sepgraph
