// Two application functors written the way the reference's samples write
// theirs (sepgraph::api::AppBase subclasses with `override`, the four
// ACCUMULATE_* codes, utils::pair results) and driven through the C++ Engine
// mirror with the reference's lifecycle: Engine(AlgoType) -> SetOptions ->
// LoadGraph -> InitGraph -> Start -> GatherValue (include/framework/framework.cuh:84-399).
//
//   LevelBFS        breadth-first levels, level-synchronous push/pull like the
//                   BFS sample's functor, accumulation by atomicMin
//   MinLabelCC      connected components by minimum-label propagation: an
//                   application the library itself does not ship
//
// Usage: dropin_functors <rmat scale> <source> <out prefix>
// Writes <prefix>_bfs_hybrid.u32, <prefix>_bfs_push.u32 and <prefix>_cc.u32
// (nv uint32 each) for the test to compare with the oracle.  Exit code 0 on
// success.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "sg_runtime.cuh"

using sepgraph::api::AppBase;

template <typename TValue, typename TBuffer, typename TWeight, typename... UnusedData>
struct LevelBFS : AppBase<TValue, TBuffer, TWeight> {
    using AppBase<TValue, TBuffer, TWeight>::AccumulateBuffer;
    static constexpr TBuffer kUnreached = 0xffffffffu;
    index_t m_root;

    explicit LevelBFS(index_t root) : m_root(root) {}

    __forceinline__ __device__ TValue GetInitValue(index_t) const override { return kUnreached; }
    __forceinline__ __device__ TBuffer GetInitBuffer(index_t node) const override {
        return node == m_root ? 0 : kUnreached;
    }
    __forceinline__ __host__ __device__ TBuffer GetIdentityElement() const override { return kUnreached; }

    __forceinline__ __device__ utils::pair<TBuffer, bool> CombineValueBuffer(index_t, TValue *p_value,
                                                                            TBuffer *p_buffer) override {
        const TBuffer offered = *p_buffer;
        bool schedule;
        TBuffer next = offered;
        if (*p_value > offered) {
            *p_value = offered;
            next = offered + 1;
            schedule = this->m_msg_passing == sepgraph::common::MsgPassing::PUSH;
        } else {
            // a pulling vertex keeps pulling until some neighbour offers it a level
            schedule = this->m_msg_passing == sepgraph::common::MsgPassing::PULL && offered == kUnreached;
        }
        return utils::pair<TBuffer, bool>(next, schedule);
    }

    __forceinline__ __device__ int AccumulateBuffer(index_t, index_t, TBuffer *p_buffer, TBuffer buffer) override {
        const TBuffer before = atomicMin(p_buffer, buffer);
        if (buffer >= before) return this->ACCUMULATE_FAILURE_CONTINUE;
        return this->m_msg_passing == sepgraph::common::MsgPassing::PUSH ? this->ACCUMULATE_SUCCESS_CONTINUE
                                                                        : this->ACCUMULATE_SUCCESS_BREAK;
    }

    __forceinline__ __device__ bool IsActiveNode(index_t, TBuffer buffer) const override {
        return buffer != kUnreached;
    }
};

template <typename TValue, typename TBuffer, typename TWeight, typename... UnusedData>
struct MinLabelCC : AppBase<TValue, TBuffer, TWeight> {
    using AppBase<TValue, TBuffer, TWeight>::AccumulateBuffer;
    static constexpr TValue kNone = 0xffffffffu;

    __forceinline__ __device__ TValue GetInitValue(index_t) const override { return kNone; }
    __forceinline__ __device__ TBuffer GetInitBuffer(index_t node) const override { return node; }
    __forceinline__ __host__ __device__ TBuffer GetIdentityElement() const override { return kNone; }

    __forceinline__ __device__ utils::pair<TBuffer, bool> CombineValueBuffer(index_t, TValue *p_value,
                                                                            TBuffer *p_buffer) override {
        const TBuffer label = *p_buffer;
        const bool lower = label < *p_value;
        if (lower) *p_value = label;
        return utils::pair<TBuffer, bool>(label, lower);
    }

    __forceinline__ __device__ int AccumulateBuffer(index_t, index_t, TBuffer *p_buffer, TBuffer buffer) override {
        return buffer < atomicMin(p_buffer, buffer) ? this->ACCUMULATE_SUCCESS_CONTINUE
                                                    : this->ACCUMULATE_FAILURE_CONTINUE;
    }

    __forceinline__ __device__ bool IsActiveNode(index_t, TBuffer) const override { return true; }
};

static bool write_u32(const char *path, const std::vector<uint32_t> &v) {
    FILE *f = std::fopen(path, "wb");
    if (!f) return false;
    const bool ok = std::fwrite(v.data(), sizeof(uint32_t), v.size(), f) == v.size();
    std::fclose(f);
    return ok;
}

#define CHECK(x)                                                                    \
    do {                                                                            \
        sg_status st_ = (x);                                                        \
        if (st_ != SG_OK) {                                                         \
            std::fprintf(stderr, "%s failed: %s\n", #x, sg_status_string(st_));     \
            return 1;                                                               \
        }                                                                           \
    } while (0)

int main(int argc, char **argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s <rmat scale> <source> <out prefix>\n", argv[0]);
        return 2;
    }
    const uint32_t scale = (uint32_t)std::atoi(argv[1]);
    const uint32_t root = (uint32_t)std::atoi(argv[2]);
    const std::string prefix = argv[3];
    using namespace sepgraph;

    sg_ctx *ctx = nullptr;
    CHECK(sg_init(0, &ctx));
    sg_hgraph *h = nullptr;
    CHECK(sg_hgraph_gen_rmat(scale, 16, 0.57, 0.19, 0.19, 1, SG_GEN_SYMMETRIC, &h));
    sg_graph *g = nullptr;
    CHECK(sg_graph_create_from_host(ctx, h, SG_GRAPH_SYMMETRIC, &g));

    {  // hybrid policy (push and pull rounds)
        engine::Engine<uint32_t, uint32_t, graphs::NoWeight, LevelBFS, index_t> e(policy::AlgoType::TRAVERSAL_SCHEME);
        common::EngineOptions opt;
        e.SetOptions(opt);
        e.LoadGraph(g);
        index_t r = root;
        e.InitGraph(r);
        CHECK(e.Start());
        e.PrintInfo();
        if (!write_u32((prefix + "_bfs_hybrid.u32").c_str(), e.GatherValue())) return 1;
    }
    {  // forced data-driven push with fine-grained load balancing
        engine::Engine<uint32_t, uint32_t, graphs::NoWeight, LevelBFS, index_t> e(policy::AlgoType::TRAVERSAL_SCHEME);
        common::EngineOptions opt;
        opt.ForceVariant(common::AlgoVariant::ASYNC_PUSH_DD);
        opt.SetLoadBalancing(common::MsgPassing::PUSH, common::LoadBalancing::FINE_GRAINED);
        e.SetOptions(opt);
        e.LoadGraph(g);
        index_t r = root;
        e.InitGraph(r);
        CHECK(e.Start());
        if (!write_u32((prefix + "_bfs_push.u32").c_str(), e.GatherValue())) return 1;
    }
    {  // connected components: every vertex active at the start, forced push
        engine::Engine<uint32_t, uint32_t, graphs::NoWeight, MinLabelCC> e(policy::AlgoType::TRAVERSAL_SCHEME);
        common::EngineOptions opt;
        opt.ForceVariant(common::AlgoVariant::ASYNC_PUSH_DD);
        e.SetOptions(opt);
        e.LoadGraph(g);
        e.InitGraph();
        e.max_iteration = 100000;
        CHECK(e.Start());
        e.PrintInfo();
        if (!write_u32((prefix + "_cc.u32").c_str(), e.GatherValue())) return 1;
    }
    CHECK(sg_graph_destroy(g));
    CHECK(sg_hgraph_destroy(h));
    CHECK(sg_destroy(ctx));
    return 0;
}
