// Selectors and engine options of the hybrid engine.
//
// Same names, enumerators and member functions as the reference's
// include/framework/common.h:13-321 (LoadBalancing, Priority, Model,
// MsgPassing, Scheduling, AlgoVariant, EngineOptions, LBToString) so that a
// sample written against the reference compiles against this header.  The
// numeric values of Model/MsgPassing/Scheduling define the variant id used on
// the device and at the C ABI: id = (model << 2) | (msg_passing << 1) | scheduling.
#pragma once
#include <cstdint>
#include <string>
#include <tuple>

namespace sepgraph {
namespace common {

enum class LoadBalancing { NONE, COARSE_GRAINED, FINE_GRAINED, HYBRID };
enum class Priority { NONE, LOW_HIGH, SAMPLING };
enum class Model { SYNC, ASYNC };
enum class MsgPassing { PUSH, PULL };
enum class Scheduling { TOPOLOGY_DRIVEN, DATA_DRIVEN };

class AlgoVariant {
   public:
    Model m_model;
    MsgPassing m_msg_passing;
    Scheduling m_scheduling;

    static const AlgoVariant ASYNC_PUSH_TD;
    static const AlgoVariant ASYNC_PUSH_DD;
    static const AlgoVariant ASYNC_PULL_TD;
    static const AlgoVariant ASYNC_PULL_DD;
    static const AlgoVariant SYNC_PUSH_TD;
    static const AlgoVariant SYNC_PUSH_DD;
    static const AlgoVariant SYNC_PULL_TD;
    static const AlgoVariant SYNC_PULL_DD;

    AlgoVariant() : m_model(Model::ASYNC), m_msg_passing(MsgPassing::PUSH), m_scheduling(Scheduling::DATA_DRIVEN) {}
    constexpr AlgoVariant(Model model, MsgPassing msg_passing, Scheduling scheduling)
        : m_model(model), m_msg_passing(msg_passing), m_scheduling(scheduling) {}

    bool operator==(const AlgoVariant &o) const {
        return m_model == o.m_model && m_msg_passing == o.m_msg_passing && m_scheduling == o.m_scheduling;
    }
    bool operator<(const AlgoVariant &o) const {
        return std::tie(m_model, m_msg_passing, m_scheduling) < std::tie(o.m_model, o.m_msg_passing, o.m_scheduling);
    }
    MsgPassing GetMsgPassing() const { return m_msg_passing; }
    Scheduling GetScheduling() const { return m_scheduling; }

    int Id() const { return ((int)m_model << 2) | ((int)m_msg_passing << 1) | (int)m_scheduling; }
    static AlgoVariant FromId(int id) {
        return AlgoVariant((Model)((id >> 2) & 1), (MsgPassing)((id >> 1) & 1), (Scheduling)(id & 1));
    }
    std::string ToString() const {
        std::string r = m_model == Model::SYNC ? "SYNC_" : "ASYNC_";
        r += m_msg_passing == MsgPassing::PUSH ? "PUSH_" : "PULL_";
        r += m_scheduling == Scheduling::DATA_DRIVEN ? "DD" : "TD";
        return r;
    }
};

inline const AlgoVariant AlgoVariant::ASYNC_PUSH_TD(Model::ASYNC, MsgPassing::PUSH, Scheduling::TOPOLOGY_DRIVEN);
inline const AlgoVariant AlgoVariant::ASYNC_PUSH_DD(Model::ASYNC, MsgPassing::PUSH, Scheduling::DATA_DRIVEN);
inline const AlgoVariant AlgoVariant::ASYNC_PULL_TD(Model::ASYNC, MsgPassing::PULL, Scheduling::TOPOLOGY_DRIVEN);
inline const AlgoVariant AlgoVariant::ASYNC_PULL_DD(Model::ASYNC, MsgPassing::PULL, Scheduling::DATA_DRIVEN);
inline const AlgoVariant AlgoVariant::SYNC_PUSH_TD(Model::SYNC, MsgPassing::PUSH, Scheduling::TOPOLOGY_DRIVEN);
inline const AlgoVariant AlgoVariant::SYNC_PUSH_DD(Model::SYNC, MsgPassing::PUSH, Scheduling::DATA_DRIVEN);
inline const AlgoVariant AlgoVariant::SYNC_PULL_TD(Model::SYNC, MsgPassing::PULL, Scheduling::TOPOLOGY_DRIVEN);
inline const AlgoVariant AlgoVariant::SYNC_PULL_DD(Model::SYNC, MsgPassing::PULL, Scheduling::DATA_DRIVEN);

inline std::string LBToString(LoadBalancing lb) {
    switch (lb) {
        case LoadBalancing::NONE: return "NONE";
        case LoadBalancing::COARSE_GRAINED: return "COARSED_GRAINED";
        case LoadBalancing::FINE_GRAINED: return "FINE_GRAINED";
        case LoadBalancing::HYBRID: return "HYBRID";
    }
    return "UNKNOWN";
}

// Mirror of EngineOptions (common.h:203-321), including its defaults.
class EngineOptions {
    Priority m_priority;
    LoadBalancing m_push_load_balancing;
    LoadBalancing m_pull_load_balancing;
    float m_priority_threshold;
    float m_cut_threshold;
    bool m_fused;
    bool m_force_push_load_balancing;
    bool m_force_pull_load_balancing;
    AlgoVariant m_algo_variant;
    bool m_force_variant;

   public:
    EngineOptions()
        : m_priority(Priority::NONE),
          m_push_load_balancing(LoadBalancing::NONE),
          m_pull_load_balancing(LoadBalancing::NONE),
          m_priority_threshold(0),
          m_cut_threshold(0),
          m_fused(false),
          m_force_push_load_balancing(false),
          m_force_pull_load_balancing(false),
          m_force_variant(false) {}

    void SetSampleBasedPriority(float cut_threshold = 0.2) {
        m_priority = Priority::SAMPLING;
        m_cut_threshold = cut_threshold;
    }
    void SetTwoLevelBasedPriority(float priority_threshold) {
        m_priority = Priority::LOW_HIGH;
        m_priority_threshold = priority_threshold;
    }
    Priority GetPriorityType() const { return m_priority; }
    float GetPriorityThreshold() const { return m_priority_threshold; }
    float GetCutThreshold() const { return m_cut_threshold; }
    void ForceVariant(AlgoVariant algo_variant) {
        m_force_variant = true;
        m_algo_variant = algo_variant;
    }
    AlgoVariant GetAlgoVariant() const { return m_algo_variant; }
    bool IsForceVariant() const { return m_force_variant; }
    void SetFused() { m_fused = true; }
    bool IsFused() const { return m_fused; }
    void SetLoadBalancing(MsgPassing msg_passing, LoadBalancing load_balancing) {
        if (msg_passing == MsgPassing::PUSH) {
            m_force_push_load_balancing = true;
            m_push_load_balancing = load_balancing;
        } else {
            m_force_pull_load_balancing = true;
            m_pull_load_balancing = load_balancing;
        }
    }
    bool IsForceLoadBalancing(MsgPassing msg_passing) const {
        return msg_passing == MsgPassing::PUSH ? m_force_push_load_balancing : m_force_pull_load_balancing;
    }
    LoadBalancing GetLoadBalancing(MsgPassing msg_passing) const {
        return msg_passing == MsgPassing::PUSH ? m_push_load_balancing : m_pull_load_balancing;
    }
};

}  // namespace common

namespace policy {
// include/framework/hybrid_policy.h:30-34
enum class AlgoType { ITERATIVE_SCHEME, TRAVERSAL_SCHEME };
}  // namespace policy
}  // namespace sepgraph
