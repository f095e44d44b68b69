// Query server with continuous batching over device-resident graphs
// (declarations and contract in include/sepgraph.h, "serving").
//
// Each slot is a worker thread with its own sg_ctx (stream, batch scratch).  A
// free slot takes the pending queries of the oldest request's algorithm (or,
// with one graph per batch, of the (algorithm, graph) group whose batches have
// run shortest so far, with an aging bound that serves the oldest query's
// group first once it waited too long),
// reserves an estimate of their device scratch against the HBM budget (waiting
// for other slots to release memory when it does not fit), runs them as one
// batched launch and completes their tickets.  Requests that arrive while a
// batch runs are taken by the next free slot, so work from different batches
// overlaps on the device.  PageRank (and BC with path counts) run as single
// queries on a view of the graph bound to the slot's own context, so they
// never share a stream or scratch with another slot or with the caller.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../../include/sepgraph.h"
#include "../sg_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct GraphInfo {
    sg_graph *g;
    uint32_t nv;
    uint64_t ne;
};

// The graph table never reallocates, so workers index it without the lock
// (a graph id is valid once sg_server_add_graph has returned it).
constexpr size_t kMaxGraphs = 4096;

struct Pending {
    uint64_t ticket;
    sg_query q;
    Clock::time_point t_submit;
};

struct TicketState {
    bool done = false;
    sg_status status = SG_OK;
    double latency_ms = 0;
};

}  // namespace

struct sg_server {
    int device = 0;
    sg_server_config cfg{};
    std::vector<GraphInfo> graphs;
    // views[slot][graph]: the graph bound to the slot's context with its own
    // workspace, made on first use by that slot's worker only
    std::vector<std::vector<sg_graph *>> views;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Pending> pending;
    std::unordered_map<uint64_t, TicketState> tickets;
    std::vector<std::thread> workers;
    std::vector<sg_ctx *> slot_ctx;
    bool stop = false;
    uint64_t next_ticket = 1;
    // accounting
    uint64_t budget = 0, in_use = 0, peak = 0;
    uint64_t submitted = 0, completed = 0, failed = 0, batches = 0;
    std::vector<double> latencies;
    // measured batch time per (algorithm, graph) group, for shortest-first selection
    std::map<std::pair<int, uint32_t>, double> group_ms;
    bool have_first = false;
    // optional batch log (one line per batch) when SEPGRAPH_SERVER_LOG names a file
    FILE *log = nullptr;
    std::mutex log_mu;
    Clock::time_point t_first, t_last;

    void worker(int slot);
    sg_graph *view(int slot, uint32_t graph_id);
    void run_batch(int slot, std::vector<Pending> &batch, std::vector<sg_status> &status);
    uint64_t estimate(const std::vector<Pending> &b) const;
};

namespace {

sg_options server_options(const sg_server_config &c, int algo) {
    sg_options o;
    sg_options_default(&o);
    o.max_iteration = 1000000;
    o.blocks_per_sm = c.blocks_per_sm ? c.blocks_per_sm : std::max(1u, 6u / std::max(1u, c.slots));  // slots share the SMs
    if (algo == SG_QUERY_SSSP) {
        // delta-stepping: data-driven push with two-level priority at the
        // configured delta, or each graph's own reference heuristic
        // 32*avg_w/avg_deg when it is 0; blocks follow their own discoveries
        // four levels deep inside a round (bit-exact, fewer rounds).  Measured
        // on B200, 85 SSSP queries over the 16 served graphs in one batch:
        // 527 ms with the hybrid policy and lookahead 16, 408 ms forced push,
        // 251 ms forced push with lookahead 4 (equal distances).
        o.variant = SG_ASYNC_PUSH_DD;
        o.priority = SG_PRIORITY_LOW_HIGH;
        o.priority_delta = c.sssp_delta;
        o.local_depth = 4;
    }
    if (algo == SG_QUERY_PAGERANK) {
        o.pr_error = c.pr_error;
        o.max_iteration = 100000;
    }
    return o;
}

}  // namespace

namespace {

// Runs q as one batched launch; a batch that fails as a whole (one query's
// path counts overflow uint64, say) runs again one query at a time, so that
// only the failing queries report the error.  idx[k] is q[k]'s slot in status.
template <typename Call>
void run_isolated(const std::vector<sg_batch_query> &q, const std::vector<size_t> &idx, std::vector<sg_status> &status,
                  Call &&call) {
    const sg_status st = call(q.data(), (uint32_t)q.size());
    if (st == SG_OK || q.size() == 1) {
        for (size_t i : idx) status[i] = st;
        return;
    }
    for (size_t k = 0; k < q.size(); ++k) status[idx[k]] = call(&q[k], 1u);
}

}  // namespace

sg_graph *sg_server::view(int slot, uint32_t graph_id) {
    std::vector<sg_graph *> &v = views[slot];
    if (v.size() <= graph_id) v.resize(graph_id + 1, nullptr);
    if (!v[graph_id]) v[graph_id] = sgb::graph_view(graphs[graph_id].g, slot_ctx[slot]);
    return v[graph_id];
}

uint64_t sg_server::estimate(const std::vector<Pending> &b) const {
    // Device scratch of one batch: per-team workspaces sized for the largest
    // graph (about 32 bytes per vertex, 56 with BC's path counts, level stack
    // and dependencies; at most one team per query and per resident block),
    // multi-source BFS masks and level rows, and staging for host outputs.
    if (b.empty()) return 0;
    const int algo = b.front().q.algo;
    uint64_t nv_max = 0, outs = 0;
    std::map<uint32_t, uint64_t> per_graph;
    for (auto &p : b) {
        const uint64_t nv = graphs[p.q.graph_id].nv;
        nv_max = std::max(nv_max, nv);
        outs += 8 * nv;
        per_graph[p.q.graph_id]++;
    }
    const uint64_t teams = std::min<uint64_t>(b.size(), 148ull * 8);
    uint64_t bytes = teams * nv_max * (algo == SG_QUERY_BC ? 56 : 32) + outs;
    if (algo == SG_QUERY_BFS)
        for (auto &kv : per_graph)
            if (kv.second >= std::max(1u, cfg.msbfs_min))
                bytes += graphs[kv.first].nv * (32 + 4 * std::min<uint64_t>(kv.second, 64));
    if (algo == SG_QUERY_BC)  // multi-source BC scratch: 32 path counts, dependencies, q, masks, lists, rows
        for (auto &kv : per_graph)
            if (kv.second >= std::max(1u, cfg.msbfs_min)) bytes += graphs[kv.first].nv * 1000ull;
    return bytes;
}

void sg_server::run_batch(int slot, std::vector<Pending> &b, std::vector<sg_status> &status) {
    sg_ctx *ctx = slot_ctx[slot];
    const int algo = b.front().q.algo;
    const sg_options o = server_options(cfg, algo);
    status.assign(b.size(), SG_OK);
    if (algo == SG_QUERY_BFS) {
        // many queries on one graph -> multi-source BFS (64 per launch); the rest -> one batched launch
        std::map<uint32_t, std::vector<size_t>> by_graph;
        for (size_t i = 0; i < b.size(); ++i) by_graph[b[i].q.graph_id].push_back(i);
        std::vector<size_t> rest;
        for (auto &kv : by_graph) {
            if (kv.second.size() < std::max(1u, cfg.msbfs_min)) {
                rest.insert(rest.end(), kv.second.begin(), kv.second.end());
                continue;
            }
            const GraphInfo &gi = graphs[kv.first];
            sg_options om = o;  // multi-source launches size their own grid unless the config fixes it
            om.blocks_per_sm = (int32_t)cfg.blocks_per_sm;
            for (size_t s = 0; s < kv.second.size(); s += 64) {
                const size_t m = std::min<size_t>(64, kv.second.size() - s);
                std::vector<uint32_t> src(m);
                std::vector<uint32_t *> rows(m);
                for (size_t k = 0; k < m; ++k) {
                    src[k] = b[kv.second[s + k]].q.source;
                    rows[k] = (uint32_t *)b[kv.second[s + k]].q.out;  // each level row straight to its query
                }
                const sg_status st = sgb::msbfs_on(ctx, gi.g, src.data(), (uint32_t)m, &om, nullptr, nullptr, rows.data());
                for (size_t k = 0; k < m; ++k) status[kv.second[s + k]] = st;
            }
        }
        if (!rest.empty()) {
            std::vector<sg_batch_query> q(rest.size());
            for (size_t k = 0; k < rest.size(); ++k)
                q[k] = {graphs[b[rest[k]].q.graph_id].g, b[rest[k]].q.source, 0, b[rest[k]].q.out};
            run_isolated(q, rest, status, [&](const sg_batch_query *qq, uint32_t n) {
                return sg_bfs_batch(ctx, qq, n, &o, nullptr, nullptr);
            });
        }
    } else if (algo == SG_QUERY_SSSP) {
        std::vector<sg_batch_query> q(b.size());
        std::vector<size_t> all(b.size());
        for (size_t k = 0; k < b.size(); ++k) {
            q[k] = {graphs[b[k].q.graph_id].g, b[k].q.source, 0, b[k].q.out};
            all[k] = k;
        }
        run_isolated(q, all, status, [&](const sg_batch_query *qq, uint32_t n) {
            return sg_sssp_batch(ctx, qq, n, &o, nullptr, nullptr);
        });
    } else if (algo == SG_QUERY_PAGERANK) {
        // PageRank has no source: one run per graph answers all its queries
        std::map<uint32_t, std::vector<size_t>> by_graph;
        for (size_t i = 0; i < b.size(); ++i) by_graph[b[i].q.graph_id].push_back(i);
        for (auto &kv : by_graph) {
            GraphInfo &gi = graphs[kv.first];
            std::vector<float> ranks(gi.nv);
            sg_graph *gv = view(slot, kv.first);
            const sg_status st = gv ? sg_pagerank(gv, &o, ranks.data(), nullptr, nullptr) : SG_ERR_OUT_OF_MEMORY;
            for (size_t i : kv.second) {
                status[i] = st;
                if (st == SG_OK) std::memcpy(b[i].q.out, ranks.data(), 4ull * gi.nv);
            }
        }
    } else {
        // BC: several queries on one graph -> multi-source BC (32 sources per
        // launch, each row straight to its query); the rest, and any group the
        // multi-source kernel declines (no in-edge view, path-count overflow),
        // -> one batched launch (forward and backward per team), which reports
        // per-query statuses; a query that also asks for path counts runs alone
        // through sg_bc
        std::vector<sg_batch_query> q;
        std::vector<size_t> in_batch;
        std::map<uint32_t, std::vector<size_t>> by_graph;
        for (size_t i = 0; i < b.size(); ++i) {
            if (b[i].q.out2) {
                sg_graph *gv = view(slot, b[i].q.graph_id);
                status[i] = gv ? sg_bc(gv, b[i].q.source, &o, (float *)b[i].q.out, (uint64_t *)b[i].q.out2, nullptr)
                               : SG_ERR_OUT_OF_MEMORY;
            } else {
                by_graph[b[i].q.graph_id].push_back(i);
            }
        }
        for (auto &kv : by_graph) {
            sg_graph *gv = kv.second.size() >= std::max(1u, cfg.msbfs_min) ? view(slot, kv.first) : nullptr;
            for (size_t s = 0; s < kv.second.size(); s += 32) {
                const size_t m = std::min<size_t>(32, kv.second.size() - s);
                bool ok = false;
                if (gv) {
                    std::vector<uint32_t> src(m);
                    std::vector<float *> rows(m);
                    for (size_t k = 0; k < m; ++k) {
                        src[k] = b[kv.second[s + k]].q.source;
                        rows[k] = (float *)b[kv.second[s + k]].q.out;
                    }
                    sg_options om = o;  // the multi-source launch sizes its own grid unless the config fixes it
                    om.blocks_per_sm = (int32_t)cfg.blocks_per_sm;
                    ok = sgb::msbc_rows(gv, src.data(), (uint32_t)m, &om, nullptr, rows.data(), nullptr) == SG_OK;
                }
                if (ok) continue;
                for (size_t k = 0; k < m; ++k) {
                    const size_t i = kv.second[s + k];
                    q.push_back({graphs[b[i].q.graph_id].g, b[i].q.source, 0, b[i].q.out});
                    in_batch.push_back(i);
                }
            }
        }
        if (!q.empty())
            run_isolated(q, in_batch, status, [&](const sg_batch_query *qq, uint32_t n) {
                return sg_bc_batch(ctx, qq, n, &o, nullptr, nullptr);
            });
    }
}

void sg_server::worker(int slot) {
    for (;;) {
        std::vector<Pending> batch;
        uint64_t est = 0;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return stop || !pending.empty(); });
            if (stop && pending.empty()) return;
            // the oldest request decides the algorithm; take its peers in arrival order.
            // BFS on a graph with enough pending queries is one multi-source launch of
            // that graph alone (up to 64 sources), and PageRank is one run per graph
            // for all its pending queries, so that other slots run the other graphs'
            // launches at the same time.
            int algo = pending.front().q.algo;
            uint32_t graph = pending.front().q.graph_id;
            const bool one_graph_batches = cfg.batch_graphs == SG_BATCH_ONE_GRAPH;
            if (one_graph_batches && cfg.order != SG_ORDER_OLDEST_FIRST) {
                // shortest expected batch first: the group whose batches have run
                // shortest so far (a group never run yet counts as shortest, which
                // also measures it), so a small query does not queue behind large
                // graphs' traversals; a query older than max_wait_ms goes first
                const double max_wait = cfg.max_wait_ms ? (double)cfg.max_wait_ms : 500.0;
                const double waited =
                    std::chrono::duration<double, std::milli>(Clock::now() - pending.front().t_submit).count();
                if (waited <= max_wait) {
                    double best = -1;
                    for (auto &p : pending) {
                        auto it = group_ms.find({p.q.algo, p.q.graph_id});
                        const double c = it == group_ms.end() ? 0.0 : it->second;
                        if (best < 0 || c < best) {
                            best = c;
                            algo = p.q.algo;
                            graph = p.q.graph_id;
                            if (c == 0.0) break;
                        }
                    }
                }
            }
            uint32_t cap = cfg.max_batch;
            // one graph per batch (SG_BATCH_ONE_GRAPH): a batch lasts as long as its
            // slowest query, so a query on a small graph batched with a large
            // graph's traversal would wait for it; mixed batches (default) run
            // more queries per launch
            bool one_graph = algo == SG_QUERY_PAGERANK || one_graph_batches;
            if (algo == SG_QUERY_BFS) {
                uint32_t same = 0;
                for (auto &p : pending)
                    if (p.q.algo == algo && p.q.graph_id == graph && ++same >= std::max(1u, cfg.msbfs_min)) break;
                if (same >= std::max(1u, cfg.msbfs_min)) {
                    one_graph = true;
                    cap = std::min(cap, 64u);
                }
            }
            for (auto it = pending.begin(); it != pending.end() && batch.size() < cap;) {
                if (it->q.algo == algo && (!one_graph || it->q.graph_id == graph)) {
                    batch.push_back(*it);
                    it = pending.erase(it);
                } else {
                    ++it;
                }
            }
            // admission against the HBM budget: shrink, or wait for other slots to release memory
            est = estimate(batch);
            while (in_use + est > budget && batch.size() > 1) {
                pending.push_front(batch.back());
                batch.pop_back();
                est = estimate(batch);
            }
            while (in_use > 0 && in_use + est > budget && !stop) cv_done.wait(lk);
            in_use += est;
            peak = std::max(peak, in_use);
            ++batches;
            if (!pending.empty()) cv_work.notify_one();
        }
        std::vector<sg_status> status;
        const auto t_run = Clock::now();
        run_batch(slot, batch, status);
        const auto now = Clock::now();
        if (log) {
            std::lock_guard<std::mutex> lk(log_mu);
            std::fprintf(log, "slot %d algo %d queries %zu est_bytes %llu ms %.3f\n", slot, batch.front().q.algo,
                         batch.size(), (unsigned long long)est,
                         std::chrono::duration<double, std::milli>(now - t_run).count());
            std::fflush(log);
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            in_use -= est;
            {  // the group's batch time, smoothed over its batches
                const double ms = std::chrono::duration<double, std::milli>(now - t_run).count();
                const auto key = std::make_pair(batch.front().q.algo, batch.front().q.graph_id);
                auto it = group_ms.find(key);
                group_ms[key] = it == group_ms.end() ? ms : 0.7 * it->second + 0.3 * ms;
            }
            for (size_t i = 0; i < batch.size(); ++i) {
                TicketState &t = tickets[batch[i].ticket];
                t.done = true;
                t.status = status[i];
                t.latency_ms = std::chrono::duration<double, std::milli>(now - batch[i].t_submit).count();
                latencies.push_back(t.latency_ms);
                ++completed;
                if (status[i] != SG_OK) ++failed;
            }
            t_last = now;
        }
        cv_done.notify_all();
    }
}

extern "C" {

sg_status sg_server_config_default(sg_server_config *c) {
    if (!c) return SG_ERR_INVALID_ARG;
    std::memset(c, 0, sizeof *c);
    c->slots = 2;
    c->max_batch = 256;
    c->max_pending = 1u << 20;
    c->msbfs_min = 4;
    c->sssp_delta = 0;
    c->pr_error = 1e-7;
    return SG_OK;
}

sg_status sg_server_create(int device, const sg_server_config *cfg, sg_server **out) {
    if (!out) return SG_ERR_INVALID_ARG;
    *out = nullptr;
    auto s = std::make_unique<sg_server>();
    s->device = device;
    s->graphs.reserve(kMaxGraphs);
    if (cfg)
        s->cfg = *cfg;
    else
        sg_server_config_default(&s->cfg);
    if (s->cfg.slots == 0) s->cfg.slots = 1;
    if (s->cfg.max_batch == 0) s->cfg.max_batch = 256;
    if (s->cfg.max_pending == 0) s->cfg.max_pending = 1u << 20;
    if (s->cfg.pr_error <= 0) s->cfg.pr_error = 1e-7;
    for (uint32_t k = 0; k < s->cfg.slots; ++k) {
        sg_ctx *c = nullptr;
        const sg_status st = sg_init(device, &c);
        if (st != SG_OK) {
            for (auto *x : s->slot_ctx) sg_destroy(x);
            return st;
        }
        // every slot's persistent grid fits beside the other slots' (a grid
        // that does not fit would wait for another slot's launch to end)
        sgb::set_resident_share(c, s->cfg.slots);
        s->slot_ctx.push_back(c);
    }
    uint64_t hbm = 0;
    sg_device_info(s->slot_ctx[0], nullptr, &hbm, nullptr, nullptr, 0);
    s->budget = s->cfg.hbm_budget_bytes ? s->cfg.hbm_budget_bytes : hbm / 4;
    s->views.resize(s->cfg.slots);
    if (const char *path = std::getenv("SEPGRAPH_SERVER_LOG")) s->log = std::fopen(path, "a");
    sg_server *raw = s.release();
    for (uint32_t k = 0; k < raw->cfg.slots; ++k) raw->workers.emplace_back([raw, k] { raw->worker((int)k); });
    *out = raw;
    return SG_OK;
}

sg_status sg_server_add_graph(sg_server *s, sg_graph *g, uint32_t *graph_id) {
    if (!s || !g || !graph_id) return SG_ERR_INVALID_ARG;
    uint32_t nv = 0;
    uint64_t ne = 0;
    sg_status st = sg_graph_info(g, &nv, &ne, nullptr, nullptr);
    if (st != SG_OK) return st;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->graphs.size() >= kMaxGraphs) return SG_ERR_BUSY;
    s->graphs.push_back({g, nv, ne});
    *graph_id = (uint32_t)s->graphs.size() - 1;
    return SG_OK;
}

sg_status sg_server_submit(sg_server *s, const sg_query *q, uint64_t *ticket) {
    if (!s || !q || !ticket || !q->out || q->algo < SG_QUERY_BFS || q->algo > SG_QUERY_BC) return SG_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (q->graph_id >= s->graphs.size()) return SG_ERR_INVALID_ARG;
        if (q->algo != SG_QUERY_PAGERANK && q->source >= s->graphs[q->graph_id].nv) return SG_ERR_INVALID_ARG;
        if (s->pending.size() >= s->cfg.max_pending) return SG_ERR_BUSY;
        const uint64_t t = s->next_ticket++;
        const auto now = Clock::now();
        if (!s->have_first) {
            s->have_first = true;
            s->t_first = now;
        }
        s->pending.push_back({t, *q, now});
        s->tickets[t] = TicketState{};
        ++s->submitted;
        *ticket = t;
    }
    s->cv_work.notify_one();
    return SG_OK;
}

sg_status sg_server_wait(sg_server *s, uint64_t ticket, double timeout_s, sg_status *result, double *latency_ms) {
    if (!s) return SG_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return SG_ERR_INVALID_ARG;
    const auto deadline = Clock::now() + std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 3600.0);
    if (!s->cv_done.wait_until(lk, deadline, [&] { return s->tickets[ticket].done; })) return SG_ERR_TIMEOUT;
    const TicketState t = s->tickets[ticket];
    s->tickets.erase(ticket);
    if (result) *result = t.status;
    if (latency_ms) *latency_ms = t.latency_ms;
    return SG_OK;
}

sg_status sg_server_drain(sg_server *s, double timeout_s) {
    if (!s) return SG_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    const auto deadline = Clock::now() + std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 3600.0);
    if (!s->cv_done.wait_until(lk, deadline, [&] { return s->completed == s->submitted; })) return SG_ERR_TIMEOUT;
    return SG_OK;
}

sg_status sg_server_get_stats(sg_server *s, sg_server_stats *st) {
    if (!s || !st) return SG_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(st, 0, sizeof *st);
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->failed = s->failed;
    st->batches = s->batches;
    st->pending = s->pending.size();
    st->hbm_budget = s->budget;
    st->hbm_in_use = s->in_use;
    st->hbm_peak = s->peak;
    if (s->have_first && s->completed)
        st->elapsed_s = std::chrono::duration<double>(s->t_last - s->t_first).count();
    if (st->elapsed_s > 0) st->qps = s->completed / st->elapsed_s;
    if (!s->latencies.empty()) {
        std::vector<double> l = s->latencies;
        std::sort(l.begin(), l.end());
        auto pct = [&](double p) { return l[std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5))]; };
        double sum = 0;
        for (double x : l) sum += x;
        st->mean_ms = sum / l.size();
        st->p50_ms = pct(0.50);
        st->p99_ms = pct(0.99);
        st->p999_ms = pct(0.999);
        st->max_ms = l.back();
    }
    return SG_OK;
}

sg_status sg_server_reset_stats(sg_server *s) {
    if (!s) return SG_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    s->latencies.clear();
    s->submitted -= s->completed;
    s->completed = s->failed = s->batches = 0;
    s->have_first = false;
    s->peak = s->in_use;
    return SG_OK;
}

sg_status sg_server_destroy(sg_server *s) {
    if (!s) return SG_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    for (auto &t : s->workers) t.join();
    for (auto &per_slot : s->views)
        for (sg_graph *v : per_slot) sgb::graph_view_destroy(v);
    for (auto *c : s->slot_ctx) sg_destroy(c);
    if (s->log) std::fclose(s->log);
    delete s;
    return SG_OK;
}

}  // extern "C"
