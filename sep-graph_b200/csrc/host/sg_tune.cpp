// Autotuner over engine options (declaration and contract in
// include/sepgraph.h, "autotuner").  Host code over the public entry points:
// every candidate runs the real engine on the caller's graph and sources and
// must reproduce the first candidate's result before its time counts.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../../include/sepgraph.h"
#include "../sg_internal.h"

namespace {

// Candidate modes of an algorithm (variant, and for SSSP the two-level priority
// delta around the reference heuristic 32*avg_w/avg_deg, hybrid_sssp.cu:196-197).
std::vector<sg_options> modes(sg_graph *g, int algo, const sg_options &base) {
    std::vector<sg_options> out;
    auto add = [&](int variant, int priority, double delta) {
        sg_options o = base;
        o.variant = variant;
        o.priority = priority;
        o.priority_delta = delta;
        o.blocking = 1;
        out.push_back(o);
    };
    if (algo == SG_QUERY_BFS || algo == SG_QUERY_BC) {
        add(SG_VARIANT_AUTO, SG_PRIORITY_NONE, 0);
        add(SG_ASYNC_PUSH_DD, SG_PRIORITY_NONE, 0);
    } else if (algo == SG_QUERY_SSSP) {
        uint32_t nv = 0;
        uint64_t ne = 0;
        sg_graph_info(g, &nv, &ne, nullptr, nullptr);
        const double avg_w = ne ? sgb::graph_weight_sum(g) / (double)ne : 1.0;
        const double avg_deg = nv ? (double)ne / nv : 1.0;
        const double heuristic = std::max(1.0, std::floor(32.0 * avg_w / std::max(avg_deg, 1e-9)));
        add(SG_VARIANT_AUTO, SG_PRIORITY_NONE, 0);
        add(SG_ASYNC_PUSH_DD, SG_PRIORITY_NONE, 0);
        for (double f : {1.0 / 16, 1.0 / 4, 1.0, 4.0})
            add(SG_ASYNC_PUSH_DD, SG_PRIORITY_LOW_HIGH, std::max(1.0, std::floor(heuristic * f)));
    } else {
        add(SG_VARIANT_AUTO, SG_PRIORITY_NONE, 0);
        add(SG_SYNC_PULL_TD, SG_PRIORITY_NONE, 0);
        add(SG_ASYNC_PUSH_DD, SG_PRIORITY_NONE, 0);
    }
    return out;
}

struct Result {
    std::vector<uint32_t> u;
    std::vector<float> f;
};

sg_status run_one(sg_graph *g, int algo, uint32_t src, const sg_options &o, uint32_t nv, Result &r, double *ms) {
    sg_stats st;
    std::memset(&st, 0, sizeof st);
    sg_status s;
    if (algo == SG_QUERY_BFS || algo == SG_QUERY_SSSP) {
        r.u.resize(nv);
        s = algo == SG_QUERY_BFS ? sg_bfs(g, src, &o, r.u.data(), &st) : sg_sssp(g, src, &o, r.u.data(), &st);
        *ms = st.time_kernel_ms;
    } else if (algo == SG_QUERY_PAGERANK) {
        r.f.resize(nv);
        s = sg_pagerank(g, &o, r.f.data(), nullptr, &st);
        *ms = st.time_kernel_ms;
    } else {
        r.f.resize(nv);
        s = sg_bc(g, src, &o, r.f.data(), nullptr, &st);
        *ms = st.time_total_ms;
    }
    if (s == SG_OK && st.max_iteration_reached) s = SG_ERR_CAPACITY;  // an unfinished run is not a result
    return s;
}

// Same result within the algorithm's tolerance: BFS/SSSP exact; PageRank L1 of
// the L1-normalised vectors within max(1e-6, 20 * residual threshold); BC 1e-4
// relative + 1e-5 absolute.
bool same(int algo, const Result &a, const Result &b, double pr_error) {
    if (algo == SG_QUERY_BFS || algo == SG_QUERY_SSSP) return a.u == b.u;
    if (a.f.size() != b.f.size()) return false;
    if (algo == SG_QUERY_PAGERANK) {
        double sa = 0, sb = 0, l1 = 0;
        for (size_t i = 0; i < a.f.size(); ++i) {
            sa += a.f[i];
            sb += b.f[i];
        }
        if (sa <= 0 || sb <= 0) return false;
        for (size_t i = 0; i < a.f.size(); ++i) l1 += std::fabs(a.f[i] / sa - b.f[i] / sb);
        return l1 <= std::max(1e-6, 20.0 * pr_error);
    }
    for (size_t i = 0; i < a.f.size(); ++i)
        if (std::fabs((double)a.f[i] - b.f[i]) > 1e-5 + 1e-4 * std::fabs((double)b.f[i])) return false;
    return true;
}

}  // namespace

// Staged search: the mode first, then, keeping the best so far, blocks per
// SM, a finer two-level delta, push load balancing, local lookahead depth
// (BFS/SSSP), the heavy-vertex split threshold and the chunk size of split
// vertices.  Every candidate must reproduce the first
// candidate's result before its time counts.
extern "C" sg_status sg_autotune(sg_graph *g, int algo, const uint32_t *sources, uint32_t nsrc, const sg_options *base,
                                 uint32_t max_candidates, sg_options *best, double *best_ms, sg_tune_entry *report,
                                 uint32_t report_capacity, uint32_t *n_report) {
    if (!g || !best || algo < SG_QUERY_BFS || algo > SG_QUERY_BC) return SG_ERR_INVALID_ARG;
    uint32_t nv = 0;
    uint64_t ne = 0;
    sg_status st = sg_graph_info(g, &nv, &ne, nullptr, nullptr);
    if (st != SG_OK) return st;
    const bool sourceless = algo == SG_QUERY_PAGERANK;
    if (!sourceless && (!sources || nsrc == 0)) return SG_ERR_INVALID_ARG;
    for (uint32_t i = 0; !sourceless && i < nsrc; ++i)
        if (sources[i] >= nv) return SG_ERR_INVALID_ARG;
    sg_options b0;
    if (base)
        b0 = *base;
    else
        sg_options_default(&b0);
    const uint32_t runs = sourceless ? 1u : nsrc;
    const uint32_t limit = max_candidates ? max_candidates : 64u;
    std::vector<Result> ref(runs);
    bool have_ref = false;
    double best_t = -1;
    uint32_t tried = 0;
    if (n_report) *n_report = 0;

    // times one candidate; returns its median ms or -1 when it failed or differed
    auto trial = [&](const sg_options &cand) -> double {
        if (tried >= limit) return -1;
        ++tried;
        std::vector<double> ts;
        sg_status cs = SG_OK;
        std::vector<Result> res(runs);
        for (uint32_t k = 0; k < runs && cs == SG_OK; ++k) {
            double ms = 0;
            cs = run_one(g, algo, sourceless ? 0u : sources[k], cand, nv, res[k], &ms);
            ts.push_back(ms);
        }
        if (cs == SG_OK) {
            if (!have_ref) {
                ref = res;
                have_ref = true;
            } else {
                for (uint32_t k = 0; k < runs; ++k)
                    if (!same(algo, res[k], ref[k], b0.pr_error)) cs = SG_ERR_FORMAT;
            }
        }
        double med = 0;
        if (!ts.empty()) {
            std::sort(ts.begin(), ts.end());
            med = ts[ts.size() / 2];
        }
        if (report && n_report && *n_report < report_capacity) {
            sg_tune_entry &e = report[(*n_report)++];
            e.options = cand;
            e.ms = med;
            e.status = cs;
            e.pad = 0;
        }
        if (cs != SG_OK) return -1;
        if (best_t < 0 || med < best_t) {
            best_t = med;
            *best = cand;
        }
        return med;
    };

    for (const sg_options &m : modes(g, algo, b0)) trial(m);
    if (best_t < 0) return SG_ERR_UNSUPPORTED;  // no candidate finished
    const bool push_mode = best->variant == SG_VARIANT_AUTO || best->variant == SG_ASYNC_PUSH_DD;
    {
        const sg_options cur = *best;
        for (int b : {1, 2, 3, 4, 8}) {
            sg_options c = cur;
            c.blocks_per_sm = b;
            trial(c);
        }
    }
    if (best->priority == SG_PRIORITY_LOW_HIGH && best->priority_delta > 0) {
        // refine the two-level delta around the coarse grid's pick: half and
        // double, then one more step in the direction that helped (SSSP on
        // RMAT-22: the grid's 4 -> 3.99 ms, 8 -> 3.86 ms per source)
        const sg_options cur = *best;
        const double d0 = cur.priority_delta;
        for (double f : {0.5, 2.0}) {
            sg_options c = cur;
            c.priority_delta = std::max(1.0, std::floor(d0 * f));
            if (c.priority_delta != d0) trial(c);
        }
        const double d1 = best->priority_delta;
        if (d1 != d0) {
            sg_options c = *best;
            c.priority_delta = std::max(1.0, std::floor(d1 * (d1 > d0 ? 2.0 : 0.5)));
            if (c.priority_delta != d1) trial(c);
        }
    }
    if (push_mode && algo != SG_QUERY_PAGERANK) {
        const sg_options cur = *best;
        const double avg_deg = nv ? (double)ne / nv : 0;
        sg_options c = cur;  // the other of the two load-balancing modes the automatic rule picks from
        c.lb_push = avg_deg >= 5 ? SG_LB_NONE : SG_LB_FINE_GRAINED;
        trial(c);
    }
    if (push_mode && (algo == SG_QUERY_BFS || algo == SG_QUERY_SSSP)) {
        const sg_options cur = *best;
        for (int d : {4, 16}) {
            sg_options c = cur;
            c.local_depth = d;
            c.variant = SG_ASYNC_PUSH_DD;  // the engine follows discoveries under forced push only
            trial(c);
        }
    }
    if (push_mode && algo != SG_QUERY_PAGERANK) {
        const sg_options cur = *best;
        sg_options c = cur;
        c.heavy_degree = 128;
        trial(c);
    }
    if (push_mode && algo != SG_QUERY_PAGERANK) {
        // edges per chunk of a split vertex: smaller chunks spread a hub's
        // first relaxations over more warps, larger ones give each lane more
        // edges in flight (SSSP on RMAT-22 with 8 edges per lane per step:
        // 256 -> 2.50 ms, 512 -> 2.60 per source)
        const sg_options cur = *best;
        for (int ce : {64, 128, 512}) {
            sg_options c = cur;
            c.chunk_edges = ce;
            trial(c);
        }
    }
    if (best->variant == SG_VARIANT_AUTO || best->variant == SG_ASYNC_PULL_DD) {
        // the two forms of the data-driven pull into small in-degree vertices
        sg_options c = *best;
        c.pull_scan = best->pull_scan == SG_PULL_SCAN_WARP ? SG_PULL_SCAN_THREAD : SG_PULL_SCAN_WARP;
        trial(c);
    }
    if (best->variant == SG_ASYNC_PUSH_DD && best->lb_push != SG_LB_NONE && !best->wl_sort) {
        // the two worklist kinds of a forced data-driven push
        const sg_options cur = *best;
        sg_options c = cur;
        c.worklist = cur.worklist == SG_WORKLIST_BITMAP ? SG_WORKLIST_QUEUE : SG_WORKLIST_BITMAP;
        trial(c);
    }
    if (best_ms) *best_ms = best_t;
    return SG_OK;
}
