// Library-internal entry points shared between the CUDA translation units and
// the host-only server (plain C++, no device code).
#pragma once
#include <cstdint>

#include "../../include/sepgraph.h"

namespace sgb {

// Multi-source BFS on a chosen context (its stream and scratch).  Levels go to
// levels_out (nsrc rows of nv, host or device) or, when row_outs is given, row
// i to row_outs[i] (host or device, nv uint32 each).
sg_status msbfs_on(sg_ctx *ctx, sg_graph *g, const uint32_t *sources, uint32_t nsrc, const sg_options *opt,
                   uint32_t *levels_out, sg_stats *stats, uint32_t *const *row_outs = nullptr);

// The context a graph was created on.
sg_ctx *graph_context(const sg_graph *g);
// Sum of the graph's edge weights (its edge count when unweighted).
double graph_weight_sum(const sg_graph *g);
// A view of g's device arrays bound to another context of the same device:
// single-query calls on the view run on that context's stream with that
// context's scratch.  The view must be released with graph_view_destroy
// before g is destroyed.
sg_graph *graph_view(sg_graph *g, sg_ctx *ctx);
void graph_view_destroy(sg_graph *view);

}  // namespace sgb
