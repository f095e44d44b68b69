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

// Multi-source BC (<= 32 sources) with row i written to row_outs[i] (host or
// device, nv floats each) when row_outs is given, else to bc_out.
sg_status msbc_rows(sg_graph *g, const uint32_t *sources, uint32_t nsrc, const sg_options *opt, float *bc_out,
                    float *const *row_outs, sg_stats *stats);
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
// Number of contexts (ctx among them) whose persistent launches run side by
// side; each launch on ctx then takes at most that share of a kernel's
// resident blocks per SM (1, the default, lets a launch fill the device).
void set_resident_share(sg_ctx *ctx, uint32_t share);

// Device graph from a CSR (host or device arrays): one upload, validation on
// the device, and the in-edge (CSC) view from the device transpose.
sg_status create_graph(sg_ctx *ctx, uint32_t nv, uint64_t ne, const uint32_t *offsets, const uint32_t *indices,
                       const uint32_t *weights, uint32_t flags, sg_graph **out);
// CSR -> CSC on the device (all pointers device memory), ordered as csr_tocsc
// orders it: by source, parallel edges by CSR position.
sg_status device_transpose(sg_ctx *ctx, uint32_t nv, uint64_t ne, const uint32_t *row, const uint32_t *col,
                           const uint32_t *w, uint32_t *crow, uint32_t *ccol, uint32_t *cw);
// In-edge view of a symmetric weighted graph: the CSR alias where the
// transpose is identical, else its own weights or a full CSC.
sg_status symmetric_weighted_csc(sg_ctx *ctx, sg_graph *g);

}  // namespace sgb
