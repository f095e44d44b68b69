"""GPU parity at scales 20-21 and on a 1024x1024 grid, through the C ABI,
against the oracle: hubs of 10^4-10^5 edges, chunk tables far from empty,
hundreds of delta-stepping rounds.

Tolerances as in test_gpu_parity.py:
  BFS levels, SSSP distances: bit-exact (SSSP against the oracle's Dijkstra,
            which returns SSSPHostNaive's distances: they are unique).
  PageRank: L1 of L1-normalised vectors <= 1e-6 against the FP64 fixed point
            of PageRankHost.
  BC: |gpu - fp64| <= 1e-4 * |fp64| + 1e-5 per vertex; path counts exact.
"""
import numpy as np
import pytest

import oracle
import sepgraph as sg

pytestmark = pytest.mark.gpu

PR_L1_TOL = 1e-6
BC_RTOL, BC_ATOL = 1e-4, 1e-5


@pytest.fixture(scope="module")
def ctx():
    c = sg.Context(0)
    yield c
    c.close()


def _pr_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a / a.sum() - b / b.sum()).sum()


@pytest.mark.parametrize("scale,sym", [(21, True), (20, False)])
def test_bfs_large(ctx, scale, sym):
    h = sg.HostGraph.rmat(scale, 16, symmetric=sym, seed=1)
    G = ctx.graph(h, symmetric=sym)
    for src in [h.max_degree_vertex()[0]] + [int(s) for s in h.pick_sources(2, 3)]:
        ref = oracle.bfs(h.offsets, h.indices, int(src))
        for kw in (dict(), dict(variant="async_push_dd"), dict(variant="async_push_dd", local_depth=16),
                   dict(variant="async_pull_dd")):
            lv, st, _ = G.bfs(int(src), max_iteration=100000, **kw)
            assert (lv == ref).all(), (kw, src)
    G.close()


def test_sssp_rmat21(ctx):
    h = sg.HostGraph.rmat(21, 16, seed=1).gen_weights(1, 64, 2)
    G = ctx.graph(h)
    for src in (int(s) for s in h.pick_sources(2, 3)):
        ref = oracle.dijkstra(h.offsets, h.indices, h.weights, src)
        for kw in (dict(variant="async_push_dd"),
                   dict(variant="async_push_dd", priority="low_high", priority_delta=4, local_depth=16,
                        blocks_per_sm=4, chunk_edges=64),
                   dict(variant="async_push_dd", priority="low_high", priority_delta=8, worklist=2,
                        chunk_edges=256),
                   dict(variant="async_push_dd", worklist=2, chunk_edges=1024, heavy_degree=64),
                   dict(variant="async_push_dd", priority="low_high", priority_delta=8, chunk_edges=256,
                        hub_stage=1),
                   dict(variant="async_push_dd", priority="low_high", priority_delta=8, chunk_edges=256,
                        hub_stage=-1),
                   dict(priority="low_high"), dict()):
            d, st, _ = G.sssp(src, max_iteration=1000000, **kw)
            assert (d == ref).all(), kw
    G.close()


def test_sssp_grid1024(ctx):
    h = sg.HostGraph.grid(1024, 1024).gen_weights(1, 1000, 2)
    G = ctx.graph(h, no_csc=True)
    for src in (0, int(h.pick_sources(1, 5)[0])):
        ref = oracle.dijkstra(h.offsets, h.indices, h.weights, src)
        for kw in (dict(variant="async_push_dd", priority="low_high", priority_delta=4001, local_depth=16,
                        blocks_per_sm=1),
                   dict(variant="async_push_dd", priority="low_high")):
            d, st, _ = G.sssp(src, max_iteration=10000000, **kw)
            assert (d == ref).all(), kw
            assert st.rounds > 100
    G.close()


@pytest.mark.parametrize("variant", ["sync_pull_td", "async_push_dd", "auto"])
def test_pagerank_rmat20(ctx, variant):
    h = sg.HostGraph.rmat(20, 16, seed=1)
    G = ctx.graph(h)
    ref64, _ = oracle.pagerank_fixed_point_f64(h.offsets, h.indices, 1e-13)
    r, st, _ = G.pagerank(variant=variant, pr_error=1e-7, max_iteration=100000)
    assert _pr_l1(r, ref64) <= PR_L1_TOL, (variant, _pr_l1(r, ref64))
    G.close()


def test_bc_rmat20(ctx):
    h = sg.HostGraph.rmat(20, 16, symmetric=True, seed=1)
    G = ctx.graph(h, symmetric=True)
    for src in [h.max_degree_vertex()[0], int(h.pick_sources(1, 3)[0])]:
        bc, sigma, st = G.bc(int(src))
        bc64, sig64, _ = oracle.bc_f64(h.offsets, h.indices, int(src))
        assert (sigma.astype(np.float64) == sig64).all()
        assert np.all(np.abs(bc - bc64) <= BC_RTOL * np.abs(bc64) + BC_ATOL), np.max(np.abs(bc - bc64))
    G.close()
