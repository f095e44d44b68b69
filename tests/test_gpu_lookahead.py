"""Local lookahead (sg_options.local_depth): a block follows its own
discoveries for a few levels inside a push round.  Results must stay
bit-exact for BFS levels and SSSP distances whatever the depth, variant,
priority or load-balancing mode, including graphs with heavy vertices."""
import glob
import os

import numpy as np
import pytest

import oracle
import sepgraph as sg

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.fixture(scope="module")
def ctx():
    c = sg.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_lookahead_golden(ctx, path):
    z = np.load(path)
    G = ctx.graph_from_csr(z["offsets"], z["indices"], z["weights"])
    src = int(z["source"])
    for depth in (1, 4, 32):
        for kw in (dict(), dict(variant="async_push_dd"), dict(variant="async_push_dd", lb_push="none"),
                   dict(priority="low_high", priority_delta=8)):
            lv, _, _ = G.bfs(src, local_depth=depth, max_iteration=100000, **kw)
            assert (lv == z["bfs"]).all(), (depth, kw)
            d, _, _ = G.sssp(src, local_depth=depth, max_iteration=1000000, **kw)
            assert (d == z["sssp"]).all(), (depth, kw)


@pytest.mark.parametrize("kind", ["rmat_dir", "rmat_sym", "grid"])
def test_lookahead_large(ctx, kind):
    if kind == "grid":
        h = sg.HostGraph.grid(300, 200).gen_weights(1, 1000, 3)
        sym = False
    else:
        sym = kind == "rmat_sym"
        h = sg.HostGraph.rmat(15, 16, symmetric=sym, seed=6).gen_weights(1, 64, 7)
    G = ctx.graph(h, symmetric=sym)
    for src in (int(s) for s in h.pick_sources(2, 8)):
        want_b = oracle.bfs(h.offsets, h.indices, src)
        want_d = oracle.sssp(h.offsets, h.indices, h.weights, src)
        for depth in (2, 8):
            for kw in (dict(), dict(variant="async_push_dd"), dict(priority="low_high"),
                       dict(variant="async_push_dd", lb_push="fine")):
                lv, st, _ = G.bfs(src, local_depth=depth, max_iteration=1000000, **kw)
                assert (lv == want_b).all(), (depth, kw)
                assert st.device_error == 0
                d, st, _ = G.sssp(src, local_depth=depth, max_iteration=1000000, **kw)
                assert (d == want_d).all(), (depth, kw)


def test_lookahead_in_batches(ctx):
    graphs = []
    for k, (scale, sym) in enumerate([(9, False), (11, True), (12, False)]):
        h = sg.HostGraph.rmat(scale, 16, symmetric=sym, seed=40 + k).gen_weights(1, 64, 50 + k)
        graphs.append((h, ctx.graph(h, symmetric=sym)))
    h = sg.HostGraph.grid(64, 50).gen_weights(1, 64, 9)
    graphs.append((h, ctx.graph(h)))
    queries, hosts = [], []
    for k in range(16):
        h, G = graphs[k % len(graphs)]
        queries.append((G, int(h.pick_sources(1, 90 + k)[0])))
        hosts.append(h)
    outs, st, _ = ctx.sssp_batch(queries, local_depth=4, variant="async_push_dd", max_iteration=1000000)
    for (G, s), h, o in zip(queries, hosts, outs):
        assert (o == oracle.sssp(h.offsets, h.indices, h.weights, s)).all()
    outs, st, _ = ctx.bfs_batch(queries, local_depth=4, max_iteration=1000000)
    for (G, s), h, o in zip(queries, hosts, outs):
        assert (o == oracle.bfs(h.offsets, h.indices, s)).all()
