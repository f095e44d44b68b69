"""Batched execution parity: every row of a multi-source BFS equals the
single-source oracle BFS from that source, bit for bit, whatever the batch
size, direction policy, duplicates or graph shape."""
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
def test_msbfs_golden(ctx, path):
    z = np.load(path)
    off, idx = z["offsets"], z["indices"]
    nv = len(off) - 1
    G = ctx.graph_from_csr(off, idx)
    srcs = np.arange(min(nv, 64), dtype=np.uint32)
    for variant in ("auto", "async_push_dd", "async_pull_dd"):
        lv, st = G.msbfs(srcs, variant=variant)
        for i, s in enumerate(srcs):
            assert (lv[i] == oracle.bfs(off, idx, int(s))).all(), (variant, s)


@pytest.mark.parametrize("scale,sym,n", [(14, True, 64), (15, False, 33), (16, True, 1), (16, True, 64)])
def test_msbfs_rmat(ctx, scale, sym, n):
    h = sg.HostGraph.rmat(scale, 16, symmetric=sym, seed=2)
    G = ctx.graph(h, symmetric=sym)
    srcs = h.pick_sources(n, 5)
    srcs[-1] = srcs[0]  # a duplicate source
    for variant in ("auto", "async_push_dd", "async_pull_dd"):
        lv, st = G.msbfs(srcs, variant=variant)
        for i in range(n):
            assert (lv[i] == oracle.bfs(h.offsets, h.indices, int(srcs[i]))).all(), (variant, i)
    deg = np.diff(h.offsets.astype(np.int64))
    reached = sum(int(deg[row != sg.INF].sum()) for row in lv)
    assert st.edges_reached == reached


def test_msbfs_matches_single_source_engine(ctx):
    h = sg.HostGraph.grid(64, 80)
    G = ctx.graph(h)
    srcs = np.array([0, 5119, 2500, 77], np.uint32)
    lv, st = G.msbfs(srcs, max_iteration=100000)
    for i, s in enumerate(srcs):
        single, _, _ = G.bfs(int(s), max_iteration=100000)
        assert (lv[i] == single).all()


def _csr(nv, src, dst):
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    off = np.zeros(nv + 1, np.uint32)
    np.add.at(off, src.astype(np.int64) + 1, 1)
    return np.cumsum(off, dtype=np.uint64).astype(np.uint32), dst.astype(np.uint32)


def test_msbfs_sparse_push_only_with_a_hub(ctx):
    """Sparse graphs (average degree below 8) run the one-barrier push-only
    kernel; a vertex of 1,500 out-edges there is expanded by a whole warp.
    Every row equals the oracle; forced pull (two-phase kernel) agrees."""
    w, hgt = 40, 50
    nv = w * hgt + 1
    hub = nv - 1
    src, dst = [], []
    for y in range(hgt):
        for x in range(w):
            v = y * w + x
            for dx, dy in ((1, 0), (-1, 0), (0, 1), (0, -1)):
                if 0 <= x + dx < w and 0 <= y + dy < hgt:
                    src.append(v)
                    dst.append((y + dy) * w + x + dx)
    rng = np.random.default_rng(3)
    far = rng.choice(nv - 1, 1500, replace=False)
    src += [hub] * len(far) + [0]
    dst += list(far) + [hub]
    off, idx = _csr(nv, np.array(src, np.int64), np.array(dst, np.int64))
    G = ctx.graph_from_csr(off, idx)
    srcs = np.array([0, hub, 777, 1999, 0], np.uint32)
    want = [oracle.bfs(off, idx, int(s)) for s in srcs]
    for variant in ("auto", "async_push_dd", "async_pull_dd"):
        lv, st = G.msbfs(srcs, variant=variant, max_iteration=100000)
        for i in range(len(srcs)):
            assert (lv[i] == want[i]).all(), (variant, i)


@pytest.mark.parametrize("max_iteration", [1, 7, 40])
def test_msbfs_max_iteration_truncates_alike(ctx, max_iteration):
    """With a round limit, both kernels settle exactly the levels up to it."""
    h = sg.HostGraph.grid(64, 80)
    G = ctx.graph(h)
    srcs = np.array([0, 5119, 2500, 77], np.uint32)
    fused, st_f = G.msbfs(srcs, max_iteration=max_iteration)
    pulled, st_p = G.msbfs(srcs, variant="async_pull_dd", max_iteration=max_iteration)
    assert (fused == pulled).all()
    for i, s in enumerate(srcs):
        full = oracle.bfs(h.offsets, h.indices, int(s))
        want = np.where(full <= max_iteration, full, full.dtype.type(sg.INF))
        assert (fused[i] == want).all(), i
    assert st_f.max_iteration_reached == st_p.max_iteration_reached


@pytest.fixture(scope="module")
def uneven_graphs(ctx):
    """Graphs of uneven size (RMAT scales 8-14, directed and symmetric, a grid), weights in [1,64)."""
    out = []
    for k, (scale, sym) in enumerate([(8, False), (10, True), (12, False), (13, True), (14, False), (11, False)]):
        h = sg.HostGraph.rmat(scale, 16, symmetric=sym, seed=10 + k).gen_weights(1, 64, 3 + k)
        out.append((h, ctx.graph(h, symmetric=sym)))
    h = sg.HostGraph.grid(40, 50).gen_weights(1, 64, 99)
    out.append((h, ctx.graph(h)))
    return out


@pytest.mark.parametrize("team_blocks", [0, 1, 8])
def test_sssp_batch_uneven_graphs(ctx, uneven_graphs, team_blocks):
    queries, refs = [], []
    for k in range(40):
        h, G = uneven_graphs[k % len(uneven_graphs)]
        s = int(h.pick_sources(1, 100 + k)[0])
        queries.append((G, s))
        refs.append(oracle.sssp(h.offsets, h.indices, h.weights, s))
    for kw in (dict(max_iteration=100000), dict(priority="low_high", max_iteration=1000000),
               dict(variant="async_push_dd", max_iteration=100000)):
        outs, st, per = ctx.sssp_batch(queries, team_blocks=team_blocks, **kw)
        for i, (o, r) in enumerate(zip(outs, refs)):
            assert (o == r).all(), (kw, i)
        assert st.edges_reached == sum(int(np.diff(h.offsets.astype(np.int64))[r != sg.INF].sum())
                                       for (h, _), r in zip([uneven_graphs[k % len(uneven_graphs)] for k in range(40)],
                                                            refs))
        assert all(p >= 0 for p in per)


def test_bfs_batch_matches_single(ctx, uneven_graphs):
    queries = [(G, int(h.pick_sources(1, k)[0])) for k, (h, G) in enumerate(uneven_graphs)] * 3
    torch = pytest.importorskip("torch")
    outs = [torch.empty(G.nv, dtype=torch.int32, device="cuda") for G, _ in queries]  # device outputs
    outs, st, _ = ctx.bfs_batch(queries, outs=outs)
    ctx.synchronize()
    for (G, s), o in zip(queries, outs):
        single, _, _ = G.bfs(s)
        assert (o.cpu().numpy().view(np.uint32) == single).all()


def test_msbfs_rejects_bad_batches(ctx):
    h = sg.HostGraph.rmat(10, 8, seed=1)
    G = ctx.graph(h)
    with pytest.raises(sg.SGError):
        G.msbfs(np.arange(65, dtype=np.uint32))
    with pytest.raises(sg.SGError):
        G.msbfs(np.array([h.nv], np.uint32))


@pytest.mark.parametrize("team_blocks", [0, 2])
def test_bc_batch_matches_single_and_oracle(ctx, team_blocks):
    """Batched BC over uneven graphs (unweighted view): each output equals sg_bc
    from that source within 1e-4 relative, and the FP64 oracle on small graphs."""
    specs = [("rmat", 9, True, 1), ("rmat", 11, True, 2), ("grid", (20, 30), False, 3), ("rmat", 12, False, 4)]
    graphs = []
    for kind, p, sym, seed in specs:
        h = sg.HostGraph.rmat(p, 8, symmetric=sym, seed=seed) if kind == "rmat" else sg.HostGraph.grid(*p)
        graphs.append((h, ctx.graph(h, symmetric=sym)))
    queries, hosts = [], []
    for k in range(18):
        h, G = graphs[k % len(graphs)]
        queries.append((G, int(h.pick_sources(1, 50 + k)[0])))
        hosts.append(h)
    queries.append((graphs[0][1], queries[0][1]))  # the same query twice in one batch
    hosts.append(graphs[0][0])
    outs, st, per = ctx.bc_batch(queries, team_blocks=team_blocks, max_iteration=100000)
    assert st.device_error == 0 and all(p >= 0 for p in per)
    for (G, s), h, o in zip(queries, hosts, outs):
        single, _, _ = G.bc(s, max_iteration=100000)
        assert np.allclose(o, single, rtol=1e-4, atol=1e-5), s
        if h.nv <= 1024:
            want, _, _ = oracle.bc_f64(h.offsets, h.indices, s)
            assert np.allclose(o, want, rtol=1e-4, atol=1e-4), s


@pytest.mark.parametrize("algo", ["sssp", "bfs", "bc"])
def test_batch_plan_replays_match_direct_batch(ctx, uneven_graphs, algo):
    """A planned batch launched three times gives the direct batch's outputs every time."""
    torch = pytest.importorskip("torch")
    queries = [(G, int(h.pick_sources(1, 70 + k)[0])) for k, (h, G) in enumerate(uneven_graphs)] * 2
    kw = dict(max_iteration=100000)
    if algo == "sssp":
        want, _, _ = ctx.sssp_batch(queries, **kw)
    elif algo == "bfs":
        want, _, _ = ctx.bfs_batch(queries, **kw)
    else:
        want, _, _ = ctx.bc_batch(queries, **kw)
    dt = torch.float32 if algo == "bc" else torch.int32
    outs = [torch.zeros(G.nv, dtype=dt, device="cuda") for G, _ in queries]
    plan = ctx.batch_plan(algo, queries, outs, **kw)
    for rep in range(3):
        for o in outs:
            o.zero_()
        torch.cuda.synchronize()  # the zeroing (torch's stream) precedes the plan's launch (the context's stream)
        plan.launch()
        st, per = plan.wait()
        assert st.device_error == 0 and len(per) == len(queries)
        for o, w in zip(outs, want):
            got = o.cpu().numpy()
            if algo == "bc":
                assert np.allclose(got, w, rtol=1e-4, atol=1e-5), rep
            else:
                assert (got.view(np.uint32) == w).all(), rep
    plan.close()


def test_batch_plan_rejects_host_outputs(ctx, uneven_graphs):
    h, G = uneven_graphs[0]
    with pytest.raises(sg.SGError):
        ctx.batch_plan("bfs", [(G, 0)], [np.zeros(h.nv, np.uint32)])


def _msbc_case(ctx, h, srcs, sym):
    G = ctx.graph(h, symmetric=sym)
    try:
        rows, st = G.msbc(srcs, max_iteration=1000000)
        assert st.device_error == 0
        for i, s in enumerate(srcs):
            single, _, _ = G.bc(int(s), max_iteration=1000000)
            assert np.allclose(rows[i], single, rtol=1e-4, atol=1e-5), (i, s)
            if h.nv <= 2048:
                want, _, _ = oracle.bc_f64(h.offsets, h.indices, int(s))
                assert np.allclose(rows[i], want, rtol=1e-4, atol=1e-4), (i, s)
    finally:
        G.close()


@pytest.mark.parametrize("scale,sym,n", [(10, True, 32), (12, False, 32), (13, True, 7), (14, True, 1)])
def test_msbc_rmat_matches_single(ctx, scale, sym, n):
    """Each row of multi-source BC equals sg_bc from that source (1e-4 relative)
    and the FP64 oracle on small graphs; directed graphs pull over the CSC."""
    h = sg.HostGraph.rmat(scale, 8, symmetric=sym, seed=scale)
    srcs = [int(s) for s in h.pick_sources(n, 70 + scale)]
    _msbc_case(ctx, h, srcs, sym)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_msbc_golden(ctx, path):
    """Small shapes (chain, star, grid, disconnected, self-loops and duplicate
    edges, single vertex) with every vertex as a source (up to 32), duplicates
    included."""
    z = np.load(path)
    h = sg.HostGraph.from_csr(z["offsets"], z["indices"])
    srcs = [v % h.nv for v in range(min(32, h.nv + 2))]
    _msbc_case(ctx, h, srcs, False)


def test_msbc_split_hubs(ctx):
    """Vertices above 4096 in- and out-edges are split into chunks in both passes:
    a directed double star (hub -> 9000 leaves, leaves -> second hub) plus a ring."""
    n = 9003
    off, idx = [0], []
    for v in range(n):
        if v == 0:
            idx += list(range(2, n))        # hub 0 -> every leaf
        elif v == 1:
            idx += [0]                      # hub 1 -> hub 0
        else:
            idx += [1, v + 1 if v + 1 < n else 2]  # leaf -> hub 1, leaf ring
        off.append(len(idx))
    h = sg.HostGraph.from_csr(np.array(off, np.uint32), np.array(idx, np.uint32))
    srcs = [0, 1, 2, 5000, 9002] + [int(x) for x in np.random.default_rng(3).integers(0, n, 27)]
    _msbc_case(ctx, h, srcs, False)


def test_msbc_level_list_retry_long_chain(ctx):
    """A two-way chain of 2000 vertices with 32 sources spread along it: each
    vertex sits at up to 32 distinct depths, so the first launch's level list
    (8 entries per vertex) overflows and the call is retried with the bound
    of 32; the overflowed launch stops before its backward pass and the rows
    still equal the oracle's."""
    n = 2000
    off, idx = [0], []
    for v in range(n):
        idx += [u for u in (v - 1, v + 1) if 0 <= u < n]
        off.append(len(idx))
    h = sg.HostGraph.from_csr(np.array(off, np.uint32), np.array(idx, np.uint32))
    srcs = [int(x) for x in np.linspace(0, n - 1, 32).round()]
    _msbc_case(ctx, h, srcs, True)


def test_msbc_rejects_bad_input(ctx):
    h = sg.HostGraph.rmat(8, 8, seed=1)
    G = ctx.graph(h)
    with pytest.raises(sg.SGError):
        G.msbc([])
    with pytest.raises(sg.SGError):
        G.msbc(list(range(33)))
    with pytest.raises(sg.SGError):
        G.msbc([h.nv])
    G.close()
    G = ctx.graph(h, no_csc=True)
    with pytest.raises(sg.SGError):
        G.msbc([0])
    G.close()
