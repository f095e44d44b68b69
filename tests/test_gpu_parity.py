"""GPU parity of the four algorithms through the C ABI against the oracle.

Tolerances (stated per algorithm, as the reference's checkers are):
  BFS levels, SSSP distances (uint32 weights): bit-exact.
  PageRank: L1 distance of L1-normalised rank vectors <= 1e-6 against the
            FP64 restatement of PageRankHost run to a 1e-12 residual.
  BC: |gpu - fp64| <= 1e-4 * |fp64| + 1e-5 per vertex; path counts exact.
"""
import glob
import os

import numpy as np
import pytest

import oracle
import sepgraph as sg

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
GIDS = [os.path.basename(p)[:-4] for p in GOLDEN]
PR_L1_TOL = 1e-6
BC_RTOL, BC_ATOL = 1e-4, 1e-5


@pytest.fixture(scope="module")
def ctx():
    c = sg.Context(0)
    yield c
    c.close()


def _load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def _graph(ctx, g, weighted=True, symmetric=False):
    return ctx.graph_from_csr(g["offsets"], g["indices"], g["weights"] if weighted and len(g["indices"]) else None,
                              symmetric=symmetric)


TRAVERSAL_VARIANTS = ["auto", "async_push_dd", "async_pull_dd"]
LBS = ["none", "fine"]


@pytest.mark.parametrize("lb", LBS)
@pytest.mark.parametrize("variant", TRAVERSAL_VARIANTS)
@pytest.mark.parametrize("path", GOLDEN, ids=GIDS)
def test_bfs_golden(ctx, path, variant, lb):
    g = _load(path)
    G = _graph(ctx, g, weighted=False)
    for non_atomic in (1, 0):
        lv, st, _ = G.bfs(int(g["source"]), variant=variant, lb_push=lb, lb_pull=lb, non_atomic=non_atomic)
        assert (lv == g["bfs"]).all(), (variant, lb, non_atomic)


@pytest.mark.parametrize("lb", LBS)
@pytest.mark.parametrize("variant", TRAVERSAL_VARIANTS + ["async_push_td", "prio"])
@pytest.mark.parametrize("path", GOLDEN, ids=GIDS)
def test_sssp_golden(ctx, path, variant, lb):
    g = _load(path)
    G = _graph(ctx, g)
    kw = dict(lb_push=lb, lb_pull=lb, max_iteration=100000)
    if variant == "prio":
        kw.update(priority="low_high")
    else:
        kw.update(variant=variant)
    d, st, _ = G.sssp(int(g["source"]), **kw)
    assert (d == g["sssp"]).all(), (variant, lb)


def _pr_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a / a.sum() - b / b.sum()).sum()


@pytest.mark.parametrize("variant", ["auto", "sync_pull_td", "async_push_td", "async_push_dd"])
@pytest.mark.parametrize("path", GOLDEN, ids=GIDS)
def test_pagerank_golden(ctx, path, variant):
    g = _load(path)
    G = _graph(ctx, g, weighted=False)
    r, st, _ = G.pagerank(variant=variant, pr_error=1e-7, max_iteration=100000)
    ref64 = oracle.pagerank_f64(g["offsets"], g["indices"], 1e-12)
    assert _pr_l1(r, ref64) <= PR_L1_TOL, (variant, _pr_l1(r, ref64))
    # the reference's own 5% checker against its float result at a 1e-4 residual threshold
    r2, _, _ = G.pagerank(variant=variant, pr_error=float(g["pr1_error"]), max_iteration=100000)
    if oracle.ref_available():
        assert oracle.ref_pagerank_check(r2, g["pr1"]) == 0


@pytest.mark.parametrize("variant", TRAVERSAL_VARIANTS)
@pytest.mark.parametrize("path", GOLDEN, ids=GIDS)
def test_bc_golden(ctx, path, variant):
    g = _load(path)
    G = _graph(ctx, g, weighted=False)
    src = int(g["source"])
    bc, sigma, st = G.bc(src, variant=variant)
    bc64, sig64, _ = oracle.bc_f64(g["offsets"], g["indices"], src)
    assert (sigma.astype(np.float64) == sig64).all()
    assert np.allclose(bc, bc64, rtol=BC_RTOL, atol=BC_ATOL), np.max(np.abs(bc - bc64))
    assert np.allclose(bc, g["bc"], rtol=0.05, atol=0.01)  # reference float result, its 5% rule


# ---------------------------------------------------------------- larger graphs, oracle at test time
@pytest.mark.parametrize("scale,sym", [(14, True), (16, True), (15, False)])
def test_bfs_rmat(ctx, scale, sym):
    h = sg.HostGraph.rmat(scale, 16, symmetric=sym, seed=1)
    G = ctx.graph(h, symmetric=sym)
    for src in [h.max_degree_vertex()[0]] + list(h.pick_sources(3, 3)):
        ref = oracle.bfs(h.offsets, h.indices, int(src))
        for variant in ("auto", "async_push_dd", "async_pull_dd"):
            lv, st, _ = G.bfs(int(src), variant=variant)
            assert (lv == ref).all(), (variant, src)
        for kw in (dict(worklist=2), dict(worklist=2, non_atomic=0, local_depth=8)):
            lv, st, _ = G.bfs(int(src), variant="async_push_dd", **kw)
            assert (lv == ref).all(), (kw, src)
        for kw in (dict(pull_scan=2), dict(pull_scan=2, variant="async_pull_dd")):  # warp-cooperative pull
            lv, st, _ = G.bfs(int(src), **kw)
            assert (lv == ref).all(), (kw, src)
        assert st.edges_reached == np.diff(h.offsets)[ref != sg.INF].sum()


@pytest.mark.parametrize("scale", [14, 16])
def test_sssp_rmat(ctx, scale):
    h = sg.HostGraph.rmat(scale, 16, symmetric=False, seed=1).gen_weights(1, 64, 2)
    G = ctx.graph(h)
    for src in h.pick_sources(4, 3):
        ref = oracle.sssp(h.offsets, h.indices, h.weights, int(src))
        for kw in (dict(), dict(variant="async_push_dd"), dict(priority="low_high"),
                   dict(priority="low_high", priority_delta=8), dict(variant="async_pull_dd"),
                   dict(variant="async_push_dd", worklist=2),
                   dict(variant="async_push_dd", priority="low_high", priority_delta=4, worklist=2, local_depth=16),
                   dict(variant="async_push_dd", priority="low_high", priority_delta=8, worklist=1, chunk_edges=37),
                   dict(variant="async_push_dd", priority="low_high", priority_delta=8, hub_stage=-1),
                   dict(variant="async_push_dd", hub_stage=1, heavy_degree=4)):
            d, st, _ = G.sssp(int(src), max_iteration=100000, **kw)
            assert (d == ref).all(), kw


def test_sssp_grid(ctx):
    h = sg.HostGraph.grid(128, 96).gen_weights(1, 1000, 2)
    G = ctx.graph(h)
    ref = oracle.sssp(h.offsets, h.indices, h.weights, 0)
    for kw in (dict(), dict(priority="low_high"), dict(variant="async_push_dd", lb_push="none")):
        d, st, _ = G.sssp(0, max_iteration=1000000, **kw)
        assert (d == ref).all(), kw


@pytest.mark.parametrize("variant", ["auto", "sync_pull_td", "async_push_dd"])
def test_pagerank_rmat(ctx, variant):
    h = sg.HostGraph.rmat(14, 16, symmetric=False, seed=1)
    G = ctx.graph(h)
    r, st, _ = G.pagerank(variant=variant, pr_error=1e-7, max_iteration=100000)
    ref64 = oracle.pagerank_f64(h.offsets, h.indices, 1e-12)
    assert _pr_l1(r, ref64) <= PR_L1_TOL


@pytest.mark.parametrize("cut", [0.05, 0.2, 1.0])
def test_pagerank_sampling_priority(ctx, cut):
    """SetSampleBasedPriority (--cut_threshold): each ASYNC_PUSH_TD round takes only
    the vertices whose residual is at or above the sampled threshold; the fixed
    point is unchanged (L1 against the FP64 oracle), and a small cut takes more
    rounds than processing every vertex."""
    h = sg.HostGraph.rmat(14, 16, symmetric=False, seed=1)
    G = ctx.graph(h)
    ref64 = oracle.pagerank_f64(h.offsets, h.indices, 1e-12)
    r, st, _ = G.pagerank(variant="async_push_td", priority="sampling", cut_threshold=cut, pr_error=1e-7,
                          max_iteration=100000)
    assert _pr_l1(r, ref64) <= PR_L1_TOL, (cut, _pr_l1(r, ref64))
    r0, st0, _ = G.pagerank(variant="async_push_td", pr_error=1e-7, max_iteration=100000)
    if cut <= 0.05:
        assert st.rounds > st0.rounds, (st.rounds, st0.rounds)
    G.close()


def test_bc_rmat(ctx):
    h = sg.HostGraph.rmat(14, 16, symmetric=True, seed=1)
    G = ctx.graph(h, symmetric=True)
    for src in [h.max_degree_vertex()[0], int(h.pick_sources(1, 3)[0])]:
        bc64, sig64, _ = oracle.bc_f64(h.offsets, h.indices, int(src))
        for kw in (dict(), dict(pull_scan=2), dict(pull_scan=2, variant="async_pull_dd")):
            bc, sigma, st = G.bc(int(src), **kw)
            assert (sigma.astype(np.float64) == sig64).all(), kw
            assert np.allclose(bc, bc64, rtol=BC_RTOL, atol=BC_ATOL), kw


@pytest.mark.parametrize("path", GOLDEN, ids=GIDS)
def test_wl_sort_golden(ctx, path):
    """--wl_sort on the small fixtures (fewer bitmap words than blocks: most
    blocks own an empty range of the sort)."""
    g = _load(path)
    G = _graph(ctx, g)
    src = int(g["source"])
    for kw in (dict(), dict(variant="async_push_dd"), dict(variant="async_push_dd", lb_push="none")):
        lv, _, _ = G.bfs(src, wl_sort=1, **kw)
        assert (lv == g["bfs"]).all(), kw
    for kw in (dict(variant="async_push_dd"), dict(priority="low_high")):
        d, _, _ = G.sssp(src, wl_sort=1, max_iteration=100000, **kw)
        assert (d == g["sssp"]).all(), kw


@pytest.mark.parametrize("path", GOLDEN, ids=GIDS)
def test_staged_hub_chunks_golden(ctx, path):
    """Hub chunks staged by bulk copies (every vertex above 1 edge is split into
    256-edge chunks here), weighted and unweighted, against the oracle."""
    g = _load(path)
    src = int(g["source"])
    for weighted in (True, False):
        G = _graph(ctx, g, weighted=weighted)
        want = g["sssp"] if weighted else g["bfs"]
        for kw in (dict(), dict(priority="low_high"), dict(blocks_per_sm=8)):
            d, _, _ = G.sssp(src, variant="async_push_dd", hub_stage=1, heavy_degree=1, chunk_edges=256,
                             max_iteration=100000, **kw)
            assert (d == want).all(), (weighted, kw)


@pytest.mark.parametrize("path", GOLDEN, ids=GIDS)
def test_bitmap_worklists_golden(ctx, path):
    """Bitmap worklists (sg_options.worklist = SG_WORKLIST_BITMAP) on the small
    fixtures: BFS and SSSP with and without two-level priority and lookahead."""
    g = _load(path)
    G = _graph(ctx, g)
    src = int(g["source"])
    for kw in (dict(), dict(non_atomic=0, local_depth=4), dict(blocks_per_sm=8)):
        lv, _, _ = G.bfs(src, variant="async_push_dd", worklist=2, **kw)
        assert (lv == g["bfs"]).all(), kw
    for kw in (dict(), dict(priority="low_high"), dict(priority="low_high", priority_delta=3, local_depth=8),
               dict(chunk_edges=32, heavy_degree=1)):
        d, _, _ = G.sssp(src, variant="async_push_dd", worklist=2, max_iteration=100000, **kw)
        assert (d == g["sssp"]).all(), kw
    r, _, _ = G.pagerank(variant="async_push_dd", worklist=2, pr_error=1e-7, max_iteration=100000)
    assert _pr_l1(r, oracle.pagerank_f64(g["offsets"], g["indices"], 1e-12)) <= PR_L1_TOL


@pytest.mark.parametrize("bps", [1, 8])
def test_wl_sort_same_results(ctx, bps):
    """--wl_sort (framework.cuh:488-496): every data-driven push round takes its
    worklist in ascending vertex order.  Results equal the oracle's, and a
    level-synchronous BFS takes the same rounds as without the sort."""
    h = sg.HostGraph.rmat(15, 16, symmetric=True, seed=1).gen_weights(1, 64, 2)
    G = ctx.graph(h, symmetric=True)
    src = int(h.max_degree_vertex()[0])
    ref = oracle.bfs(h.offsets, h.indices, src)
    for kw in (dict(), dict(variant="async_push_dd"), dict(variant="async_push_dd", lb_push="none"),
               dict(variant="async_push_dd", local_depth=16)):
        lv0, st0, _ = G.bfs(src, blocks_per_sm=bps, **kw)
        lv, st, _ = G.bfs(src, blocks_per_sm=bps, wl_sort=1, **kw)
        assert (lv == ref).all() and (lv0 == ref).all(), kw
        if "local_depth" not in kw:
            assert st.rounds == st0.rounds, (kw, st.rounds, st0.rounds)
    ref = oracle.sssp(h.offsets, h.indices, h.weights, src)
    for kw in (dict(variant="async_push_dd"), dict(priority="low_high"),
               dict(priority="low_high", priority_delta=8, variant="async_push_dd", local_depth=16)):
        d, _, _ = G.sssp(src, blocks_per_sm=bps, wl_sort=1, max_iteration=100000, **kw)
        assert (d == ref).all(), kw
    bc, sigma, _ = G.bc(src, blocks_per_sm=bps, wl_sort=1, variant="async_push_dd")
    bc64, sig64, _ = oracle.bc_f64(h.offsets, h.indices, src)
    assert (sigma.astype(np.float64) == sig64).all()
    assert np.allclose(bc, bc64, rtol=BC_RTOL, atol=BC_ATOL)
    hp = sg.HostGraph.rmat(14, 16, symmetric=False, seed=1)
    Gp = ctx.graph(hp)
    r, _, _ = Gp.pagerank(variant="async_push_dd", wl_sort=1, blocks_per_sm=bps, pr_error=1e-7,
                          max_iteration=100000)
    assert _pr_l1(r, oracle.pagerank_f64(hp.offsets, hp.indices, 1e-12)) <= PR_L1_TOL


# ---------------------------------------------------------------- engine behaviour
def test_policy_switches_direction_and_trace(ctx):
    h = sg.HostGraph.rmat(16, 16, symmetric=True, seed=1)
    G = ctx.graph(h, symmetric=True)
    src = h.max_degree_vertex()[0]
    lv, st, tr = G.bfs(src, trace_capacity=64)
    assert st.rounds_by_variant[7] > 0 and st.rounds_by_variant[5] > 0, "push and pull rounds"
    assert len(tr) == st.rounds and tr[0]["variant"] == 5
    assert tr[-1]["out_nodes"] == 0
    assert (lv == oracle.bfs(h.offsets, h.indices, src)).all()


def test_forced_unsupported_variant(ctx):
    g = _load(GOLDEN[0])
    G = _graph(ctx, g)
    for v in ("async_pull_td", "sync_push_td", "sync_push_dd"):
        with pytest.raises(sg.SGError) as e:
            G.bfs(0, variant=v)
        assert e.value.status == 6
    G.bfs(0)  # context still usable


def test_invalid_source(ctx):
    g = _load(GOLDEN[0])
    G = _graph(ctx, g)
    with pytest.raises(sg.SGError) as e:
        G.bfs(len(g["offsets"]) - 1)
    assert e.value.status == 1


def test_max_iteration_stops(ctx):
    g = _load([p for p in GOLDEN if "chain16" in p][0])
    G = _graph(ctx, g)
    lv, st, _ = G.bfs(0, max_iteration=5, variant="async_push_dd")
    assert st.rounds == 5 and st.max_iteration_reached == 1
    assert (lv[:5] == np.arange(5)).all() and (lv[6:] == sg.INF).all()


def test_device_output_buffer(ctx):
    torch = pytest.importorskip("torch")
    h = sg.HostGraph.rmat(12, 16, symmetric=True, seed=1)
    G = ctx.graph(h, symmetric=True)
    out = torch.empty(h.nv, dtype=torch.int32, device="cuda")
    G.bfs(0, out=out)
    ctx.synchronize()
    ref = oracle.bfs(h.offsets, h.indices, 0)
    assert (out.cpu().numpy().view(np.uint32) == ref).all()


def test_repeat_runs_deterministic(ctx):
    h = sg.HostGraph.rmat(13, 16, symmetric=False, seed=3).gen_weights(1, 64, 2)
    G = ctx.graph(h)
    outs = [G.sssp(int(h.pick_sources(1, 1)[0]))[0] for _ in range(3)]
    assert all((o == outs[0]).all() for o in outs)


@pytest.mark.parametrize("no_csc", [False, True])
def test_invalid_csr_rejected(ctx, no_csc):
    """Malformed CSR is rejected both by the host check (graphs that build a
    CSC on the host) and by the device check (graphs uploaded as they are)."""
    good_off = np.array([0, 2, 3, 3], np.uint32)
    good_idx = np.array([1, 2, 0], np.uint32)
    for off, idx in ((np.array([1, 2, 3, 3], np.uint32), good_idx),      # does not start at 0
                     (np.array([0, 2, 1, 3], np.uint32), good_idx),      # not monotone
                     (good_off, np.array([1, 3, 0], np.uint32))):        # index out of range
        with pytest.raises(sg.SGError) as e:
            ctx.graph_from_csr(off, idx, no_csc=no_csc)
        assert e.value.status == 1
    G = ctx.graph_from_csr(good_off, good_idx, no_csc=no_csc)  # the context is still usable
    assert (G.bfs(0, variant="async_push_dd")[0] == np.array([0, 1, 1], np.uint32)).all()


def test_device_checked_upload_matches_host_path(ctx):
    torch = pytest.importorskip("torch")
    h = sg.HostGraph.rmat(13, 16, seed=3).gen_weights(1, 64, 4)
    off = torch.from_numpy(h.offsets.astype(np.int32)).cuda()
    idx = torch.from_numpy(h.indices.astype(np.int32)).cuda()
    w = torch.from_numpy(h.weights.astype(np.int32)).cuda()
    Gd = ctx.graph_from_csr(off, idx, w, no_csc=True)    # device inputs, device check
    Gh = ctx.graph(h)                                      # host inputs, host check + CSC
    for s in (int(x) for x in h.pick_sources(3, 5)):
        # default two-level delta comes from the weight sum each path computed
        a, _, _ = Gd.sssp(s, priority="low_high", max_iteration=1000000)
        b, _, _ = Gh.sssp(s, priority="low_high", max_iteration=1000000)
        assert (a == b).all() and (a == oracle.sssp(h.offsets, h.indices, h.weights, s)).all()


def test_device_wait_timeout_reports_status_and_context_recovers(ctx):
    """Failure detection without a fault: a star's hub expanded by one thread
    (push load balancing off) holds every other block at the round barrier far
    longer than a 1 ns bound, so their bounded waits give up, the launch
    returns SG_ERR_TIMEOUT (a leader that gives up releases the others with an
    abort bit), and the same context then runs a normal query exactly."""
    n = 1 << 20
    off = np.full(n + 2, n, np.uint32)
    off[0] = 0
    idx = np.arange(1, n + 1, dtype=np.uint32)
    G = ctx.graph_from_csr(off, idx, no_csc=True)
    seen = None
    for _ in range(3):
        try:
            G.bfs(0, variant="async_push_dd", lb_push="none", timeout_s=1e-9)
        except sg.SGError as e:
            seen = e.status
            break
    assert seen == 4, seen  # SG_ERR_TIMEOUT
    lv, st, _ = G.bfs(0, variant="async_push_dd", lb_push="none")
    assert st.device_error == 0
    assert lv[0] == 0 and (lv[1:] == 1).all()
    G.close()
