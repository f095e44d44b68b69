"""GPU graph construction (sg_graph_build, the device CSR -> CSC transpose of
sg_graph_create) against the reference converter's golden output, the oracle
restatements of gtools and csr_tocsc, and, at full size, against the host
generators (a shuffled raw edge stream must rebuild the same CSR)."""
import glob
import os

import numpy as np
import pytest

import oracle
import sepgraph as sg

pytestmark = pytest.mark.gpu

CONVERT = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "convert", "*.npz")))


@pytest.fixture(scope="module")
def ctx():
    c = sg.Context(0)
    yield c
    c.close()


def _load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def _rows_of(off):
    return np.repeat(np.arange(len(off) - 1, dtype=np.uint32), np.diff(off.astype(np.int64)))


def _stable_csr(nv, s, d, w):
    o = np.argsort(s, kind="stable")
    off = np.zeros(nv + 1, np.uint32)
    off[1:] = np.cumsum(np.bincount(s, minlength=nv))
    return off, d[o].astype(np.uint32), (None if w is None else w[o].astype(np.uint32))


def _coo(h):
    return _rows_of(h.offsets), h.indices.copy(), (None if h.weights is None else h.weights.copy())


def _same(a, b):
    return all((x is None and y is None) or np.array_equal(x, y) for x, y in zip(a, b))


def _build(ctx, nv, s, d, w, code, sort_rows=False, **kw):
    G = ctx.build_graph(nv, s, d, w, deself_cycle=bool(code & 1), deduplicate=bool(code & 2), d2ud=bool(code & 4),
                        sort_rows=sort_rows, **kw)
    try:
        return G.copy_out()
    finally:
        G.close()


@pytest.mark.parametrize("path", CONVERT, ids=[os.path.basename(p)[:-4] for p in CONVERT])
def test_converter_matches_reference_output(ctx, path):
    g = _load(path)
    nv, w = int(g["nv"]), g.get("weights")
    for code in range(8):
        off, idx, ww = _build(ctx, nv, g["src"], g["dst"], w, code)
        assert np.array_equal(_rows_of(off), g[f"g{code}_src"]), code
        assert np.array_equal(idx, g[f"g{code}_dst"]), code
        if w is not None:
            assert np.array_equal(ww, g[f"g{code}_w"]), code


@pytest.mark.parametrize("path", CONVERT, ids=[os.path.basename(p)[:-4] for p in CONVERT])
def test_transpose_matches_reference_golden(ctx, path):
    g = _load(path)
    nv, w = int(g["nv"]), g.get("weights")
    off, idx, ww = _stable_csr(nv, g["src"], g["dst"], w)
    G = ctx.graph_from_csr(off, idx, ww)
    co, ci, cw = G.copy_out(csc=True)
    G.close()
    assert np.array_equal(co, g["csc_offsets"]) and np.array_equal(ci, g["csc_indices"])
    if w is not None:
        assert np.array_equal(cw, g["csc_weights"])


@pytest.mark.parametrize("seed", [1, 2])
@pytest.mark.parametrize("code", range(8))
@pytest.mark.parametrize("sort_rows", [False, True])
def test_build_matches_oracle_random(ctx, seed, code, sort_rows):
    rng = np.random.default_rng(seed * 100 + code)
    nv, m = 3000, 40000
    s = rng.integers(0, nv, m).astype(np.uint32)
    d = rng.integers(0, nv, m).astype(np.uint32)
    s[:5000] = 17  # a long row (merge passes) and a long in-edge list
    d[5000:9000] = 23
    w = rng.integers(1, 100, m).astype(np.uint32) if seed == 1 else None
    got = _build(ctx, nv, s, d, w, code, sort_rows=sort_rows)
    want = oracle.gtools_build(nv, s, d, w, code & 1, code & 2, code & 4, sort_rows=sort_rows)
    assert _same(got, want)


@pytest.mark.parametrize("hub", [4096, 4097, 8193, 20000, 70001])
def test_long_rows_merge_passes(ctx, hub):
    """Rows longer than one shared-memory sort take 1-5 merge passes (odd and even
    counts end in different buffers); every entry of the hub row is distinct."""
    rng = np.random.default_rng(hub)
    nv = 100000
    m = hub + 20000
    s = np.concatenate([np.full(hub, 5, np.uint32), rng.integers(0, nv, 20000).astype(np.uint32)])
    d = np.concatenate([rng.permutation(nv)[:hub].astype(np.uint32) if hub <= nv else rng.integers(0, nv, hub).astype(np.uint32),
                        rng.integers(0, nv, 20000).astype(np.uint32)])
    p = rng.permutation(m)
    s, d = s[p], d[p]
    for code, sort_rows in ((0, False), (0, True), (2, False), (4, False)):
        got = _build(ctx, nv, s, d, None, code, sort_rows=sort_rows)
        assert _same(got, oracle.gtools_build(nv, s, d, None, code & 1, code & 2, code & 4, sort_rows=sort_rows))
    G = ctx.graph_from_csr(*_stable_csr(nv, s, d, None))
    got = G.copy_out(csc=True)
    G.close()
    assert _same(got, oracle.csr_tocsc(*_stable_csr(nv, s, d, None)))


def test_transpose_rmat20_with_parallel_edges(ctx):
    h = sg.HostGraph.rmat(20, 16, seed=3, keep_self_loops=True, keep_duplicates=True).gen_weights(1, 64, 4)
    G = ctx.graph(h)
    got = G.copy_out(csc=True)
    G.close()
    assert _same(got, oracle.csr_tocsc(h.offsets, h.indices, h.weights))


def test_symmetric_weighted_views(ctx):
    """Symmetric flag with weights: identical transpose -> alias; asymmetric weights ->
    own CSC weights; a structure whose transpose lists a row in another order -> full
    CSC.  The in-edge view always equals csr_tocsc of the CSR."""
    h = sg.HostGraph.rmat(12, 8, symmetric=True, seed=2)
    off, idx = h.offsets.copy(), h.indices.copy()
    src = _rows_of(off)
    w_sym = ((np.minimum(src, idx).astype(np.uint64) * 31 + np.maximum(src, idx)) % 97 + 1).astype(np.uint32)
    w_asym = ((src.astype(np.uint64) * 7 + idx) % 50 + 1).astype(np.uint32)
    sizes = {}
    for name, w in (("sym", w_sym), ("asym", w_asym)):
        G = ctx.graph_from_csr(off, idx, w, symmetric=True)
        sizes[name] = G.info()["device_bytes"]
        got = G.copy_out(csc=True)
        G.close()
        assert _same(got, oracle.csr_tocsc(off, idx, w)), name
    assert sizes["asym"] > sizes["sym"]
    # parallel edges 0->1 (w 5, w 9) and 1->0 (w 9, w 5): same structure, the
    # transpose lists the weights the other way round
    # row 0 listed as (2, 1): the transpose orders it (1, 2), a different structure
    for off2, idx2, w2 in ((np.array([0, 2, 4], np.uint32), np.array([1, 1, 0, 0], np.uint32),
                            np.array([5, 9, 9, 5], np.uint32)),
                           (np.array([0, 2, 3, 4], np.uint32), np.array([2, 1, 0, 0], np.uint32),
                            np.array([3, 4, 4, 3], np.uint32))):
        G = ctx.graph_from_csr(off2, idx2, w2, symmetric=True)
        got = G.copy_out(csc=True)
        G.close()
        assert _same(got, oracle.csr_tocsc(off2, idx2, w2))


def test_full_size_rebuild_from_shuffled_edges(ctx):
    """RMAT-22 raw edge stream (self-loops and duplicates kept), shuffled: deself +
    deduplicate + row order rebuilds the host generator's directed CSR exactly, and
    --d2ud rebuilds its symmetric CSR."""
    raw = sg.HostGraph.rmat(22, 16, seed=1, keep_self_loops=True, keep_duplicates=True)
    s, d, _ = _coo(raw)
    nv = raw.nv
    del raw
    p = np.random.default_rng(9).permutation(len(s))
    s, d = s[p], d[p]
    hd = sg.HostGraph.rmat(22, 16, seed=1)
    off, idx, _ = _build(ctx, nv, s, d, None, 3, sort_rows=True)
    assert np.array_equal(off, hd.offsets) and np.array_equal(idx, hd.indices)
    del hd
    hs = sg.HostGraph.rmat(22, 16, symmetric=True, seed=1)
    off, idx, _ = _build(ctx, nv, s, d, None, 5)
    assert np.array_equal(off, hs.offsets) and np.array_equal(idx, hs.indices)


def test_built_graph_runs_algorithms(ctx):
    h = sg.HostGraph.rmat(14, 16, symmetric=True, seed=4)
    s, d, _ = _coo(sg.HostGraph.rmat(14, 16, seed=4, keep_self_loops=True, keep_duplicates=True))
    G = ctx.build_graph(h.nv, s, d, d2ud=True, deself_cycle=True)
    src = h.max_degree_vertex()[0]
    lv, _, _ = G.bfs(src)
    assert np.array_equal(lv, oracle.bfs(h.offsets, h.indices, src))
    G.close()


def test_build_rejects_bad_input(ctx):
    with pytest.raises(sg.SGError):
        ctx.build_graph(4, np.array([0, 4], np.uint32), np.array([1, 2], np.uint32))
    with pytest.raises(sg.SGError):
        ctx.build_graph(4, np.array([0, 1], np.uint32), np.array([9, 2], np.uint32), d2ud=True)
    G = ctx.build_graph(4, np.array([0, 1], np.uint32), np.array([1, 2], np.uint32))  # context still usable
    assert np.array_equal(G.copy_out()[0], np.array([0, 1, 2, 2, 2], np.uint32))
    G.close()


def test_device_inputs(ctx):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(6)
    s = rng.integers(0, 500, 5000).astype(np.uint32)
    d = rng.integers(0, 500, 5000).astype(np.uint32)
    ts = torch.from_numpy(s.view(np.int32)).cuda()
    td = torch.from_numpy(d.view(np.int32)).cuda()
    G = ctx.build_graph(500, ts, td, deduplicate=True, sort_rows=True)
    got = G.copy_out()
    G.close()
    assert _same(got, oracle.gtools_build(500, s, d, None, False, True, False, sort_rows=True))


BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "sep-graph_b200", "bin")


@pytest.mark.parametrize("path", CONVERT, ids=[os.path.basename(p)[:-4] for p in CONVERT])
def test_gtools_cli_matches_reference_output(path, tmp_path):
    """bin/gtools (the converter's flags and text outputs, preprocessing on the GPU)
    on the golden edge lists: same edge list as the reference converter, and the
    out-degree file agrees with it."""
    import subprocess

    exe = os.path.join(BIN, "gtools")
    if not os.path.exists(exe):
        pytest.skip("samples not built")
    g = _load(path)
    nv, w = int(g["nv"]), g.get("weights")
    gr = str(tmp_path / "g.gr")
    sg.HostGraph.from_csr(*_stable_csr(nv, g["src"], g["dst"], w)).write_gr(gr)
    b = lambda x: "true" if x else "false"
    for code in range(8):
        out, deg = str(tmp_path / "e.txt"), str(tmp_path / "d.txt")
        r = subprocess.run([exe, f"--graphfile={gr}", f"--output={out}", f"--out_degree={deg}",
                            f"--deself_cycle={b(code & 1)}", f"--deduplicate={b(code & 2)}", f"--d2ud={b(code & 4)}"],
                           capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        rows = np.loadtxt(out, dtype=np.int64, ndmin=2) if os.path.getsize(out) else np.zeros((0, 3 if w is not None else 2))
        assert np.array_equal(rows[:, 0], g[f"g{code}_src"]) and np.array_equal(rows[:, 1], g[f"g{code}_dst"]), code
        if w is not None:
            assert np.array_equal(rows[:, 2], g[f"g{code}_w"]), code
        d = np.loadtxt(deg, dtype=np.int64, ndmin=2)
        assert np.array_equal(d[:, 1], np.bincount(g[f"g{code}_src"].astype(np.int64), minlength=nv)), code


def test_released_arena_is_reused(ctx):
    """sg_graph_destroy keeps the graph's arena in its context; the next graph that
    fits (half to all of it) reuses it, results unchanged; sg_ctx_release_cached
    frees it."""
    c = sg.Context(0)
    try:
        h = sg.HostGraph.rmat(12, 8, seed=5)
        G = c.graph(h)
        b1 = G.info()["device_bytes"]
        G.close()
        h2 = sg.HostGraph.rmat(12, 8, seed=6)  # a little smaller or larger, same scale
        G = c.graph(h2)
        if G.info()["ne"] * 2 >= h.indices.size:
            assert G.info()["device_bytes"] >= b1 // 2
        src = h2.max_degree_vertex()[0]
        assert np.array_equal(G.bfs(src)[0], oracle.bfs(h2.offsets, h2.indices, src))
        assert _same(G.copy_out(csc=True), oracle.csr_tocsc(h2.offsets, h2.indices, None))
        G.close()
        c.release_cached()
        G = c.graph(sg.HostGraph.rmat(14, 8, seed=7))  # larger than the old arena: its own allocation
        assert G.info()["device_bytes"] > b1
        G.close()
    finally:
        c.close()
