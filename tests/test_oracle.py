"""Pins the oracle (oracle/sg_oracle.c) against the committed golden vectors
produced by the reference's own host checkers, and — where the reference
tree was available at build time — against those checkers directly."""
import glob
import os

import numpy as np
import pytest

import oracle
import sepgraph as sg

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_golden(path):
    g = _load(path)
    off, idx, w, src = g["offsets"], g["indices"], g["weights"], int(g["source"])
    assert (oracle.bfs(off, idx, src) == g["bfs"]).all()
    assert (oracle.sssp(off, idx, w, src) == g["sssp"]).all()
    for k in range(2):
        pr = oracle.pagerank_f32(off, idx, float(g[f"pr{k}_error"]))
        assert (pr.view(np.uint32) == g[f"pr{k}"].view(np.uint32)).all(), "PageRankHost float restatement"
    bc, sigma, _ = oracle.bc_f32(off, idx, src)
    assert (bc.view(np.uint32) == g["bc"].view(np.uint32)).all()
    assert (sigma == g["bc_sigma"]).all()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_f64_oracle_close_to_reference_float(path):
    g = _load(path)
    off, idx, src = g["offsets"], g["indices"], int(g["source"])
    bc64, sig64, lv = oracle.bc_f64(off, idx, src)
    assert np.allclose(bc64, g["bc"], rtol=1e-5, atol=1e-5)
    assert np.allclose(sig64, g["bc_sigma"], rtol=1e-6)
    assert ((lv == g["bfs"])).all()  # BC levels are BFS levels
    pr64 = oracle.pagerank_f64(off, idx, float(g["pr1_error"]))
    if len(off) > 1:
        assert np.allclose(pr64, g["pr1"], rtol=1e-4, atol=1e-5)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference checkers not compiled here")
@pytest.mark.parametrize("scale,sym,seed", [(10, True, 1), (11, False, 5), (13, True, 9), (12, False, 11)])
def test_oracle_bit_exact_vs_compiled_reference(scale, sym, seed):
    h = sg.HostGraph.rmat(scale, 16, symmetric=sym, seed=seed).gen_weights(1, 64, 2)
    off, idx, w = h.offsets, h.indices, h.weights
    for src in [h.max_degree_vertex()[0], int(h.pick_sources(1, seed)[0])]:
        assert (oracle.bfs(off, idx, src) == oracle.ref_bfs(off, idx, src)).all()
        assert (oracle.sssp(off, idx, w, src) == oracle.ref_sssp(off, idx, w, src)).all()
        a, b = oracle.bc_f32(off, idx, src)[:2], oracle.ref_bc(off, idx, src)
        assert (a[0].view(np.uint32) == b[0].view(np.uint32)).all() and (a[1] == b[1]).all()
    for err in (1e-2, 1e-6):
        a, b = oracle.pagerank_f32(off, idx, err), oracle.ref_pagerank(off, idx, err)
        assert (a.view(np.uint32) == b.view(np.uint32)).all()


def test_oracle_plants_detected():
    """A planted error in the oracle's input is caught by the reference-style checkers."""
    g = _load(GOLDEN[0])
    off, idx, src = g["offsets"], g["indices"], int(g["source"])
    lv = oracle.bfs(off, idx, src)
    bad = lv.copy()
    reached = np.flatnonzero(bad != oracle.INF)
    bad[reached[-1]] += 1
    assert (bad != g["bfs"]).sum() == 1
    if oracle.ref_available():
        r = oracle.ref().sgref_bfs_check(len(lv), bad.ctypes.data, g["bfs"].ctypes.data)
        assert r == 1


# ---------------------------------------------------------------- graph construction
CONVERT = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "convert", "*.npz")))


def _rows_of(off):
    return np.repeat(np.arange(len(off) - 1, dtype=np.uint32), np.diff(off.astype(np.int64)))


def _stable_csr(nv, s, d, w):
    o = np.argsort(s, kind="stable")
    off = np.zeros(nv + 1, np.uint32)
    off[1:] = np.cumsum(np.bincount(s, minlength=nv))
    return off, d[o].astype(np.uint32), (None if w is None else w[o].astype(np.uint32))


@pytest.mark.parametrize("path", CONVERT, ids=[os.path.basename(p)[:-4] for p in CONVERT])
def test_converter_oracle_matches_golden(path):
    """oracle.gtools_build against the reference converter's own output, all eight
    --deself_cycle/--deduplicate/--d2ud combinations; oracle.csr_tocsc against the
    reference's CSCGraph."""
    g = _load(path)
    nv, w = int(g["nv"]), g.get("weights")
    for code in range(8):
        off, idx, ww = oracle.gtools_build(nv, g["src"], g["dst"], w, code & 1, code & 2, code & 4)
        assert np.array_equal(_rows_of(off), g[f"g{code}_src"]), code
        assert np.array_equal(idx, g[f"g{code}_dst"]), code
        if w is not None:
            assert np.array_equal(ww, g[f"g{code}_w"]), code
    co, ci, cw = oracle.csr_tocsc(*_stable_csr(nv, g["src"], g["dst"], w))
    assert np.array_equal(co, g["csc_offsets"]) and np.array_equal(ci, g["csc_indices"])
    if w is not None:
        assert np.array_equal(cw, g["csc_weights"])


def test_converter_golden_covers_first_insert_rule():
    """d2ud_order6: edge 5->1 (w 10) comes before 1->5 (w 20) in the input, but 1->5
    is first in CSR order, so both directions keep weight 20."""
    g = _load(os.path.join(os.path.dirname(__file__), "golden", "convert", "d2ud_order6.npz"))
    src, dst, w = g["g4_src"], g["g4_dst"], g["g4_w"]
    pairs = {(int(a), int(b)): int(c) for a, b, c in zip(src, dst, w)}
    assert pairs[(1, 5)] == 20 and pairs[(5, 1)] == 20


@pytest.mark.skipif(not oracle.ref_gtools_available(), reason="reference converter not compiled here")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_converter_oracle_vs_reference_random(seed, tmp_path):
    rng = np.random.default_rng(seed)
    for trial in range(6):
        nv, m = int(rng.integers(1, 50)), int(rng.integers(0, 400))
        s = rng.integers(0, nv, m).astype(np.uint32)
        d = rng.integers(0, nv, m).astype(np.uint32)
        w = rng.integers(1, 9, m).astype(np.uint32) if trial % 2 else None
        off, idx, ww = _stable_csr(nv, s, d, w)
        gr = str(tmp_path / "g.gr")
        sg.HostGraph.from_csr(off, idx, ww).write_gr(gr)
        for code in range(8):
            rs, rd, rw = oracle.ref_gtools(gr, str(tmp_path / "o.txt"), code & 1, code & 2, code & 4)
            o2, i2, w2 = oracle.gtools_build(nv, s, d, w, code & 1, code & 2, code & 4)
            assert np.array_equal(rs, _rows_of(o2)) and np.array_equal(rd, i2), (trial, code)
            if w is not None:
                assert np.array_equal(rw, w2), (trial, code)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference checkers not compiled here")
def test_csr_tocsc_oracle_vs_reference():
    h = sg.HostGraph.rmat(10, 8, seed=5, keep_self_loops=True, keep_duplicates=True).gen_weights(1, 9, 3)
    a = oracle.csr_tocsc(h.offsets, h.indices, h.weights)
    b = oracle.ref_csr_tocsc(h.offsets, h.indices, h.weights)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


# ---------------------------------------------------------------- full-size inputs and checkers
@pytest.mark.parametrize("scale,sym,loops,dups", [(10, False, False, False), (12, True, False, False),
                                                  (11, False, True, True), (16, False, False, False),
                                                  (14, True, False, False)])
def test_oracle_generator_equals_library_generator(scale, sym, loops, dups):
    """The benchmark's reference arm builds its graph with the oracle's generator
    (it must not load the library): CSR, weights and sources equal word for word."""
    g = oracle.rmat(scale, 16, symmetric=sym, keep_self_loops=loops, keep_duplicates=dups)
    h = sg.HostGraph.rmat(scale, 16, symmetric=sym, seed=1, keep_self_loops=loops, keep_duplicates=dups)
    assert np.array_equal(g.offsets, h.offsets) and np.array_equal(g.indices, h.indices)
    g.gen_weights(1, 64, 2)
    h.gen_weights(1, 64, 2)
    assert np.array_equal(g.weights, h.weights)
    assert np.array_equal(g.pick_sources(8, 3), h.pick_sources(8, 3))
    assert g.max_degree_vertex()[0] == h.max_degree_vertex()[0]


def test_oracle_grid_equals_library_grid():
    for r, c in ((1, 1), (1, 7), (6, 1), (7, 5), (33, 64)):
        g, h = oracle.grid(r, c), sg.HostGraph.grid(r, c)
        assert np.array_equal(g.offsets, h.offsets) and np.array_equal(g.indices, h.indices)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_dijkstra_equals_ssspnaive_golden(path):
    g = _load(path)
    assert (oracle.dijkstra(g["offsets"], g["indices"], g["weights"], int(g["source"])) == g["sssp"]).all()


@pytest.mark.parametrize("kind", ["rmat_dir", "rmat_sym", "grid"])
def test_dijkstra_equals_ssspnaive(kind):
    if kind == "grid":
        h = oracle.grid(64, 48).gen_weights(1, 1000, 2)
    else:
        h = oracle.rmat(14, 16, symmetric=kind == "rmat_sym").gen_weights(1, 64, 2)
    for src in h.pick_sources(3, 7):
        want = oracle.ref_sssp(h.offsets, h.indices, h.weights, int(src)) if oracle.ref_available() else \
            oracle.sssp(h.offsets, h.indices, h.weights, int(src))
        assert np.array_equal(oracle.dijkstra(h.offsets, h.indices, h.weights, int(src)), want)


@pytest.mark.parametrize("path", GOLDEN + ["rmat14"], ids=[os.path.basename(p)[:-4] for p in GOLDEN] + ["rmat14"])
def test_pagerank_fixed_point_equals_residual_push(path):
    """The parallel Jacobi FP64 oracle used at full size converges to PageRankHost's
    fixed point: it agrees with the FP64 residual-push restatement run to 1e-14."""
    if path == "rmat14":
        h = oracle.rmat(14, 16)
        off, idx = h.offsets, h.indices
    else:
        g = _load(path)
        off, idx = g["offsets"], g["indices"]
    if len(off) < 2:
        return
    jac, sweeps = oracle.pagerank_fixed_point_f64(off, idx, 1e-14)
    push = oracle.pagerank_f64(off, idx, 1e-14)
    assert sweeps < 2000
    assert np.abs(jac / jac.sum() - push / push.sum()).sum() <= 1e-11
    assert np.allclose(jac, push, rtol=1e-9, atol=1e-12)
