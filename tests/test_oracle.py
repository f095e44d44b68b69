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
