"""Regenerates tests/golden/*.npz: small graphs and the outputs of the
reference's own host checkers (BFSHost, SSSPHostNaive, PageRankHost,
BetweennessCentralityHost) compiled from the reference sources into
oracle/_ref/libsgref.so (`make -C oracle ref`); and tests/golden/convert/*.npz:
edge lists with the output of the reference's graph converter
(samples/tools/gtools.cpp, built as oracle/_ref/gtools) under every
combination of --deself_cycle/--deduplicate/--d2ud, and the reference's
CSCGraph transpose (csr_tocsc) of the edge list's CSR.

Run from the repository root:  python tests/golden/make_golden.py
The fixtures pin the oracle restatement (oracle/sg_oracle.c) on machines
where the reference tree is not available.
"""
import os
import shutil
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "sep-graph_b200"))

import oracle  # noqa: E402
import sepgraph as sg  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
PR_ERRORS = (1e-2, 1e-4)


def csr_from_edges(n, edges):
    edges = sorted(edges)
    off = np.zeros(n + 1, np.uint32)
    for s, _ in edges:
        off[s + 1] += 1
    off = np.cumsum(off).astype(np.uint32)
    idx = np.array([d for _, d in edges], np.uint32)
    return off, idx


def cases():
    h = sg.HostGraph.rmat(8, 16, symmetric=True, seed=1).gen_weights(1, 64, 2)
    yield "rmat8_sym", h.offsets.copy(), h.indices.copy(), h.weights.copy(), h.max_degree_vertex()[0]
    h = sg.HostGraph.rmat(9, 16, symmetric=False, seed=7).gen_weights(1, 64, 2)
    yield "rmat9_dir", h.offsets.copy(), h.indices.copy(), h.weights.copy(), int(h.pick_sources(1, 3)[0])
    h = sg.HostGraph.grid(6, 7).gen_weights(1, 1000, 2)
    yield "grid6x7", h.offsets.copy(), h.indices.copy(), h.weights.copy(), 0
    off, idx = csr_from_edges(16, [(i, i + 1) for i in range(15)])
    yield "chain16", off, idx, np.arange(1, 16, dtype=np.uint32) % 5 + 1, 0
    off, idx = csr_from_edges(21, [(0, i) for i in range(1, 21)] + [(i, 0) for i in range(1, 21)])
    yield "star21", off, idx, np.ones(40, np.uint32), 0
    e = [(0, 1), (1, 2), (2, 0), (1, 3), (5, 6), (6, 7), (7, 5)]
    off, idx = csr_from_edges(10, e)
    yield "disconnected10", off, idx, np.array([3, 1, 4, 1, 5, 9, 2], np.uint32), 1
    yield "single1", np.zeros(2, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint32), 0
    # self-loops and duplicate edges kept in the CSR
    e = [(0, 0), (0, 1), (0, 1), (1, 2), (2, 2), (2, 3), (3, 0), (3, 1), (3, 1)]
    off, idx = csr_from_edges(5, e)
    yield "loops_dups5", off, idx, np.array([2, 7, 1, 3, 5, 1, 4, 2, 6], np.uint32), 0


def build_cases():
    rng = np.random.default_rng(11)
    for name, nv, m, weighted in (("mixed40w", 40, 300, True), ("mixed25", 25, 120, False),
                                  ("hub300w", 300, 2500, True)):
        s = rng.integers(0, nv, m).astype(np.uint32)
        d = rng.integers(0, nv, m).astype(np.uint32)
        if name.startswith("hub"):  # one source and one destination with many parallel edges
            s[: m // 3] = 7
            d[m // 3: 2 * m // 3] = 7
        w = rng.integers(1, 9, m).astype(np.uint32) if weighted else None
        yield name, nv, s, d, w
    # the first inserted edge wins under --d2ud: (1,5) comes first in CSR order
    yield "d2ud_order6", 6, np.array([5, 1, 2, 2], np.uint32), np.array([1, 5, 2, 3], np.uint32), \
        np.array([10, 20, 30, 40], np.uint32)
    yield "loops4", 4, np.array([0, 1, 1, 3, 3], np.uint32), np.array([0, 1, 1, 3, 2], np.uint32), None
    yield "empty3", 3, np.zeros(0, np.uint32), np.zeros(0, np.uint32), None


def stable_csr(nv, s, d, w):
    o = np.argsort(s, kind="stable")
    off = np.zeros(nv + 1, np.uint32)
    off[1:] = np.cumsum(np.bincount(s, minlength=nv))
    return off, d[o].astype(np.uint32), (None if w is None else w[o].astype(np.uint32))


def main_build():
    if not oracle.ref_gtools_available():
        sys.exit("oracle/_ref/gtools missing: run make -C oracle ref")
    os.makedirs(os.path.join(OUT, "convert"), exist_ok=True)
    tmp = tempfile.mkdtemp(dir=OUT)
    for name, nv, s, d, w in build_cases():
        rec = dict(nv=np.uint32(nv), src=s, dst=d)
        if w is not None:
            rec["weights"] = w
        off, idx, ww = stable_csr(nv, s, d, w)
        co, ci, cw = oracle.ref_csr_tocsc(off, idx, ww)
        rec["csc_offsets"], rec["csc_indices"] = co, ci
        if cw is not None:
            rec["csc_weights"] = cw
        gr = os.path.join(tmp, "g.gr")
        sg.HostGraph.from_csr(off, idx, ww).write_gr(gr)
        for code in range(8):
            ds, dd, du = bool(code & 1), bool(code & 2), bool(code & 4)
            rs, rd, rw = oracle.ref_gtools(gr, os.path.join(tmp, "o.txt"), ds, dd, du)
            rec[f"g{code}_src"], rec[f"g{code}_dst"] = rs, rd
            if rw is not None:
                rec[f"g{code}_w"] = rw
        np.savez_compressed(os.path.join(OUT, "convert", f"{name}.npz"), **rec)
        print("convert", name, nv, len(s))
    shutil.rmtree(tmp)


def main():
    main_build()
    if not oracle.ref_available():
        sys.exit("oracle/_ref/libsgref.so missing: run make -C oracle ref")
    for name, off, idx, w, src in cases():
        rec = dict(offsets=off, indices=idx, weights=w, source=np.uint32(src))
        rec["bfs"] = oracle.ref_bfs(off, idx, src)
        rec["sssp"] = oracle.ref_sssp(off, idx, w, src)
        for k, err in enumerate(PR_ERRORS):
            rec[f"pr{k}"] = oracle.ref_pagerank(off, idx, err)
            rec[f"pr{k}_error"] = np.float64(err)
        bc, sigma = oracle.ref_bc(off, idx, src)
        rec["bc"], rec["bc_sigma"] = bc, sigma
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **rec)
        print(name, len(off) - 1, len(idx))


if __name__ == "__main__":
    main()
