"""ORACLE — test infrastructure only (never imported by the product library).

Loads two CPU checkers through ctypes:
  * liboracle.so       — plain-C restatement of the reference's host algorithms
                         (oracle/sg_oracle.c; each function cites its source);
  * _ref/libsgref.so   — the reference's own host checkers compiled from its
                         sources by `make -C oracle ref` (present when the
                         reference tree was available at build time).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm may use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(_HERE, "liboracle.so")
REF_LIB = os.path.join(_HERE, "_ref", "libsgref.so")
INF = 0xFFFFFFFF

_o = None
_r = None
_P = C.c_void_p


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def lib() -> C.CDLL:
    global _o
    if _o is None:
        if not os.path.exists(ORACLE_LIB):
            subprocess.run(["make", "-C", _HERE, "liboracle.so"], check=True, capture_output=True)
        L = C.CDLL(ORACLE_LIB)
        for n in ("sgo_bfs",):
            getattr(L, n).argtypes = [C.c_uint32, _P, _P, C.c_uint32, _P]
        L.sgo_sssp.argtypes = [C.c_uint32, _P, _P, _P, C.c_uint32, _P]
        L.sgo_pagerank_f32.argtypes = [C.c_uint32, _P, _P, C.c_double, _P, _P]
        L.sgo_pagerank_f64.argtypes = [C.c_uint32, _P, _P, C.c_double, _P, _P]
        L.sgo_bc_f32.argtypes = [C.c_uint32, _P, _P, C.c_uint32, _P, _P, _P]
        L.sgo_bc_f64.argtypes = [C.c_uint32, _P, _P, C.c_uint32, _P, _P, _P]
        L.sgo_rmat_edges.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_int,
                                     _P, _P]
        L.sgo_build_csr.argtypes = [C.c_uint32, C.c_uint64, _P, _P, C.c_int, C.c_int, _P, _P, C.POINTER(C.c_uint64)]
        L.sgo_gen_weights.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, _P]
        L.sgo_pick_sources.argtypes = [C.c_uint32, _P, C.c_uint32, C.c_uint64, _P]
        L.sgo_dijkstra.argtypes = [C.c_uint32, _P, _P, _P, C.c_uint32, _P]
        L.sgo_pagerank_jacobi_f64.argtypes = [C.c_uint32, _P, _P, C.c_double, C.c_uint32, _P, C.POINTER(C.c_uint32)]
        _o = L
    return _o


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref() -> C.CDLL:
    global _r
    if _r is None:
        L = C.CDLL(REF_LIB)
        L.sgref_bfs.argtypes = [C.c_uint32, C.c_uint32, _P, _P, C.c_uint32, _P]
        L.sgref_bfs_check.argtypes = [C.c_uint32, _P, _P]
        L.sgref_sssp.argtypes = [C.c_uint32, C.c_uint32, _P, _P, _P, C.c_uint32, _P]
        L.sgref_sssp_check.argtypes = [C.c_uint32, _P, _P]
        L.sgref_pagerank.argtypes = [C.c_uint32, C.c_uint32, _P, _P, C.c_double, _P]
        L.sgref_pagerank_check.argtypes = [C.c_uint32, _P, _P, C.c_int]
        L.sgref_bc.argtypes = [C.c_uint32, C.c_uint32, _P, _P, C.c_uint32, _P, _P]
        L.sgref_bc_check.argtypes = [C.c_uint32, _P, _P]
        L.sgref_csr_tocsc.argtypes = [C.c_uint32, C.c_uint32, _P, _P, _P, _P, _P, _P]
        _r = L
    return _r


def _p(a):
    return a.ctypes.data if a is not None else None


# ---------------------------------------------------------------- restatement
def bfs(offsets, indices, src):
    o, i = _u32(offsets), _u32(indices)
    out = np.empty(len(o) - 1, np.uint32)
    assert lib().sgo_bfs(len(o) - 1, _p(o), _p(i), src, _p(out)) == 0
    return out


def sssp(offsets, indices, weights, src):
    o, i = _u32(offsets), _u32(indices)
    w = _u32(weights) if weights is not None else None
    out = np.empty(len(o) - 1, np.uint32)
    assert lib().sgo_sssp(len(o) - 1, _p(o), _p(i), _p(w), src, _p(out)) == 0
    return out


def pagerank_f32(offsets, indices, error):
    o, i = _u32(offsets), _u32(indices)
    out = np.empty(len(o) - 1, np.float32)
    it = C.c_uint32()
    assert lib().sgo_pagerank_f32(len(o) - 1, _p(o), _p(i), error, _p(out), C.byref(it)) == 0
    return out


def pagerank_f64(offsets, indices, error):
    o, i = _u32(offsets), _u32(indices)
    out = np.empty(len(o) - 1, np.float64)
    it = C.c_uint32()
    assert lib().sgo_pagerank_f64(len(o) - 1, _p(o), _p(i), error, _p(out), C.byref(it)) == 0
    return out


def bc_f32(offsets, indices, src):
    o, i = _u32(offsets), _u32(indices)
    n = len(o) - 1
    bc, sg, lv = np.empty(n, np.float32), np.empty(n, np.float32), np.empty(n, np.uint32)
    assert lib().sgo_bc_f32(n, _p(o), _p(i), src, _p(bc), _p(sg), _p(lv)) == 0
    return bc, sg, lv


def bc_f64(offsets, indices, src):
    o, i = _u32(offsets), _u32(indices)
    n = len(o) - 1
    bc, sg, lv = np.empty(n, np.float64), np.empty(n, np.float64), np.empty(n, np.uint32)
    assert lib().sgo_bc_f64(n, _p(o), _p(i), src, _p(bc), _p(sg), _p(lv)) == 0
    return bc, sg, lv


# ---------------------------------------------------------------- full-size inputs and checkers
class Graph:
    """A CSR graph made by the oracle's generators (numpy arrays)."""

    def __init__(self, offsets, indices, weights=None):
        self.offsets, self.indices, self.weights = offsets, indices, weights
        self.nv, self.ne = len(offsets) - 1, len(indices)

    def max_degree_vertex(self):
        """GetMaxOutDgrNode (include/groute/graphs/csr_graph.h:241-259): lowest id among the maximum out-degree."""
        d = np.diff(self.offsets.astype(np.int64))
        v = int(np.argmax(d))
        return v, int(d[v])

    def pick_sources(self, n, seed):
        out = np.empty(n, np.uint32)
        assert lib().sgo_pick_sources(self.nv, _p(self.offsets), n, seed, _p(out)) == 0
        return out

    def gen_weights(self, lo, hi, seed):
        w = np.empty(self.ne, np.uint32)
        assert lib().sgo_gen_weights(self.ne, lo, hi, seed, _p(w)) == 0
        self.weights = w
        return self


def rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1, symmetric=False, keep_self_loops=False,
         keep_duplicates=False) -> Graph:
    """The seeded RMAT graph (the same CSR as the product library's generator, word for word)."""
    m = edge_factor << scale
    tot = 2 * m if symmetric else m
    src, dst = np.empty(tot, np.uint32), np.empty(tot, np.uint32)
    assert lib().sgo_rmat_edges(scale, edge_factor, a, b, c, seed, int(symmetric), _p(src), _p(dst)) == 0
    off = np.empty((1 << scale) + 1, np.uint32)
    ne = C.c_uint64()
    assert lib().sgo_build_csr(1 << scale, tot, _p(src), _p(dst), int(keep_self_loops), int(keep_duplicates),
                               _p(off), _p(dst_buf := np.empty(tot, np.uint32)), C.byref(ne)) == 0
    del src, dst
    return Graph(off, dst_buf[: ne.value].copy())


def grid(rows, cols) -> Graph:
    """4-neighbour grid, both directions, each row's neighbours in increasing id order."""
    nv = rows * cols
    v = np.arange(nv, dtype=np.int64)
    r, c = v // cols, v % cols
    nb = np.stack([np.where(r > 0, v - cols, -1), np.where(c > 0, v - 1, -1),
                   np.where(c + 1 < cols, v + 1, -1), np.where(r + 1 < rows, v + cols, -1)], axis=1)
    ok = nb >= 0
    off = np.zeros(nv + 1, np.uint32)
    off[1:] = np.cumsum(ok.sum(axis=1))
    return Graph(off, nb[ok].astype(np.uint32))


def dijkstra(offsets, indices, weights, src):
    """Shortest-path distances (unique for uint32 weights: what SSSPHostNaive returns)."""
    o, i = _u32(offsets), _u32(indices)
    w = _u32(weights) if weights is not None else None
    out = np.empty(len(o) - 1, np.uint32)
    assert lib().sgo_dijkstra(len(o) - 1, _p(o), _p(i), _p(w), src, _p(out)) == 0
    return out


def pagerank_fixed_point_f64(offsets, indices, tol=1e-13, max_iter=2000):
    """PageRankHost's fixed point in double, by parallel Jacobi sweeps; returns (ranks, sweeps)."""
    o, i = _u32(offsets), _u32(indices)
    out = np.empty(len(o) - 1, np.float64)
    it = C.c_uint32()
    assert lib().sgo_pagerank_jacobi_f64(len(o) - 1, _p(o), _p(i), tol, max_iter, _p(out), C.byref(it)) == 0
    return out, it.value


def host_threads() -> int:
    return int(lib().sgo_threads())


# ---------------------------------------------------------------- graph construction
def csr_tocsc(offsets, indices, weights=None):
    """CSR -> CSC as csr_tocsc builds it (include/groute/graphs/csr_graph.h:329-397):
    a stable counting sort of the edges by destination, so each in-edge list is
    ordered by source and parallel edges keep their CSR order."""
    o, i = _u32(offsets), _u32(indices)
    n = len(o) - 1
    src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(o.astype(np.int64)))
    order = np.argsort(i, kind="stable")
    coff = np.zeros(n + 1, np.uint32)
    coff[1:] = np.cumsum(np.bincount(i, minlength=n))
    return coff, src[order], (None if weights is None else _u32(weights)[order])


def gtools_build(nv, src, dst, weights=None, deself_cycle=False, deduplicate=False, d2ud=False,
                 sort_rows=False):
    """Edge list -> CSR under the reference converter's options
    (samples/tools/gtools.cpp:56-328), applied to the CSR whose rows hold each
    source's edges in input order:
      --deself_cycle (56-128): drop u->u, order kept;
      --deduplicate (130-197): per source keep the first edge to each
        destination (with its weight), order kept;
      --d2ud (199-328): in CSR order every edge (u, v, w) inserts v:w into u's
        map, then u:w into v's map, first insert wins; rows come out sorted by
        destination.
    sort_rows (not a converter option) orders rows by destination, CSR order
    among equal destinations.  Returns (offsets, indices, weights or None)."""
    s, d = _u32(src).astype(np.int64), _u32(dst).astype(np.int64)
    w = None if weights is None else _u32(weights)
    idx = np.arange(len(s))
    if deself_cycle:
        idx = idx[s[idx] != d[idx]]
    idx = idx[np.argsort(s[idx], kind="stable")]  # CSR order
    if deduplicate:
        rank = np.arange(len(idx))
        order = np.lexsort((rank, d[idx], s[idx]))
        so, do = s[idx][order], d[idx][order]
        first = np.ones(len(order), bool)
        first[1:] = (so[1:] != so[:-1]) | (do[1:] != do[:-1])
        idx = idx[np.sort(order[first])]
    rows, cols = s[idx], d[idx]
    ws = None if w is None else w[idx]
    if d2ud:
        r = np.arange(len(idx), dtype=np.int64)
        R, Cc, T = np.concatenate([rows, cols]), np.concatenate([cols, rows]), np.concatenate([2 * r, 2 * r + 1])
        order = np.lexsort((T, Cc, R))
        R, Cc = R[order], Cc[order]
        first = np.ones(len(order), bool)
        first[1:] = (R[1:] != R[:-1]) | (Cc[1:] != Cc[:-1])
        rows, cols = R[first], Cc[first]
        if ws is not None:
            ws = np.concatenate([ws, ws])[order][first]
    elif sort_rows:
        order = np.lexsort((np.arange(len(rows)), cols, rows))
        rows, cols = rows[order], cols[order]
        if ws is not None:
            ws = ws[order]
    off = np.zeros(nv + 1, np.uint32)
    off[1:] = np.cumsum(np.bincount(rows, minlength=nv))
    return off, cols.astype(np.uint32), (None if ws is None else ws.astype(np.uint32))


# ---------------------------------------------------------------- reference (compiled)
def ref_bfs(offsets, indices, src):
    o, i = _u32(offsets), _u32(indices)
    out = np.empty(len(o) - 1, np.uint32)
    ref().sgref_bfs(len(o) - 1, len(i), _p(o), _p(i), src, _p(out))
    return out


def ref_sssp(offsets, indices, weights, src):
    o, i, w = _u32(offsets), _u32(indices), _u32(weights)
    out = np.empty(len(o) - 1, np.uint32)
    ref().sgref_sssp(len(o) - 1, len(i), _p(o), _p(i), _p(w), src, _p(out))
    return out


def ref_pagerank(offsets, indices, error):
    o, i = _u32(offsets), _u32(indices)
    out = np.empty(len(o) - 1, np.float32)
    ref().sgref_pagerank(len(o) - 1, len(i), _p(o), _p(i), error, _p(out))
    return out


def ref_pagerank_check(ranks, regression, norm=False) -> int:
    a = np.ascontiguousarray(ranks, np.float32)
    b = np.ascontiguousarray(regression, np.float32)
    return ref().sgref_pagerank_check(len(a), _p(a), _p(b), int(norm))


def ref_bc(offsets, indices, src):
    o, i = _u32(offsets), _u32(indices)
    n = len(o) - 1
    bc, sg = np.empty(n, np.float32), np.empty(n, np.float32)
    ref().sgref_bc(n, len(i), _p(o), _p(i), src, _p(bc), _p(sg))
    return bc, sg


def ref_bc_check(regression, values) -> int:
    a = np.ascontiguousarray(regression, np.float32)
    b = np.ascontiguousarray(values, np.float32)
    return ref().sgref_bc_check(len(a), _p(a), _p(b))


def ref_csr_tocsc(offsets, indices, weights=None):
    """The reference's own CSCGraph(csr, undirected=false) construction."""
    o, i = _u32(offsets), _u32(indices)
    w = None if weights is None else _u32(weights)
    n, m = len(o) - 1, len(i)
    co, ci = np.empty(n + 1, np.uint32), np.empty(m, np.uint32)
    cw = None if w is None else np.empty(m, np.uint32)
    ref().sgref_csr_tocsc(n, m, _p(o), _p(i), _p(w), _p(co), _p(ci), _p(cw))
    return co, ci, cw


REF_GTOOLS = os.path.join(_HERE, "_ref", "gtools")


def ref_gtools_available() -> bool:
    return os.path.exists(REF_GTOOLS)


def ref_gtools(gr_path, out_path, deself_cycle=False, deduplicate=True, d2ud=False, fmt="gr"):
    """Runs the reference's converter (samples/tools/gtools.cpp, built by
    `make -C oracle ref`) on a graph file (Galois .gr, or MatrixMarket with
    fmt="market"); returns its edge list as (src, dst, weights or None) arrays
    in output order."""
    b = lambda x: "true" if x else "false"
    subprocess.run([REF_GTOOLS, f"--graphfile={gr_path}", f"--format={fmt}", f"--output={out_path}",
                    f"--deself_cycle={b(deself_cycle)}", f"--deduplicate={b(deduplicate)}", f"--d2ud={b(d2ud)}"],
                   check=True, capture_output=True)
    rows = np.loadtxt(out_path, dtype=np.int64, ndmin=2) if os.path.getsize(out_path) else np.zeros((0, 2))
    if rows.size == 0:
        return np.zeros(0, np.uint32), np.zeros(0, np.uint32), None
    w = rows[:, 2].astype(np.uint32) if rows.shape[1] > 2 else None
    return rows[:, 0].astype(np.uint32), rows[:, 1].astype(np.uint32), w
