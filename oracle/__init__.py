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
