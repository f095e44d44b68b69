"""Python binding of libsepgraph_b200.so (the C ABI in include/sepgraph.h).

Thin ctypes layer used by the tests, bench.py and scripts: host graphs are
numpy views of the library's own buffers; device work goes through the C
entry points only.  There is no Python or CPU fallback: if the shared
library is missing, ``load()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsepgraph_b200.so")

SG_OK = 0
STATUS_NAMES = {
    0: "SG_OK", 1: "SG_ERR_INVALID_ARG", 2: "SG_ERR_CUDA", 3: "SG_ERR_OUT_OF_MEMORY", 4: "SG_ERR_TIMEOUT",
    5: "SG_ERR_CAPACITY", 6: "SG_ERR_UNSUPPORTED", 7: "SG_ERR_OVERFLOW", 8: "SG_ERR_NO_DEVICE", 9: "SG_ERR_IO",
    10: "SG_ERR_FORMAT", 11: "SG_ERR_BUSY",
}

# selectors (include/sepgraph.h)
LB = {"auto": -1, "none": 0, "coarse": 1, "fine": 2, "hybrid": 3}
VARIANTS = {
    "auto": -1, "sync_push_td": 0, "sync_push_dd": 1, "sync_pull_td": 2, "sync_pull_dd": 3,
    "async_push_td": 4, "async_push_dd": 5, "async_pull_td": 6, "async_pull_dd": 7,
}
VARIANT_NAMES = {v: k.upper() for k, v in VARIANTS.items() if v >= 0}
GRAPH_SYMMETRIC = 0x1
GRAPH_NO_CSC = 0x2
BUILD_DESELF_CYCLE = 0x1  # sg_graph_build flags (the reference converter's options)
BUILD_DEDUPLICATE = 0x2
BUILD_D2UD = 0x4
BUILD_SORT_ROWS = 0x8
GEN_SYMMETRIC = 0x1
GEN_KEEP_SELF_LOOPS = 0x2
GEN_KEEP_DUPLICATES = 0x4
INF = 0xFFFFFFFF


class SGError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)} {detail}".strip())


class Options(C.Structure):
    _fields_ = [
        ("variant", C.c_int32), ("lb_push", C.c_int32), ("lb_pull", C.c_int32), ("priority", C.c_int32),
        ("priority_delta", C.c_double), ("cut_threshold", C.c_double), ("alpha", C.c_double),
        ("beta", C.c_double), ("edge_factor", C.c_double), ("max_iteration", C.c_int32), ("fused", C.c_int32),
        ("block_size", C.c_int32), ("non_atomic", C.c_int32), ("trace", C.c_int32), ("pr_error", C.c_double),
        ("timeout_s", C.c_double), ("blocking", C.c_int32), ("blocks_per_sm", C.c_int32),
        ("heavy_degree", C.c_int32), ("chunk_edges", C.c_int32), ("team_blocks", C.c_int32),
        ("local_depth", C.c_int32), ("wl_sort", C.c_int32), ("worklist", C.c_int32),
        ("l2_persist", C.c_int32), ("pull_scan", C.c_int32), ("hub_stage", C.c_int32), ("reserved", C.c_int32 * 1),
    ]


class TuneEntry(C.Structure):
    _fields_ = [("options", Options), ("ms", C.c_double), ("status", C.c_int32), ("pad", C.c_int32)]


TUNED_FIELDS = ("variant", "blocks_per_sm", "heavy_degree", "chunk_edges", "priority", "priority_delta", "lb_push",
                "local_depth", "worklist", "pull_scan")
VARIANT_NAMES = {-1: "auto", 0: "sync_push_td", 1: "sync_push_dd", 2: "sync_pull_td", 3: "sync_pull_dd",
                 4: "async_push_td", 5: "async_push_dd", 6: "async_pull_td", 7: "async_pull_dd"}


def options_dict(o: Options, fields=TUNED_FIELDS) -> dict:
    d = {k: getattr(o, k) for k in fields}
    if "variant" in d:
        d["variant"] = VARIANT_NAMES.get(d["variant"], d["variant"])
    if d.get("priority") == 0:
        d.pop("priority")
        d.pop("priority_delta", None)
    elif "priority" in d:
        d["priority"] = {1: "low_high", 2: "sampling"}.get(d["priority"], d["priority"])
    return d


class RoundTrace(C.Structure):
    _fields_ = [
        ("round", C.c_uint32), ("variant", C.c_int32), ("in_nodes", C.c_uint32), ("out_nodes", C.c_uint32),
        ("in_workload", C.c_uint64), ("out_workload", C.c_uint64), ("total_workload", C.c_int64),
        ("time_ms", C.c_float), ("pad", C.c_uint32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("rounds", C.c_uint32), ("max_iteration_reached", C.c_uint32), ("rounds_by_variant", C.c_uint32 * 8),
        ("time_total_ms", C.c_double), ("time_kernel_ms", C.c_double), ("edges_processed", C.c_uint64),
        ("vertices_processed", C.c_uint64), ("edges_reached", C.c_uint64), ("vertices_reached", C.c_uint32),
        ("search_depth", C.c_uint32), ("device_error", C.c_uint32), ("n_trace", C.c_uint32),
        ("trace", C.POINTER(RoundTrace)), ("trace_capacity", C.c_uint32), ("pad", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("trace", "pad", "rounds_by_variant")}
        d["rounds_by_variant"] = {VARIANT_NAMES[i]: int(self.rounds_by_variant[i]) for i in range(8)
                                  if self.rounds_by_variant[i]}
        return d


class BatchQuery(C.Structure):
    _fields_ = [("graph", C.c_void_p), ("source", C.c_uint32), ("pad", C.c_uint32), ("out", C.c_void_p)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("slots", C.c_uint32), ("max_batch", C.c_uint32),
                ("max_pending", C.c_uint32), ("msbfs_min", C.c_uint32), ("sssp_delta", C.c_uint32),
                ("pad", C.c_uint32), ("pr_error", C.c_double), ("batch_graphs", C.c_int32),
                ("order", C.c_int32), ("max_wait_ms", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("reserved", C.c_int32 * 4)]


class Query(C.Structure):
    _fields_ = [("algo", C.c_int32), ("graph_id", C.c_uint32), ("source", C.c_uint32), ("pad", C.c_uint32),
                ("out", C.c_void_p), ("out2", C.c_void_p)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("batches", C.c_uint64), ("pending", C.c_uint64), ("elapsed_s", C.c_double), ("qps", C.c_double),
                ("mean_ms", C.c_double), ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("p999_ms", C.c_double),
                ("max_ms", C.c_double), ("hbm_budget", C.c_uint64), ("hbm_in_use", C.c_uint64),
                ("hbm_peak", C.c_uint64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


QUERY_ALGOS = {"bfs": 0, "sssp": 1, "pagerank": 2, "bc": 3}


_lib = None
_P = C.c_void_p
_U32P = C.POINTER(C.c_uint32)


def load() -> C.CDLL:
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} not built (run make -C sep-graph_b200)")
    L = C.CDLL(LIB_PATH)
    sig = {
        "sg_status_string": (C.c_char_p, [C.c_int]),
        "sg_abi_version": (C.c_int, []),
        "sg_init": (C.c_int, [C.c_int, C.POINTER(_P)]),
        "sg_destroy": (C.c_int, [_P]),
        "sg_ctx_set_stream": (C.c_int, [_P, _P]),
        "sg_ctx_get_stream": (C.c_int, [_P, C.POINTER(_P)]),
        "sg_ctx_synchronize": (C.c_int, [_P]),
        "sg_ctx_release_cached": (C.c_int, [_P]),
        "sg_last_error": (C.c_char_p, [_P]),
        "sg_device_info": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                     C.c_char_p, C.c_size_t]),
        "sg_graph_create": (C.c_int, [_P, C.c_uint32, C.c_uint64, _P, _P, _P, C.c_uint32, C.POINTER(_P)]),
        "sg_graph_create_from_host": (C.c_int, [_P, _P, C.c_uint32, C.POINTER(_P)]),
        "sg_graph_destroy": (C.c_int, [_P]),
        "sg_msbc": (C.c_int, [_P, _P, C.c_uint32, C.POINTER(Options), _P, C.POINTER(Stats)]),
        "sg_graph_build": (C.c_int, [_P, C.c_uint32, C.c_uint64, _P, _P, _P, C.c_uint32, C.c_uint32, C.POINTER(_P)]),
        "sg_graph_copy_out": (C.c_int, [_P, C.c_int, _P, _P, _P]),
        "sg_graph_info": (C.c_int, [_P, _U32P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                    C.POINTER(C.c_int)]),
        "sg_options_default": (C.c_int, [C.POINTER(Options)]),
        "sg_bfs": (C.c_int, [_P, C.c_uint32, C.POINTER(Options), _P, C.POINTER(Stats)]),
        "sg_sssp": (C.c_int, [_P, C.c_uint32, C.POINTER(Options), _P, C.POINTER(Stats)]),
        "sg_pagerank": (C.c_int, [_P, C.POINTER(Options), _P, _P, C.POINTER(Stats)]),
        "sg_bc": (C.c_int, [_P, C.c_uint32, C.POINTER(Options), _P, _P, C.POINTER(Stats)]),
        "sg_msbfs": (C.c_int, [_P, _U32P, C.c_uint32, C.POINTER(Options), _P, C.POINTER(Stats)]),
        "sg_sssp_batch": (C.c_int, [_P, C.POINTER(BatchQuery), C.c_uint32, C.POINTER(Options), C.POINTER(Stats),
                                    C.POINTER(C.c_float)]),
        "sg_bfs_batch": (C.c_int, [_P, C.POINTER(BatchQuery), C.c_uint32, C.POINTER(Options), C.POINTER(Stats),
                                   C.POINTER(C.c_float)]),
        "sg_bc_batch": (C.c_int, [_P, C.POINTER(BatchQuery), C.c_uint32, C.POINTER(Options), C.POINTER(Stats),
                                  C.POINTER(C.c_float)]),
        "sg_batch_plan_create": (C.c_int, [_P, C.c_int, C.POINTER(BatchQuery), C.c_uint32, C.POINTER(Options),
                                           C.POINTER(_P)]),
        "sg_batch_plan_launch": (C.c_int, [_P]),
        "sg_batch_plan_wait": (C.c_int, [_P, C.POINTER(Stats), C.POINTER(C.c_float)]),
        "sg_batch_plan_captured": (C.c_int, [_P]),
        "sg_batch_plan_destroy": (C.c_int, [_P]),
        "sg_autotune": (C.c_int, [_P, C.c_int, _U32P, C.c_uint32, C.POINTER(Options), C.c_uint32,
                                  C.POINTER(Options), C.POINTER(C.c_double), C.POINTER(TuneEntry), C.c_uint32,
                                  C.POINTER(C.c_uint32)]),
        "sg_msbfs_on": (C.c_int, [_P, _P, _U32P, C.c_uint32, C.POINTER(Options), _P, C.POINTER(Stats)]),
        "sg_server_config_default": (C.c_int, [C.POINTER(ServerConfig)]),
        "sg_server_create": (C.c_int, [C.c_int, C.POINTER(ServerConfig), C.POINTER(_P)]),
        "sg_server_add_graph": (C.c_int, [_P, _P, _U32P]),
        "sg_server_submit": (C.c_int, [_P, C.POINTER(Query), C.POINTER(C.c_uint64)]),
        "sg_server_wait": (C.c_int, [_P, C.c_uint64, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
        "sg_server_drain": (C.c_int, [_P, C.c_double]),
        "sg_server_get_stats": (C.c_int, [_P, C.POINTER(ServerStats)]),
        "sg_server_reset_stats": (C.c_int, [_P]),
        "sg_server_destroy": (C.c_int, [_P]),
        "sg_hgraph_gen_rmat": (C.c_int, [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double,
                                         C.c_uint64, C.c_uint32, C.POINTER(_P)]),
        "sg_hgraph_gen_grid": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(_P)]),
        "sg_hgraph_gen_random": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(_P)]),
        "sg_hgraph_from_csr": (C.c_int, [C.c_uint32, C.c_uint64, _P, _P, _P, C.POINTER(_P)]),
        "sg_hgraph_gen_weights": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint64]),
        "sg_hgraph_read_gr": (C.c_int, [C.c_char_p, C.POINTER(_P)]),
        "sg_hgraph_write_gr": (C.c_int, [_P, C.c_char_p]),
        "sg_hgraph_read_market": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(_P)]),
        "sg_hgraph_read_metis": (C.c_int, [C.c_char_p, C.POINTER(_P)]),
        "sg_hgraph_info": (C.c_int, [_P, _U32P, C.POINTER(C.c_uint64), C.POINTER(_U32P), C.POINTER(_U32P),
                                     C.POINTER(_U32P)]),
        "sg_hgraph_max_degree_vertex": (C.c_int, [_P, _U32P, _U32P]),
        "sg_hgraph_pick_sources": (C.c_int, [_P, C.c_uint32, C.c_uint64, _U32P]),
        "sg_hgraph_destroy": (C.c_int, [_P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _check(st: int, where: str, ctx=None):
    if st != SG_OK:
        detail = ""
        if ctx is not None:
            detail = load().sg_last_error(ctx).decode(errors="replace")
        raise SGError(st, where, detail)


def _ptr(a) -> Optional[int]:
    """Address of a numpy array, an int device pointer, or a torch tensor."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    raise TypeError(type(a))


def _ptr32(a) -> Optional[int]:
    """_ptr for arrays the library reads as 32-bit words (indices, weights)."""
    if a is not None and not isinstance(a, int):
        size = a.itemsize if isinstance(a, np.ndarray) else a.element_size()
        if size != 4:
            raise TypeError(f"expected 32-bit elements, got {getattr(a, 'dtype', type(a))}")
        if hasattr(a, "is_contiguous") and not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
    return _ptr(a)


def make_options(**kw) -> Options:
    o = Options()
    _check(load().sg_options_default(C.byref(o)), "sg_options_default")
    for k, v in kw.items():
        if v is None:
            continue
        if k == "variant" and isinstance(v, str):
            v = VARIANTS[v.lower()]
        elif k in ("lb_push", "lb_pull") and isinstance(v, str):
            v = LB[v.lower()]
        elif k == "priority" and isinstance(v, str):
            v = {"none": 0, "low_high": 1, "sampling": 2}[v.lower()]
        if not hasattr(o, k):
            raise KeyError(f"unknown option {k}")
        setattr(o, k, int(v) if isinstance(v, bool) else v)
    return o


class HostGraph:
    """Host CSR graph owned by the library (generators and file I/O)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def rmat(cls, scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, seed: int = 1,
             symmetric: bool = False, keep_self_loops=False, keep_duplicates=False) -> "HostGraph":
        h = _P()
        flags = (GEN_SYMMETRIC if symmetric else 0) | (GEN_KEEP_SELF_LOOPS if keep_self_loops else 0) | \
            (GEN_KEEP_DUPLICATES if keep_duplicates else 0)
        _check(load().sg_hgraph_gen_rmat(scale, edge_factor, a, b, c, seed, flags, C.byref(h)), "gen_rmat")
        return cls(h)

    @classmethod
    def grid(cls, rows: int, cols: int) -> "HostGraph":
        h = _P()
        _check(load().sg_hgraph_gen_grid(rows, cols, 0, C.byref(h)), "gen_grid")
        return cls(h)

    @classmethod
    def random(cls, nv: int, gen_factor: int, seed: int = 1) -> "HostGraph":
        h = _P()
        _check(load().sg_hgraph_gen_random(nv, gen_factor, seed, C.byref(h)), "gen_random")
        return cls(h)

    @classmethod
    def from_csr(cls, offsets, indices, weights=None) -> "HostGraph":
        offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
        indices = np.ascontiguousarray(indices, dtype=np.uint32)
        if weights is not None:
            weights = np.ascontiguousarray(weights, dtype=np.uint32)
        h = _P()
        _check(load().sg_hgraph_from_csr(len(offsets) - 1, len(indices), _ptr(offsets), _ptr(indices),
                                         _ptr(weights), C.byref(h)), "from_csr")
        return cls(h)

    @classmethod
    def read_gr(cls, path: str) -> "HostGraph":
        h = _P()
        _check(load().sg_hgraph_read_gr(path.encode(), C.byref(h)), "read_gr")
        return cls(h)

    @classmethod
    def read_market(cls, path: str, symmetrize: bool = False) -> "HostGraph":
        h = _P()
        _check(load().sg_hgraph_read_market(path.encode(), int(symmetrize), C.byref(h)), "read_market")
        return cls(h)

    @classmethod
    def read_metis(cls, path: str) -> "HostGraph":
        h = _P()
        _check(load().sg_hgraph_read_metis(path.encode(), C.byref(h)), "read_metis")
        return cls(h)

    def write_gr(self, path: str):
        _check(load().sg_hgraph_write_gr(self._h, path.encode()), "write_gr")

    def gen_weights(self, lo: int, hi: int, seed: int = 2) -> "HostGraph":
        _check(load().sg_hgraph_gen_weights(self._h, lo, hi, seed), "gen_weights")
        return self

    def _info(self):
        nv, ne = C.c_uint32(), C.c_uint64()
        o, i, w = _U32P(), _U32P(), _U32P()
        _check(load().sg_hgraph_info(self._h, C.byref(nv), C.byref(ne), C.byref(o), C.byref(i), C.byref(w)),
               "hgraph_info")
        return nv.value, ne.value, o, i, w

    @property
    def nv(self) -> int:
        return self._info()[0]

    @property
    def ne(self) -> int:
        return self._info()[1]

    @property
    def offsets(self) -> np.ndarray:
        nv, ne, o, _, _ = self._info()
        return np.ctypeslib.as_array(o, shape=(nv + 1,))

    @property
    def indices(self) -> np.ndarray:
        nv, ne, _, i, _ = self._info()
        return np.ctypeslib.as_array(i, shape=(ne,)) if ne else np.zeros(0, np.uint32)

    @property
    def weights(self) -> Optional[np.ndarray]:
        nv, ne, _, _, w = self._info()
        if not w:
            return None
        return np.ctypeslib.as_array(w, shape=(ne,)) if ne else np.zeros(0, np.uint32)

    def max_degree_vertex(self):
        v, d = C.c_uint32(), C.c_uint32()
        _check(load().sg_hgraph_max_degree_vertex(self._h, C.byref(v), C.byref(d)), "max_degree_vertex")
        return v.value, d.value

    def pick_sources(self, n: int, seed: int = 3) -> np.ndarray:
        out = np.zeros(n, np.uint32)
        _check(load().sg_hgraph_pick_sources(self._h, n, seed, out.ctypes.data_as(_U32P)), "pick_sources")
        return out

    def close(self):
        if self._h:
            load().sg_hgraph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One CUDA device + stream (sg_ctx)."""

    def __init__(self, device: int = 0):
        self._c = _P()
        self._graphs = weakref.WeakSet()
        self._plans = weakref.WeakSet()
        _check(load().sg_init(device, C.byref(self._c)), "sg_init")
        self.device = device

    @property
    def handle(self):
        return self._c

    @property
    def stream(self) -> int:
        s = _P()
        _check(load().sg_ctx_get_stream(self._c, C.byref(s)), "get_stream", self._c)
        return s.value or 0

    def set_stream(self, stream_ptr: Optional[int]):
        _check(load().sg_ctx_set_stream(self._c, stream_ptr), "set_stream", self._c)

    def synchronize(self):
        _check(load().sg_ctx_synchronize(self._c), "synchronize", self._c)

    def device_info(self) -> dict:
        sm, hbm, l2 = C.c_int(), C.c_uint64(), C.c_uint64()
        name = C.create_string_buffer(256)
        _check(load().sg_device_info(self._c, C.byref(sm), C.byref(hbm), C.byref(l2), name, 256), "device_info")
        return {"sm_count": sm.value, "hbm_bytes": hbm.value, "l2_bytes": l2.value, "name": name.value.decode()}

    def _batch(self, fn, name, queries, outs, team_blocks, opts, dtype=np.uint32):
        n = len(queries)
        arr = (BatchQuery * n)()
        if outs is None:
            outs = [np.empty(g.nv, dtype) for g, _ in queries]
        for i, ((g, s), o) in enumerate(zip(queries, outs)):
            arr[i].graph = g.handle
            arr[i].source = int(s)
            arr[i].out = _ptr(o)
        o = make_options(**opts)
        if team_blocks:
            o.team_blocks = int(team_blocks)
        st = Stats()
        per = (C.c_float * n)()
        _check(fn(self._c, arr, n, C.byref(o), C.byref(st), per), name, self._c)
        return outs, st, list(per)

    def sssp_batch(self, queries, outs=None, team_blocks: int = 0, **opts):
        """queries: list of (Graph, source).  One launch; returns (outputs, stats, per-query ms)."""
        return self._batch(load().sg_sssp_batch, "sg_sssp_batch", queries, outs, team_blocks, opts)

    def bfs_batch(self, queries, outs=None, team_blocks: int = 0, **opts):
        return self._batch(load().sg_bfs_batch, "sg_bfs_batch", queries, outs, team_blocks, opts)

    def batch_plan(self, algo: str, queries, outs, team_blocks: int = 0, **opts) -> "BatchPlan":
        """Plans queries [(Graph, source)] of `algo` ("bfs", "sssp", "bc") once for repeated launches
        (sg_batch_plan_*); outs are device arrays (e.g. torch CUDA tensors) of each graph's nv elements."""
        return BatchPlan(self, algo, queries, outs, team_blocks, opts)

    def bc_batch(self, queries, outs=None, team_blocks: int = 0, **opts):
        """Single-source BC of every (Graph, source) in one launch; outputs are float32 arrays."""
        return self._batch(load().sg_bc_batch, "sg_bc_batch", queries, outs, team_blocks, opts, np.float32)

    def graph(self, hg: HostGraph, symmetric: bool = False, no_csc: bool = False) -> "Graph":
        g = _P()
        flags = (GRAPH_SYMMETRIC if symmetric else 0) | (GRAPH_NO_CSC if no_csc else 0)
        _check(load().sg_graph_create_from_host(self._c, hg._h, flags, C.byref(g)), "graph_create", self._c)
        return Graph(self, g)

    def graph_from_csr(self, offsets, indices, weights=None, symmetric=False, no_csc=False, nv=None,
                       ne=None) -> "Graph":
        """Arrays may be numpy (host), torch tensors, or raw int pointers (then pass nv and ne)."""
        g = _P()
        flags = (GRAPH_SYMMETRIC if symmetric else 0) | (GRAPH_NO_CSC if no_csc else 0)
        if nv is None:
            nv = len(offsets) - 1
        if ne is None:
            ne = len(indices)
        _check(load().sg_graph_create(self._c, nv, ne, _ptr32(offsets), _ptr32(indices), _ptr32(weights), flags,
                                      C.byref(g)), "graph_create", self._c)
        return Graph(self, g)

    def build_graph(self, nv: int, src, dst, weights=None, deself_cycle=False, deduplicate=False, d2ud=False,
                    sort_rows=False, symmetric=False, no_csc=False, m=None) -> "Graph":
        """Edge list -> device graph built on the GPU (sg_graph_build); the flags are the
        reference converter's --deself_cycle / --deduplicate / --d2ud plus row ordering.
        Arrays may be numpy (converted to uint32), torch tensors, or int device pointers
        (then pass m)."""
        def u32(a):
            return np.ascontiguousarray(a, dtype=np.uint32) if isinstance(a, (np.ndarray, list, tuple)) else a
        src, dst, weights = u32(src), u32(dst), u32(weights)
        if m is None:
            m = len(src)
        bflags = ((BUILD_DESELF_CYCLE if deself_cycle else 0) | (BUILD_DEDUPLICATE if deduplicate else 0)
                  | (BUILD_D2UD if d2ud else 0) | (BUILD_SORT_ROWS if sort_rows else 0))
        gflags = (GRAPH_SYMMETRIC if symmetric else 0) | (GRAPH_NO_CSC if no_csc else 0)
        g = _P()
        _check(load().sg_graph_build(self._c, nv, m, _ptr32(src), _ptr32(dst), _ptr32(weights), bflags, gflags,
                                     C.byref(g)), "sg_graph_build", self._c)
        return Graph(self, g)

    def release_cached(self):
        """Frees the context's cached device memory (spare graph arena, call scratch)."""
        _check(load().sg_ctx_release_cached(self._c), "sg_ctx_release_cached", self._c)

    def close(self):
        """Releases the context; graphs still open on it are released first."""
        if self._c:
            for p in list(self._plans):  # plans hold graphs and the context's stream
                p.close()
            for g in list(self._graphs):
                g.close()
            load().sg_destroy(self._c)
            self._c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchPlan:
    """A batch planned once; each launch replays one CUDA graph (see sg_batch_plan_create)."""

    def __init__(self, ctx, algo, queries, outs, team_blocks, opts):
        n = len(queries)
        arr = (BatchQuery * n)()
        for i, ((g, s), o) in enumerate(zip(queries, outs)):
            arr[i].graph = g.handle
            arr[i].source = int(s)
            arr[i].out = _ptr(o)
        o = make_options(**opts)
        if team_blocks:
            o.team_blocks = int(team_blocks)
        self.ctx, self.n, self._outs = ctx, n, list(outs)
        self._p = _P()
        _check(load().sg_batch_plan_create(ctx.handle, QUERY_ALGOS[algo], arr, n, C.byref(o), C.byref(self._p)),
               "sg_batch_plan_create", ctx.handle)
        ctx._plans.add(self)

    @property
    def captured(self) -> bool:
        return bool(load().sg_batch_plan_captured(self._p))

    def launch(self):
        _check(load().sg_batch_plan_launch(self._p), "sg_batch_plan_launch", self.ctx.handle)

    def wait(self):
        st = Stats()
        per = (C.c_float * self.n)()
        _check(load().sg_batch_plan_wait(self._p, C.byref(st), per), "sg_batch_plan_wait", self.ctx.handle)
        return st, list(per)

    def close(self):
        if self._p:
            load().sg_batch_plan_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching query server (sg_server_*)."""

    def __init__(self, device: int = 0, **cfg):
        c = ServerConfig()
        _check(load().sg_server_config_default(C.byref(c)), "server_config_default")
        for k, v in cfg.items():
            setattr(c, k, v)
        self._s = _P()
        _check(load().sg_server_create(device, C.byref(c), C.byref(self._s)), "sg_server_create")
        self._keep = {}

    def add_graph(self, g: "Graph") -> int:
        gid = C.c_uint32()
        _check(load().sg_server_add_graph(self._s, g.handle, C.byref(gid)), "sg_server_add_graph")
        return gid.value

    def submit(self, algo: str, graph_id: int, source: int, out, out2=None) -> int:
        q = Query(QUERY_ALGOS[algo], graph_id, source, 0, _ptr(out), _ptr(out2))
        t = C.c_uint64()
        _check(load().sg_server_submit(self._s, C.byref(q), C.byref(t)), "sg_server_submit")
        self._keep[t.value] = (out, out2)  # host buffers must outlive the query
        return t.value

    def wait(self, ticket: int, timeout_s: float = 600.0):
        st, lat = C.c_int(), C.c_double()
        _check(load().sg_server_wait(self._s, ticket, timeout_s, C.byref(st), C.byref(lat)), "sg_server_wait")
        self._keep.pop(ticket, None)
        return st.value, lat.value

    def drain(self, timeout_s: float = 600.0):
        _check(load().sg_server_drain(self._s, timeout_s), "sg_server_drain")

    def stats(self) -> dict:
        s = ServerStats()
        _check(load().sg_server_get_stats(self._s, C.byref(s)), "sg_server_get_stats")
        return s.as_dict()

    def reset_stats(self):
        _check(load().sg_server_reset_stats(self._s), "sg_server_reset_stats")

    def close(self):
        if self._s:
            load().sg_server_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Graph:
    """Device-resident graph (sg_graph) and the four algorithms."""

    def __init__(self, ctx: Context, handle):
        self.ctx = ctx
        self._g = handle
        ctx._graphs.add(self)

    @property
    def handle(self):
        return self._g

    def info(self) -> dict:
        nv, ne, b, w = C.c_uint32(), C.c_uint64(), C.c_uint64(), C.c_int()
        _check(load().sg_graph_info(self._g, C.byref(nv), C.byref(ne), C.byref(b), C.byref(w)), "graph_info")
        return {"nv": nv.value, "ne": ne.value, "device_bytes": b.value, "weighted": bool(w.value)}

    @property
    def nv(self) -> int:
        return self.info()["nv"]

    def copy_out(self, csc: bool = False):
        """(offsets, indices, weights or None) of the CSR, or of the in-edge CSC view."""
        inf = self.info()
        off = np.empty(inf["nv"] + 1, np.uint32)
        idx = np.empty(inf["ne"], np.uint32)
        w = np.empty(inf["ne"], np.uint32) if inf["weighted"] else None
        _check(load().sg_graph_copy_out(self._g, 1 if csc else 0, _ptr(off), _ptr(idx), _ptr(w)),
               "sg_graph_copy_out", self.ctx.handle)
        return off, idx, w

    def _stats(self, trace_capacity: int):
        st = Stats()
        buf = None
        if trace_capacity:
            buf = (RoundTrace * trace_capacity)()
            st.trace = C.cast(buf, C.POINTER(RoundTrace))
            st.trace_capacity = trace_capacity
        return st, buf

    @staticmethod
    def _trace(buf, st):
        if buf is None:
            return None
        return [{k: getattr(buf[i], k) for k, _ in RoundTrace._fields_ if k != "pad"} for i in range(st.n_trace)]

    def _prep(self, out, dtype, trace_capacity, opts):
        o = make_options(**opts)
        if trace_capacity:
            o.trace = 1
        if out is None:
            out = np.empty(self.nv, dtype)
        st, buf = self._stats(trace_capacity)
        return o, out, st, buf

    def bfs(self, source: int, out=None, trace_capacity: int = 0, **opts):
        o, out, st, buf = self._prep(out, np.uint32, trace_capacity, opts)
        _check(load().sg_bfs(self._g, source, C.byref(o), _ptr(out), C.byref(st)), "sg_bfs", self.ctx.handle)
        return out, st, self._trace(buf, st)

    def sssp(self, source: int, out=None, trace_capacity: int = 0, **opts):
        o, out, st, buf = self._prep(out, np.uint32, trace_capacity, opts)
        _check(load().sg_sssp(self._g, source, C.byref(o), _ptr(out), C.byref(st)), "sg_sssp", self.ctx.handle)
        return out, st, self._trace(buf, st)

    def pagerank(self, out=None, residual_out=None, trace_capacity: int = 0, **opts):
        o, out, st, buf = self._prep(out, np.float32, trace_capacity, opts)
        _check(load().sg_pagerank(self._g, C.byref(o), _ptr(out), _ptr(residual_out), C.byref(st)), "sg_pagerank",
               self.ctx.handle)
        return out, st, self._trace(buf, st)

    def autotune(self, algo: str, sources=(), max_candidates: int = 0, **base_opts):
        """Times the library's candidate options for `algo` on these sources (sg_autotune).

        Returns (best options as a dict of keyword arguments, best ms, report)."""
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        base = make_options(**base_opts)
        best, best_ms = Options(), C.c_double()
        rep = (TuneEntry * 64)()
        n = C.c_uint32()
        _check(load().sg_autotune(self._g, QUERY_ALGOS[algo], src.ctypes.data_as(_U32P), len(src), C.byref(base),
                                  max_candidates, C.byref(best), C.byref(best_ms), rep, 64, C.byref(n)),
               "sg_autotune", self.ctx.handle)
        report = [dict(options_dict(rep[i].options), ms=rep[i].ms, status=rep[i].status) for i in range(n.value)]
        return options_dict(best), best_ms.value, report

    def msbfs(self, sources, out=None, **opts):
        """BFS from up to 64 sources in one launch; returns (levels[nsrc, nv], stats)."""
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        o = make_options(**opts)
        if out is None:
            out = np.empty((len(src), self.nv), np.uint32)
        st = Stats()
        _check(load().sg_msbfs(self._g, src.ctypes.data_as(_U32P), len(src), C.byref(o), _ptr(out), C.byref(st)),
               "sg_msbfs", self.ctx.handle)
        return out, st

    def msbc(self, sources, out=None, **opts):
        """Betweenness centrality from up to 32 sources in one launch; returns (bc[nsrc, nv], stats)."""
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        o = make_options(**opts)
        if out is None:
            out = np.empty((len(src), self.nv), np.float32)
        st = Stats()
        _check(load().sg_msbc(self._g, src.ctypes.data, len(src), C.byref(o), _ptr(out), C.byref(st)),
               "sg_msbc", self.ctx.handle)
        return out, st

    def bc(self, source: int, out=None, sigma_out=None, trace_capacity: int = 0, **opts):
        o = make_options(**opts)
        if trace_capacity:
            o.trace = 1
        if out is None:
            out = np.empty(self.nv, np.float32)
        if sigma_out is None:
            sigma_out = np.empty(self.nv, np.uint64)
        st, buf = self._stats(trace_capacity)
        _check(load().sg_bc(self._g, source, C.byref(o), _ptr(out), _ptr(sigma_out), C.byref(st)), "sg_bc",
               self.ctx.handle)
        return out, sigma_out, st

    def close(self):
        if self._g:
            load().sg_graph_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
