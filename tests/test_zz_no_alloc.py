"""sg_bfs_noalloc: BFS for callers that cannot allocate device memory.

Callers inside another framework's memory pool, or under a device-memory
budget that forbids new allocations, cannot let the library cudaMalloc its
worklists.  sg_bfs_noalloc runs the same engine with all scratch in a fixed
file-scope device array.  This test calls it through the C ABI on device
arrays the test owns and checks its levels against the allocating sg_bfs,
bit for bit (BFS levels are integers), on two calls in a row, plus the size
limit; with default options it must also run the same rounds as sg_bfs (same
load balancing and block count), at the largest graph the fixed array takes
(hub chunks included), push-only (no in-edge arrays) and with explicit
options, and after the first call no call may change the device's free
memory.  Collected last so that a failure here comes after every other test.
"""
import ctypes as C

import numpy as np
import pytest

import sepgraph as sg

pytestmark = pytest.mark.gpu

MAX_V = 1 << 18
MAX_E = 1 << 23


def _fn():
    L = sg.load()
    f = L.sg_bfs_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_uint32,
                  C.POINTER(sg.Options), C.c_void_p, C.c_void_p, C.POINTER(sg.Stats), C.c_char_p, C.c_size_t]
    return f


@pytest.fixture(scope="module")
def torch():
    return pytest.importorskip("torch")


@pytest.mark.parametrize("scale,sym", [(14, True), (15, False)])
def test_noalloc_matches_allocating_bfs(torch, scale, sym):
    h = sg.HostGraph.rmat(scale, 16, symmetric=sym, seed=1)
    ctx = sg.Context(0)
    G = ctx.graph(h, symmetric=sym)
    dev = torch.device("cuda", 0)
    off = torch.from_numpy(h.offsets.astype(np.int32)).to(dev)
    idx = torch.from_numpy(h.indices.astype(np.int32)).to(dev)
    if sym:
        ioff, iidx = off, idx
    else:  # in-edge arrays (CSC) built on the host for the hybrid policy's pull rounds
        order = np.lexsort((np.repeat(np.arange(h.nv), np.diff(h.offsets)), h.indices))
        src = np.repeat(np.arange(h.nv, dtype=np.uint32), np.diff(h.offsets))[order]
        coff = np.zeros(h.nv + 1, np.int64)
        np.add.at(coff, h.indices.astype(np.int64) + 1, 1)
        ioff = torch.from_numpy(np.cumsum(coff).astype(np.int32)).to(dev)
        iidx = torch.from_numpy(src.astype(np.int32)).to(dev)
    out = torch.empty(h.nv, dtype=torch.int32, device=dev)
    f = _fn()
    err = C.create_string_buffer(256)
    sources = [h.max_degree_vertex()[0]] + [int(s) for s in h.pick_sources(1, 3)]
    for src in sources:  # two calls in a row on the shared scratch
        st = sg.Stats()
        rc = f(off.data_ptr(), idx.data_ptr(), h.nv, h.ne, ioff.data_ptr(), iidx.data_ptr(), src, None,
               out.data_ptr(), None, C.byref(st), err, 256)
        assert rc == 0, err.value
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.uint32)
        want, _, _ = G.bfs(src)
        assert (got == want).all()
        assert st.rounds > 0
    G.close()
    ctx.close()


def _call(f, off, idx, h, ioff, iidx, src, opt, out):
    st = sg.Stats()
    st.time_kernel_ms = 123.0  # must be overwritten
    st.edges_reached = 77
    err = C.create_string_buffer(256)
    rc = f(off.data_ptr(), idx.data_ptr(), h.nv, h.ne, ioff.data_ptr() if ioff is not None else None,
           iidx.data_ptr() if iidx is not None else None, src, C.byref(opt) if opt is not None else None,
           out.data_ptr(), None, C.byref(st), err, 256)
    assert rc == 0, err.value
    return st


def test_noalloc_default_options_run_sg_bfs_rounds(torch):
    """opt=NULL: same variant sequence as sg_bfs's defaults (load balancing from the
    average degree, blocks per SM from the graph size); unfilled stats fields are zeroed."""
    h = sg.HostGraph.rmat(16, 16, symmetric=True, seed=1)
    ctx = sg.Context(0)
    G = ctx.graph(h, symmetric=True)
    dev = torch.device("cuda", 0)
    off = torch.from_numpy(h.offsets.astype(np.int32)).to(dev)
    idx = torch.from_numpy(h.indices.astype(np.int32)).to(dev)
    out = torch.empty(h.nv, dtype=torch.int32, device=dev)
    f = _fn()
    src = h.max_degree_vertex()[0]
    st = _call(f, off, idx, h, off, idx, src, None, out)
    want, wst, _ = G.bfs(src)
    torch.cuda.synchronize()
    assert (out.cpu().numpy().view(np.uint32) == want).all()
    assert list(st.rounds_by_variant) == list(wst.rounds_by_variant)
    assert st.time_kernel_ms == 0 and st.time_total_ms == 0 and st.edges_reached == 0 and st.n_trace == 0
    G.close()
    ctx.close()


def test_noalloc_at_fixed_limits_push_only_and_explicit_options(torch):
    """The largest graph the array takes: RMAT scale 18 symmetric (2^18 vertices,
    just under 2^23 edges, hubs of thousands of edges split into chunks); a
    push-only call (NULL in-edge arrays) and a call with explicit options, each
    against sg_bfs; the device's free memory does not move across calls."""
    h = sg.HostGraph.rmat(18, 16, symmetric=True, seed=1)
    assert h.nv == MAX_V and h.ne <= MAX_E and np.diff(h.offsets).max() > 4096
    ctx = sg.Context(0)
    G = ctx.graph(h, symmetric=True)
    dev = torch.device("cuda", 0)
    off = torch.from_numpy(h.offsets.astype(np.int32)).to(dev)
    idx = torch.from_numpy(h.indices.astype(np.int32)).to(dev)
    out = torch.empty(h.nv, dtype=torch.int32, device=dev)
    f = _fn()
    srcs = [h.max_degree_vertex()[0]] + [int(s) for s in h.pick_sources(2, 5)]
    want = {s: G.bfs(s)[0] for s in srcs}
    _call(f, off, idx, h, off, idx, srcs[0], None, out)  # first call: address look-up
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    opt = sg.Options()
    sg.load().sg_options_default(C.byref(opt))
    opt.variant = 5  # ASYNC_PUSH_DD
    opt.lb_push = 2  # FINE
    opt.blocks_per_sm = 1
    opt.max_iteration = 10000
    for src in srcs:
        for ioff, iidx, o in ((off, idx, None), (None, None, None), (off, idx, opt)):
            st = _call(f, off, idx, h, ioff, iidx, src, o, out)
            torch.cuda.synchronize()
            assert (out.cpu().numpy().view(np.uint32) == want[src]).all(), (src, ioff is None, o is not None)
            assert st.device_error == 0 and st.rounds > 0
            if ioff is None or o is not None:  # push-only rounds
                assert st.rounds_by_variant[5] == st.rounds
    assert torch.cuda.mem_get_info(0)[0] == free0
    G.close()
    ctx.close()


def test_noalloc_rejects_oversized_graph(torch):
    f = _fn()
    dev = torch.device("cuda", 0)
    off = torch.zeros(16, dtype=torch.int32, device=dev)
    out = torch.empty(16, dtype=torch.int32, device=dev)
    err = C.create_string_buffer(256)
    rc = f(off.data_ptr(), off.data_ptr(), MAX_V + 1, 0, None, None, 0, None, out.data_ptr(), None, None, err, 256)
    assert rc == 5 and b"exceeds" in err.value  # SG_ERR_CAPACITY
    rc = f(off.data_ptr(), off.data_ptr(), 15, MAX_E + 1, None, None, 0, None, out.data_ptr(), None, None, err, 256)
    assert rc == 5
