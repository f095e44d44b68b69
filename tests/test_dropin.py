"""The reference's plugin contract through the C++ Engine mirror.

tests/dropin/dropin_functors.cu holds two application functors written the way
the reference's samples write theirs (AppBase subclasses with `override`
methods, the ACCUMULATE_* codes, utils::pair combine results) — a
breadth-first search and a connected-components functor the library does not
ship — and drives them with the reference's Engine lifecycle (Engine(AlgoType)
-> SetOptions -> LoadGraph -> InitGraph(data...) -> Start -> GatherValue,
include/framework/framework.cuh:84-399).  The CPU test proves it compiles
against the library's headers with nvcc; the GPU test runs it and checks the
levels against the oracle (bit-exact) and the component labels against the
minimum vertex id of each connected component.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
import sepgraph as sg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "dropin", "dropin_functors.cu")
PKG = os.path.join(ROOT, "sep-graph_b200")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def _build(out):
    cmd = [NVCC, "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "--expt-relaxed-constexpr",
           "-Xcudafe", "--diag_suppress=esa_on_defaulted_function_ignored", "-Xptxas", "-dlcm=cg",
           "-I", os.path.join(PKG, "csrc"), "-I", os.path.join(ROOT, "include"), SRC, "-o", out,
           "-L", PKG, "-lsepgraph_b200", "-Xlinker", "-rpath", "-Xlinker", PKG]
    return subprocess.run(cmd, capture_output=True, text=True, timeout=600)


@pytest.fixture(scope="module")
def dropin_exe(tmp_path_factory):
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    sg.load()  # the library must be built
    exe = str(tmp_path_factory.mktemp("dropin") / "dropin_functors")
    r = _build(exe)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def test_reference_style_functors_compile(dropin_exe):
    assert os.path.exists(dropin_exe)


def _min_labels(off, idx):
    """Minimum vertex id of each vertex's connected component (symmetric graph)."""
    n = len(off) - 1
    parent = np.arange(n, dtype=np.int64)

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    src = np.repeat(np.arange(n), np.diff(off.astype(np.int64)))
    for u, v in zip(src.tolist(), idx.tolist()):
        ru, rv = find(u), find(v)
        if ru != rv:
            parent[max(ru, rv)] = min(ru, rv)
    return np.array([find(x) for x in range(n)], dtype=np.uint32)


@pytest.mark.gpu
@pytest.mark.parametrize("scale", [12, 15])
def test_reference_style_functors_run(dropin_exe, tmp_path, scale):
    h = sg.HostGraph.rmat(scale, 16, symmetric=True, seed=1)
    root = int(h.max_degree_vertex()[0])
    prefix = str(tmp_path / "out")
    r = subprocess.run([dropin_exe, str(scale), str(root), prefix], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    want = oracle.bfs(h.offsets, h.indices, root)
    for name in ("bfs_hybrid", "bfs_push"):
        got = np.fromfile(f"{prefix}_{name}.u32", dtype=np.uint32)
        assert np.array_equal(got, want), name
    cc = np.fromfile(f"{prefix}_cc.u32", dtype=np.uint32)
    assert np.array_equal(cc, _min_labels(h.offsets, h.indices))
    assert "rounds" in r.stdout  # PrintInfo
