"""Host-side logic of the library (no GPU): seeded generators, CSR build,
graph file formats, source selection, and the C ABI symbol table."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
import sepgraph as sg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rows_sorted_unique(off, idx):
    for v in range(len(off) - 1):
        r = idx[off[v]:off[v + 1]]
        if len(r) > 1 and not (np.diff(r.astype(np.int64)) > 0).all():
            return False
    return True


def test_rmat_properties_symmetric():
    h = sg.HostGraph.rmat(12, 16, symmetric=True, seed=1)
    off, idx = h.offsets, h.indices
    assert h.nv == 4096 and off[0] == 0 and off[-1] == h.ne == len(idx)
    src = np.repeat(np.arange(h.nv, dtype=np.uint32), np.diff(off))
    assert not (src == idx).any(), "self-loops removed"
    assert _rows_sorted_unique(off, idx), "rows sorted, duplicates removed"
    fwd = set(zip(src.tolist(), idx.tolist()))
    assert all((d, s) in fwd for s, d in list(fwd)[:5000]), "symmetric"
    assert h.ne <= 2 * 16 * 4096


def test_rmat_deterministic_and_seeded():
    a = sg.HostGraph.rmat(11, 8, seed=3)
    b = sg.HostGraph.rmat(11, 8, seed=3)
    c = sg.HostGraph.rmat(11, 8, seed=4)
    assert (a.offsets == b.offsets).all() and (a.indices == b.indices).all()
    assert a.ne != c.ne or not (a.indices == c.indices).all()


def test_rmat_skew_matches_quadrant_probabilities():
    # a+b = 0.76 of edges leave the lower half of the id space at every level
    h = sg.HostGraph.rmat(14, 16, symmetric=False, seed=1, keep_duplicates=True, keep_self_loops=True)
    src = np.repeat(np.arange(h.nv), np.diff(h.offsets))
    frac_low = (src < h.nv // 2).mean()
    assert abs(frac_low - 0.76) < 0.01
    dst = h.indices
    assert abs((dst < h.nv // 2).mean() - 0.76) < 0.01
    assert h.ne == 16 * h.nv


def test_grid_structure():
    h = sg.HostGraph.grid(5, 7)
    assert h.nv == 35 and h.ne == 2 * (5 * 6 + 4 * 7)
    off, idx = h.offsets, h.indices
    assert _rows_sorted_unique(off, idx)
    # corner (0,0) has right and down neighbours
    assert list(idx[off[0]:off[1]]) == [1, 7]
    # interior vertex (2,3) -> 17 has 4 neighbours
    assert list(idx[off[17]:off[18]]) == [10, 16, 18, 24]


def test_weights_range_and_seed():
    h = sg.HostGraph.rmat(10, 16, seed=1).gen_weights(1, 64, 2)
    w = h.weights
    assert w.min() >= 1 and w.max() < 64 and len(w) == h.ne
    h2 = sg.HostGraph.rmat(10, 16, seed=1).gen_weights(1, 64, 2)
    assert (h2.weights == w).all()
    assert abs(w.mean() - 32) < 1.0


def test_max_degree_vertex_lowest_id_on_ties():
    off = np.array([0, 2, 4, 5], np.uint32)
    idx = np.array([1, 2, 0, 2, 0], np.uint32)
    h = sg.HostGraph.from_csr(off, idx)
    assert h.max_degree_vertex() == (0, 2)


def test_pick_sources_have_out_edges():
    h = sg.HostGraph.rmat(12, 16, seed=1)
    s = h.pick_sources(8, 3)
    deg = np.diff(h.offsets)
    assert len(set(s.tolist())) == 8 and (deg[s] > 0).all()
    assert (h.pick_sources(8, 3) == s).all()


def test_gr_roundtrip(tmp_path):
    h = sg.HostGraph.rmat(9, 16, seed=2).gen_weights(1, 100, 5)
    p = str(tmp_path / "g.gr")
    h.write_gr(p)
    g = sg.HostGraph.read_gr(p)
    assert (g.offsets == h.offsets).all() and (g.indices == h.indices).all() and (g.weights == h.weights).all()
    # unweighted, odd edge count
    u = sg.HostGraph.from_csr(np.array([0, 1, 3, 3], np.uint32), np.array([1, 0, 2], np.uint32))
    u.write_gr(p)
    g = sg.HostGraph.read_gr(p)
    assert g.weights is None and list(g.indices) == [1, 0, 2]


def test_gr_layout_matches_galois_v1(tmp_path):
    """Header {1, 4, nv, ne}, u64 row ends, u32 dsts, pad on odd ne, u32 weights (parser.cpp:409-506)."""
    u = sg.HostGraph.from_csr(np.array([0, 2, 3], np.uint32), np.array([1, 0, 0], np.uint32),
                              np.array([5, 6, 7], np.uint32))
    p = str(tmp_path / "g.gr")
    u.write_gr(p)
    raw = open(p, "rb").read()
    hdr = np.frombuffer(raw[:32], np.uint64)
    assert list(hdr) == [1, 4, 2, 3]
    assert list(np.frombuffer(raw[32:48], np.uint64)) == [2, 3]
    assert list(np.frombuffer(raw[48:60], np.uint32)) == [1, 0, 0]
    assert list(np.frombuffer(raw[64:76], np.uint32)) == [5, 6, 7]
    assert len(raw) == 76


def test_gr_rejects_malformed(tmp_path):
    p = tmp_path / "bad.gr"
    p.write_bytes(np.array([2, 0, 3, 1], np.uint64).tobytes())
    with pytest.raises(sg.SGError) as e:
        sg.HostGraph.read_gr(str(p))
    assert e.value.status == 10
    with pytest.raises(sg.SGError) as e:
        sg.HostGraph.read_gr(str(tmp_path / "missing.gr"))
    assert e.value.status == 9


def test_market_reader_dedups_sorted(tmp_path):
    p = tmp_path / "m.mtx"
    p.write_text("%%MatrixMarket matrix coordinate integer general\n% c\n4 4 6\n1 2 3\n1 2 3\n2 1 4\n4 3 1\n1 3 2\n3 3 9\n")
    g = sg.HostGraph.read_market(str(p))
    assert list(g.offsets) == [0, 2, 3, 4, 5]
    assert list(g.indices) == [1, 2, 0, 2, 2]
    assert list(g.weights) == [3, 2, 4, 9, 1]


def test_from_csr_validates():
    with pytest.raises(sg.SGError):
        sg.HostGraph.from_csr(np.array([0, 2, 1], np.uint32), np.array([0, 1], np.uint32))
    with pytest.raises(sg.SGError):
        sg.HostGraph.from_csr(np.array([0, 1], np.uint32), np.array([5], np.uint32))


def test_abi_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "sepgraph.h")).read()
    declared = set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(sg_\w+)\s*\(", hdr, re.M))
    assert len(declared) > 20
    out = subprocess.run(["nm", "-D", "--defined-only", sg.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (sg_\w+)", out))
    missing = declared - exported
    assert not missing, missing
    lib = sg.load()
    for name in declared:
        assert hasattr(lib, name)


def test_no_device_reports_status_not_crash():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(sg.SGError) as e:
        sg.Context(0)
    assert e.value.status == 8


BIN = os.path.join(ROOT, "sep-graph_b200", "bin")
# gflags names of the reference samples: app_skeleton.h:42-87 plus each sample's DEFINEs
COMMON_FLAGS = {"interactive", "cmdfile", "max_iteration", "priority", "prio_delta", "edge_factor", "alpha", "beta",
                "output", "check", "verbose", "trace", "lb_push", "lb_pull", "graphfile", "format", "undirected",
                "json", "stats", "gen_graph", "gen_nnodes", "gen_factor", "gen_method", "gen_weights",
                "gen_weight_range", "block_size", "grid_size", "wl_alloc_factor", "wl_sort", "wl_unique"}
SAMPLE_FLAGS = {
    "hybrid_bfs": {"source_node", "sparse", "variant", "non_atomic"},
    "hybrid_sssp": {"source_node", "sparse", "variant"},
    "hybrid_pr": {"cut_threshold", "sparse", "variant", "error", "top_ranks", "print_ranks", "norm"},
    "hybrid_bc": {"source_node", "sparse", "src"},
}


GTOOLS_FLAGS = {"graphfile", "ggr", "output", "out_degree", "splitter", "deself_cycle", "deduplicate", "format",
                "d2ud"}  # samples/tools/gtools.cpp:15-23


def test_gtools_flag_surface():
    exe = os.path.join(BIN, "gtools")
    if not os.path.exists(exe):
        pytest.skip("samples not built")
    out = subprocess.run([exe, "--help"], capture_output=True, text=True, timeout=30)
    assert out.returncode == 0
    names = set(re.findall(r"^\s+--(\w+)", out.stdout, re.M))
    assert not GTOOLS_FLAGS - names, GTOOLS_FLAGS - names
    out = subprocess.run([exe], capture_output=True, text=True, timeout=30)
    assert out.returncode == 0 and "A Graph File must be provided" in out.stdout
    bad = subprocess.run([exe, "--no_such_flag=1"], capture_output=True, text=True, timeout=30)
    assert bad.returncode != 0


@pytest.mark.parametrize("sample", sorted(SAMPLE_FLAGS))
def test_cli_flag_surface(sample):
    exe = os.path.join(BIN, sample)
    if not os.path.exists(exe):
        pytest.skip("samples not built")
    out = subprocess.run([exe, "--help"], capture_output=True, text=True, timeout=30)
    assert out.returncode == 0
    names = set(re.findall(r"^\s+--(\w+)", out.stdout, re.M))
    missing = (COMMON_FLAGS | SAMPLE_FLAGS[sample]) - names
    assert not missing, missing
    bad = subprocess.run([exe, "--no_such_flag=1"], capture_output=True, text=True, timeout=30)
    assert bad.returncode != 0 and "unknown command line flag" in bad.stderr
    bad = subprocess.run([exe, "--max_iteration=abc"], capture_output=True, text=True, timeout=30)
    assert bad.returncode != 0 and "illegal value" in bad.stderr


def test_random_generator_shape():
    h = sg.HostGraph.random(2000, 10, seed=4)
    deg = np.diff(h.offsets)
    assert deg.min() >= 1 and deg.max() <= 10
    src = np.repeat(np.arange(h.nv), deg)
    assert not (src == h.indices).any() and _rows_sorted_unique(h.offsets, h.indices)
    assert (sg.HostGraph.random(2000, 10, seed=4).indices == h.indices).all()


def test_options_defaults_match_reference_flags():
    o = sg.make_options()
    assert o.alpha == 15 and o.beta == 18 and o.max_iteration == 200  # app_skeleton.h:44-51
    assert o.non_atomic == 1  # hybrid_bfs main.cpp:37
    assert abs(o.pr_error - 0.01) < 1e-12  # hybrid_pr main.cpp:37
    assert o.variant == -1 and o.lb_push == -1 and o.blocking == 1


def _write(p, text):
    p.write_text(text)
    return str(p)


def test_metis_reader(tmp_path):
    """ReadGraph (src/utils/parser.cpp:230-396): comments, 1-based lists in file
    order, m counted once per undirected edge, fmt digits for vertex sizes /
    vertex weights (ncon) / edge weights, empty lines for isolated vertices."""
    h = sg.HostGraph.read_metis(_write(tmp_path / "a.graph", "% c\n4 3\n3 2\n1\n1 4\n% mid\n3\n"))
    assert h.offsets.tolist() == [0, 2, 3, 5, 6] and h.indices.tolist() == [2, 1, 0, 0, 3, 2]
    assert h.weights is None
    h = sg.HostGraph.read_metis(_write(tmp_path / "b.graph", "3 2 1\n2 7 3 9\n1 7\n1 9\n"))
    assert h.indices.tolist() == [1, 2, 0, 0] and h.weights.tolist() == [7, 9, 7, 9]
    h = sg.HostGraph.read_metis(_write(tmp_path / "c.graph", "3 1 111 2\n5 1 2 2 4\n6 3 4 1 4\n0 1 1\n"))
    assert h.offsets.tolist() == [0, 1, 2, 2] and h.indices.tolist() == [1, 0] and h.weights.tolist() == [4, 4]
    h = sg.HostGraph.read_metis(_write(tmp_path / "d.graph", "3 1\n\n3\n2\n"))
    assert h.offsets.tolist() == [0, 0, 1, 2] and h.indices.tolist() == [2, 1]
    for bad in ("3 2\n2\n1\n\n",          # fewer entries than 2m
                "2 1\n2 2\n1\n",           # more entries than 2m
                "2 1\n3\n1\n",             # neighbour out of range
                "2 1 112\n2\n1\n",         # unknown fmt
                "2 1 1 2\n2 1\n1 1\n",     # ncon without vertex weights
                "2 1 1\n2 0\n1 0\n",       # edge weight must be positive
                "0 1\n"):
        with pytest.raises(sg.SGError):
            sg.HostGraph.read_metis(_write(tmp_path / "bad.graph", bad))


@pytest.mark.skipif(not oracle.ref_gtools_available(), reason="reference converter not compiled here")
@pytest.mark.parametrize("weighted", [False, True])
def test_market_reader_matches_reference(tmp_path, weighted):
    """Our MatrixMarket reader against the reference's ReadGraphMarket, read through
    the reference converter with --deduplicate=false (it prints the CSR as read)."""
    rng = np.random.default_rng(3 + weighted)
    n, m = 60, 500
    s, d = rng.integers(1, n + 1, m), rng.integers(1, n + 1, m)
    w = rng.integers(1, 20, m)
    lines = ["%%MatrixMarket matrix coordinate integer general", f"{n} {n} {m}"]
    lines += [f"{a} {b} {c}" if weighted else f"{a} {b}" for a, b, c in zip(s, d, w)]
    path = _write(tmp_path / "g.mtx", "\n".join(lines) + "\n")
    rs, rd, rw = oracle.ref_gtools(path, str(tmp_path / "o.txt"), deduplicate=False, fmt="market")
    h = sg.HostGraph.read_market(path)
    src = np.repeat(np.arange(h.nv, dtype=np.uint32), np.diff(h.offsets.astype(np.int64)))
    assert np.array_equal(src, rs) and np.array_equal(h.indices, rd)
    if weighted:
        assert np.array_equal(h.weights, rw)


def test_ctypes_mirrors_match_c_header_layout(tmp_path):
    """Every ctypes structure of the binding has the size and field offsets
    that a C compiler gives the matching struct of include/sepgraph.h."""
    import shutil
    import ctypes as C

    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    pairs = {"sg_options": sg.Options, "sg_round_trace": sg.RoundTrace, "sg_stats": sg.Stats,
             "sg_batch_query": sg.BatchQuery, "sg_server_config": sg.ServerConfig, "sg_query": sg.Query,
             "sg_server_stats": sg.ServerStats, "sg_tune_entry": sg.TuneEntry}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "sepgraph.h"', "int main(void) {"]
    for cname, py in pairs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            lines.append(f'printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    r = subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=30).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in pairs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f in py._fields_:
            assert got[(cname, f[0])] == getattr(py, f[0]).offset, (cname, f[0])
    assert sg.make_options().wl_sort == 0


def test_sample_run_record_format(tmp_path):
    """The samples' --json record: every key of the reference's
    Engine::SaveToJson (framework.cuh:205-257) with its value type, the trace
    lines under "round", keys sorted, strings escaped (built on the CPU from
    synthetic statistics through the samples' own PrintRun)."""
    import json
    import shutil

    cxx = shutil.which("g++")
    lib = os.path.join(ROOT, "sep-graph_b200", "libsepgraph_b200.so")
    if not cxx or not os.path.exists(lib):
        pytest.skip("no C++ compiler or library not built")
    out = tmp_path / "rec.json"
    src = tmp_path / "rec.cpp"
    src.write_text(r'''
#include "sg_skeleton.h"
int main(int argc, char **argv) {
    sgflags::ParseCommandLineFlags(&argc, &argv, true);
    sg_round_trace tr[2] = {{1, SG_ASYNC_PUSH_DD, 1, 5, 3, 40, 100, 0.5f, 0}, {2, SG_ASYNC_PULL_DD, 5, 0, 0, 0, 60, 0.25f, 0}};
    sg_stats st{};
    st.rounds = 2; st.time_total_ms = 1.5; st.time_kernel_ms = 1.25; st.trace = tr; st.n_trace = 2; st.trace_capacity = 2;
    sg_options o; sg_options_default(&o);
    o.variant = SG_ASYNC_PUSH_DD; o.lb_push = SG_LB_FINE_GRAINED; o.priority = SG_PRIORITY_LOW_HIGH; o.priority_delta = 8;
    LoadedGraph g; g.nv = 10; g.ne = 30;
    JsonRecord js;
    PrintRun(st, o, g, false, js);
    js.put("non_atomic", "YES");
    std::printf("wl_sort=%d\n", CommonOptions().wl_sort);
    return 0;
}
''')
    exe = tmp_path / "rec"
    inc = os.path.join(ROOT, "sep-graph_b200", "csrc", "samples")
    r = subprocess.run([cxx, "-std=c++17", "-O0", "-I", inc, str(src), "-o", str(exe), "-L",
                        os.path.dirname(lib), "-lsepgraph_b200", "-Wl,-rpath," + os.path.dirname(lib)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe), "--trace", "--wl_sort", f"--json={out}", '--graphfile=a "quoted"\\path.gr'],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    text = out.read_text()
    rec = json.loads(text)
    save_to_json = {"time_input_active_node", "time_output_active_node", "time_input_workload",
                    "time_output_workload", "time_queue2bitmap", "time_bitmap2queue", "time_rebuild_worklist",
                    "time_priority_sample", "time_sort_worklist", "time_unique_worklist", "time_kernel", "time_total",
                    "time_per_round", "num_iteration", "force_variant", "force_push_load_balancing",
                    "priority_type", "priority_delta", "fused_kernel", "max_iteration_reached", "dataset", "nnodes",
                    "nedges", "algo_type", "round"}
    assert save_to_json <= set(rec), save_to_json - set(rec)
    assert "force_pull_load_balancing" not in rec and "device" not in rec  # not forced; no context
    assert rec["num_iteration"] == 2 and rec["nnodes"] == 10 and rec["nedges"] == 30
    assert rec["time_total"] == 1.5 and rec["time_per_round"] == 0.75 and rec["time_kernel"] == 1.25
    assert rec["force_variant"] == "ASYNC_PUSH_DD" and rec["force_push_load_balancing"] == "FINE_GRAINED"
    assert rec["priority_type"] == "low_high" and rec["priority_delta"] == 8
    assert rec["algo_type"] == "TRAVERSAL_SCHEME" and rec["fused_kernel"] == "NO" and rec["non_atomic"] == "YES"
    assert rec["dataset"] == 'a "quoted"\\path.gr'
    assert rec["round"] == [l for l in r.stdout.splitlines() if l.startswith("Round: ")]
    assert len(rec["round"]) == 2 and "ASYNC_PULL_DD" in rec["round"][1]
    assert list(rec) == sorted(rec) and text.startswith("{\n    \"")
    assert "wl_sort=1" in r.stdout  # --wl_sort reaches sg_options
