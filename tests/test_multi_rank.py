"""The replica benchmark's multi-rank bookkeeping on CPU (gloo, world size 2):
the maximum (device time) and sum (work) over ranks, the barrier, each rank's
own sources (rank 0's equal the single-process run's), and the reference arm
doing no work off rank 0."""
import datetime
import os
import socket
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "sep-graph_b200")]
    import torch
    import torch.distributed as tdist

    import bench
    import sepgraph as sg

    try:
        tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        r = bench.Ranks(world, torch.device("cpu"))
        r.barrier()
        out = {"max": r.max(float(rank + 1)), "sum": r.sum(float(rank + 1))}
        h = sg.HostGraph.rmat(10, 8, seed=1)
        srcs = bench.replica_sources(h, rank)
        gathered = [None] * world
        tdist.all_gather_object(gathered, srcs)
        out["all"] = gathered
        r.barrier()
        tdist.destroy_process_group()
        q.put((rank, out))
    except Exception as e:  # reported to the parent instead of hanging it
        q.put((rank, {"error": repr(e)}))


def test_two_gloo_ranks():
    import multiprocessing as mp

    sys.path[:0] = [ROOT, os.path.join(ROOT, "sep-graph_b200")]
    import bench
    import sepgraph as sg

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = {}
    try:
        for _ in procs:
            rank, out = q.get(timeout=180)
            results[rank] = out
    finally:
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
    for rank, out in results.items():
        assert "error" not in out, out
        assert out["max"] == 2.0 and out["sum"] == 3.0
    h = sg.HostGraph.rmat(10, 8, seed=1)
    all_srcs = results[0]["all"]
    assert all_srcs == results[1]["all"]
    assert all_srcs[0] == bench.replica_sources(h, 0) == [int(s) for s in h.pick_sources(bench.N_SOURCES, 3)]
    assert all_srcs[0] != all_srcs[1] and len(all_srcs[1]) == bench.N_SOURCES


def test_single_process_ranks_are_identity():
    sys.path[:0] = [ROOT]
    import bench

    r = bench.Ranks(1)
    r.barrier()
    assert r.max(3.5) == 3.5 and r.sum(3.5) == 3.5


def test_reference_arm_runs_on_rank0_only(monkeypatch):
    sys.path[:0] = [ROOT]
    import bench

    monkeypatch.setenv("RANK", "1")
    t0 = __import__("time").perf_counter()
    assert bench.run_reference(types.SimpleNamespace(scale=22, steps=1, warmup=1)) is None
    assert __import__("time").perf_counter() - t0 < 1.0  # returned without building the graph


def test_reference_arm_line_on_rank0(monkeypatch, capsys):
    """The reference arm on rank 0 times the reference's CPU SSSP on a small
    graph and prints one JSON line with the fields the driver reads."""
    import json

    sys.path[:0] = [ROOT, os.path.join(ROOT, "sep-graph_b200")]
    import bench

    monkeypatch.setenv("RANK", "0")
    bench.run_reference(types.SimpleNamespace(scale=12, steps=1, warmup=0, gpus=1))
    lines = [l for l in capsys.readouterr().out.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["metric"] == rec["unit"] == bench.METRIC and rec["value"] > 0
    assert rec["steps"] == 1 and rec["n_gpus"] == 1 and rec["higher_is_better"] is True
    assert rec["cpu_baseline"]["kind"] in ("reference", "port") and rec["cpu_baseline"]["cores"] >= 1
    assert rec["cpu_baseline"]["value"] == rec["value"]
    assert rec["e2e"] == {"value": rec["value"], "unit": rec["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert rec["config"]["workload"] == bench.WORKLOAD and rec["config"]["nv"] == 4096
