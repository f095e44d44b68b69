#!/usr/bin/env python
"""Benchmark of the B200 hybrid graph engine through its C ABI.

Headline (one JSON line): single-source SSSP on RMAT scale 22 (edge factor 16,
a/b/c/d = .57/.19/.19/.05, seed 1, directed, uint32 weights uniform in [1,64)
seed 2), eight seeded sources (seed 3) per step.  GTEPS = edges of the reached
component / solve time, summed over the step's sources and over ranks
(replicas, one process per GPU, weak scaling).

At N=1 the line also carries, under "extra" (skip with --quick):
  per_algo  BFS RMAT-16 symmetric (the reference's host-checker case, its
            BFSHost timed beside), SSSP on the 4096x4096 grid (weights
            [1,1000), delta autotuned), PageRank on RMAT-23 directed
            (data-driven push and topology-driven pull, residual 1e-7), BC on
            RMAT-23 symmetrised — GTEPS and fraction of the HBM roofline each;
  batched   64-source BFS and 32-source BC on RMAT-22 symmetric, 256 SSSP
            instances over RMAT scale 12-20 graphs: one launch vs one plain
            launch per query, results compared;
  served    a Poisson stream of mixed BFS/SSSP/PageRank/BC queries
            (60/25/10/5 %) over 16 device-resident graphs (RMAT 14-22, grids
            1024^2-4096^2) through the query server: queries/s and
            p50/p99/p999 latency, against the plain one-query-per-launch path
            timed on a uniform sample of the same stream, results compared.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--quick]

--impl reference times the reference's own single-threaded SSSPHostNaive
(compiled from its sources into oracle/_ref; the oracle's C port otherwise)
on the host cores, one source per thread, on the same graph and sources.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import datetime
import json
import os
import random
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "sep-graph_b200"))

import numpy as np  # noqa: E402

METRIC = "GTEPS"
WORKLOAD = "sssp_rmat22_directed_w1-64"
SCALE, EDGE_FACTOR, N_SOURCES = 22, 16, 8
FALLBACK_HBM_GBS = 6650.0
INF = 0xFFFFFFFF


def args_parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--quick", action="store_true", help="headline line only")
    p.add_argument("--served-queries", type=int, default=2000)
    p.add_argument("--served-slots", type=int, default=2)
    p.add_argument("--served-bps", type=int, default=0, help="server blocks per SM per slot (0 = library choice)")
    p.add_argument("--extras", default="per_algo,batched,ingest,served", help="extra sections at N=1 (comma list)")
    p.add_argument("--scale", type=int, default=SCALE)
    p.add_argument("--profile", choices=["sssp_push", "sssp_delta", "bfs", "pr_pull", "pr_push", "bc", "msbfs", "msbc",
                                         "msbfs_grid", "sssp_batch", "transpose"],
                   help="run one warm-up and one measured solve of that kernel only (for ncu captures)")
    p.add_argument("--opts", default="", help="--profile: JSON object of sg_options fields overriding the mode's")
    return p.parse_args()


def run_profile(a):
    """Two solves of one engine instantiation (the second is the one to capture)."""
    import sepgraph as sg

    ctx = sg.Context(int(os.environ.get("LOCAL_RANK", "0")))
    if a.profile in ("msbfs", "msbc", "msbfs_grid", "sssp_batch", "transpose"):
        run_profile_batch(a, ctx)
        ctx.close()
        return
    sym = a.profile in ("bfs", "bc")
    h = sg.HostGraph.rmat(a.scale, EDGE_FACTOR, 0.57, 0.19, 0.19, seed=1, symmetric=sym)
    if a.profile.startswith("sssp"):
        h.gen_weights(1, 64, 2)
    G = ctx.graph(h, symmetric=sym)
    src = h.max_degree_vertex()[0] if sym else int(h.pick_sources(1, 3)[0])
    extra = json.loads(a.opts) if a.opts else {}
    for _ in range(2):
        if a.profile == "sssp_push":
            _, st, _ = G.sssp(src, **dict(dict(variant="async_push_dd", max_iteration=100000), **extra))
        elif a.profile == "sssp_delta":
            # delta-stepping as the autotuner's candidates run it (override with --opts)
            _, st, _ = G.sssp(src, **dict(dict(variant="async_push_dd", priority="low_high", priority_delta=8,
                                               blocks_per_sm=2, chunk_edges=256, max_iteration=1000000), **extra))
        elif a.profile == "bfs":
            _, st, _ = G.bfs(src, **extra)
        elif a.profile == "pr_pull":
            _, st, _ = G.pagerank(**dict(dict(variant="sync_pull_td", pr_error=1e-7, max_iteration=1000), **extra))
        elif a.profile == "pr_push":
            _, st, _ = G.pagerank(**dict(dict(variant="async_push_dd", pr_error=1e-7, max_iteration=1000), **extra))
        else:
            _, _, st = G.bc(src, **extra)
        print(json.dumps({"profile": a.profile, "scale": a.scale, "ms": st.time_kernel_ms, "rounds": st.rounds,
                          "edges_reached": st.edges_reached, "edges_processed": st.edges_processed}), flush=True)
    G.close()
    ctx.close()


def run_profile_batch(a, ctx):
    """Two runs of one batched / multi-source / graph-construction call (the second is the one to capture):
    msbfs 64 sources and msbc 32 sources on the symmetric RMAT graph of --scale; msbfs_grid 64 sources
    on the 2^(scale/2) x 2^(scale/2) 4-neighbour grid (interleaved masks); sssp_batch 64 SSSP
    queries over RMAT graphs of scales 12 .. --scale; transpose = sg_graph_create of the directed
    weighted RMAT CSR of --scale from device arrays (validation and the CSC transpose)."""
    import sepgraph as sg
    import torch

    for _ in range(2):
        t0 = time.perf_counter()
        if a.profile in ("msbfs", "msbc"):
            if _ == 0:
                h = sg.HostGraph.rmat(a.scale, EDGE_FACTOR, seed=1, symmetric=True)
                G = ctx.graph(h, symmetric=True)
            n = 64 if a.profile == "msbfs" else 32
            srcs = [int(x) for x in h.pick_sources(n, 11)]
            out = G.msbfs(srcs) if a.profile == "msbfs" else G.msbc(srcs)
            ms = out[1].time_kernel_ms
        elif a.profile == "msbfs_grid":
            if _ == 0:
                side = 1 << (a.scale // 2)
                h = sg.HostGraph.grid(side, side)
                G = ctx.graph(h)
                srcs = [int(x) for x in np.random.default_rng(5).integers(0, h.nv, 64)]
            ms = G.msbfs(srcs, max_iteration=1000000)[1].time_kernel_ms
        elif a.profile == "sssp_batch":
            if _ == 0:
                graphs = []
                for sc in range(12, a.scale + 1):
                    hh = sg.HostGraph.rmat(sc, 16, seed=100 + sc).gen_weights(1, 64, 200 + sc)
                    graphs.append((hh, ctx.graph(hh, no_csc=True)))
                rng = random.Random(5)
                queries = [(graphs[k % len(graphs)][1], rng.randrange(graphs[k % len(graphs)][0].nv))
                           for k in range(64)]
            _, st, _ = ctx.sssp_batch(queries, variant="async_push_dd", max_iteration=1000000)
            ms = st.time_kernel_ms
        else:
            if _ == 0:
                h = sg.HostGraph.rmat(a.scale, EDGE_FACTOR, seed=1).gen_weights(1, 64, 2)
                dev = [torch.from_numpy(x.view(np.int32)).cuda() for x in (h.offsets, h.indices, h.weights)]
            torch.cuda.synchronize()
            gg = ctx.graph_from_csr(*dev, nv=h.nv, ne=h.ne)
            torch.cuda.synchronize()
            gg.close()
            ms = 1e3 * (time.perf_counter() - t0)
        print(json.dumps({"profile": a.profile, "scale": a.scale, "ms": ms}), flush=True)


def peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region: the sampler is started first and the
    timed region begins only after its first sample arrived (nvidia-smi can take a second
    to start on a fresh box), so short timed regions still get samples."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.p = None
        self.lines = []
        self.t = None

    def _read(self):
        for line in self.p.stdout:
            self.lines.append(line)

    def __enter__(self):
        import threading

        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 10 and self.p.poll() is None:
                time.sleep(0.01)
            self.lines.clear()  # keep samples from the timed region on
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            time.sleep(0.12)
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            if self.t:
                self.t.join(timeout=5)
        self.out = "".join(self.lines)

    def summary(self):
        rows = [r.split(", ") for r in (self.out or "").strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def make_graph(scale, rank=0):
    """The headline graph and the sources one rank runs: every rank holds the
    whole graph (replicas) and answers its own independent sources; rank 0's
    are the single-GPU run's."""
    import sepgraph as sg

    h = sg.HostGraph.rmat(scale, EDGE_FACTOR, 0.57, 0.19, 0.19, seed=1).gen_weights(1, 64, 2)
    return h, replica_sources(h, rank)


def make_graph_reference(scale):
    """The same graph and rank-0 sources from the oracle's generator (a CPU test
    proves its CSR, weights and sources equal to the library's, word for word),
    so the reference arm never loads the library."""
    import oracle

    h = oracle.rmat(scale, EDGE_FACTOR, 0.57, 0.19, 0.19, seed=1).gen_weights(1, 64, 2)
    return h, replica_sources(h, 0)


def config_of(nv, ne, n_sources, world):
    """The workload description both arms print (identical keys and values)."""
    return {"workload": WORKLOAD, "nv": nv, "ne": ne, "sources_per_step": n_sources,
            "l2": "inputs larger than L2 (graph arrays %.0f MB vs 126 MB L2)" % ((4 * (nv + 1) + 8 * ne) / 1e6),
            "parallelism": f"replicas{world}"}


def replica_sources(h, rank):
    return [int(s) for s in h.pick_sources(N_SOURCES, 3 if rank == 0 else 3 + 1000 * rank)]


class Ranks:
    """Replica bookkeeping over torch.distributed: a barrier, and the maximum
    (device time) and sum (work) over ranks; single-process when world == 1."""

    def __init__(self, world, device=None):
        self.world = world
        self.device = device  # tensors for the all-reduce live here (cuda for NCCL, cpu for gloo)

    def barrier(self):
        import torch

        if self.world > 1:
            torch.distributed.barrier()
        if self.device is not None and self.device.type == "cuda":
            torch.cuda.synchronize()

    def _reduce(self, x, op):
        import torch

        if self.world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        torch.distributed.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        import torch

        return self._reduce(x, torch.distributed.ReduceOp.MAX if self.world > 1 else None)

    def sum(self, x):
        import torch

        return self._reduce(x, torch.distributed.ReduceOp.SUM if self.world > 1 else None)


def sssp_bytes(nv, e_reached):
    # algorithmic bytes of one SSSP: offsets + (index + weight) per reached edge + distances
    return 4 * (nv + 1) + 8 * e_reached + 4 * nv


def bfs_bytes(nv, e_reached):
    # offsets + index per reached edge + levels
    return 4 * (nv + 1) + 4 * e_reached + 4 * nv


def reached_edges(h, values):
    deg = np.diff(h.offsets.astype(np.int64))
    return int(deg[np.asarray(values) != INF].sum())


# ---------------------------------------------------------------- reference arm / CPU baseline
def cpu_sssp_one(h, src):
    import oracle

    if oracle.ref_available():
        return oracle.ref_sssp(h.offsets, h.indices, h.weights, src), "reference"
    return oracle.sssp(h.offsets, h.indices, h.weights, src), "port"


def cpu_baseline(h, srcs, budget_s=20.0):
    """Single thread, as many sources as fit the budget (>= 1); also returns each
    computed distance array under "results" (the caller checks the GPU's against them)."""
    t_tot, e_tot, n = 0.0, 0, 0
    kind = "port"
    results = {}
    for s in srcs:
        t0 = time.perf_counter()
        d, kind = cpu_sssp_one(h, s)
        t_tot += time.perf_counter() - t0
        e_tot += reached_edges(h, d)
        results[s] = d
        n += 1
        if t_tot > budget_s:
            break
    return {"value": e_tot / t_tot / 1e9, "unit": METRIC, "cores": 1, "kind": kind,
            "sample": f"SSSPHostNaive from {n} of the {len(srcs)} sources on the full RMAT-{SCALE} graph, 1 thread",
            "seconds": t_tot, "results": results}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    h, srcs = make_graph_reference(a.scale)
    ncores = os.cpu_count() or 1
    nthreads = min(ncores, len(srcs))

    def step():
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(nthreads) as ex:  # ctypes releases the GIL during the C call
            outs = list(ex.map(lambda s: cpu_sssp_one(h, s), srcs))
        dt = time.perf_counter() - t0
        e = sum(reached_edges(h, d) for d, _ in outs)
        return e, dt, outs[0][1]

    for _ in range(a.warmup):
        step()
    tot_e, tot_t, kind = 0, 0.0, "port"
    for _ in range(a.steps):
        e, dt, kind = step()
        tot_e += e
        tot_t += dt
    v = tot_e / tot_t / 1e9
    line = {"metric": METRIC, "value": v, "unit": METRIC, "impl": "reference", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * tot_t / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": config_of(h.nv, h.ne, len(srcs), a.gpus),
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": nthreads, "kind": kind,
                             "sample": f"all {len(srcs)} sources of the step on {nthreads} threads (one source "
                                       "per thread at a time), full graph"},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm
def run_ours(a):
    import torch

    import sepgraph as sg

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = world > 1
    torch.cuda.set_device(local)
    if dist:
        import torch.distributed as tdist

        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    ranks = Ranks(world, torch.device("cuda", local))
    barrier, max_over_ranks, sum_over_ranks = ranks.barrier, ranks.max, ranks.sum

    ctx = sg.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    h, srcs = make_graph(a.scale, rank)
    nv, ne = h.nv, h.ne
    G = ctx.graph(h)
    dout = torch.empty(nv, dtype=torch.int32, device="cuda")

    # ---- options from the library's autotuner (sg_autotune: mode/delta, blocks
    # per SM, load balancing, lookahead depth, heavy threshold, chunk size;
    # every candidate must reproduce the first one's distances), untimed, on
    # four sources drawn apart from the measured ones
    tune_srcs = [int(s) for s in h.pick_sources(4, 97)]
    tuned, tuned_ms, report = G.autotune("sssp", tune_srcs, max_iteration=1000000)
    kw = dict(tuned, max_iteration=1000000)
    best = "{variant}{d}".format(variant=tuned["variant"], d=f"_delta{tuned['priority_delta']:g}"
                                 if "priority" in tuned else "")
    mode_ms = [dict(r) for r in report]
    e_reached, gpu_dist = {}, {}
    for s in srcs:
        d, st, _ = G.sssp(s, **kw)
        e_reached[s] = st.edges_reached
        gpu_dist[s] = d
    step_edges = sum(e_reached[s] for s in srcs)
    step_bytes = sum(sssp_bytes(nv, e_reached[s]) for s in srcs)
    kw_async = dict(kw, blocking=0)

    def step(evs=None):
        with torch.cuda.stream(stream):
            for k, s in enumerate(srcs):
                if evs is not None:
                    evs[k][0].record(stream)
                G.sssp(s, out=dout, **kw_async)
                if evs is not None:
                    evs[k][1].record(stream)

    for _ in range(a.warmup):
        step()
    ctx.synchronize()
    launch_evs = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in srcs] for _ in range(a.steps)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with Clocks(local) as clk:
        start.record(stream)
        for k in range(a.steps):
            step(launch_evs[k])
        end.record(stream)
        end.synchronize()
    barrier()
    ctx.synchronize()
    ms = start.elapsed_time(end)
    ms_max = max_over_ranks(ms)
    launch_ms = [b.elapsed_time(e) for row in launch_evs for (b, e) in row]
    value = sum_over_ranks(step_edges * a.steps) / (ms_max * 1e-3) / 1e9

    # ---- end to end through the C ABI: pinned host CSR + weights uploaded every
    # step, eight queries with host distance buffers, graph released
    off_p = torch.from_numpy(h.offsets.copy()).pin_memory()
    idx_p = torch.from_numpy(h.indices.copy()).pin_memory()
    w_p = torch.from_numpy(h.weights.copy()).pin_memory()
    host_out = torch.empty(nv, dtype=torch.int32).pin_memory()
    e2e_steps = max(1, min(a.steps, 3))
    e2e_kw = dict(kw, blocking=1)
    barrier()
    t0 = time.perf_counter()
    parts = {"upload_and_check": 0.0, "queries": 0.0, "release": 0.0}
    for _ in range(e2e_steps):
        ta = time.perf_counter()
        G2 = ctx.graph_from_csr(off_p.data_ptr(), idx_p.data_ptr(), w_p.data_ptr(), nv=nv, ne=ne,
                                no_csc=tuned["variant"] == "async_push_dd")
        tb = time.perf_counter()
        for s in srcs:
            G2.sssp(s, out=host_out.numpy(), **e2e_kw)
        tc = time.perf_counter()
        G2.close()
        parts["upload_and_check"] += tb - ta
        parts["queries"] += tc - tb
        parts["release"] += time.perf_counter() - tc
    ctx.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = sum_over_ranks(step_edges * e2e_steps) / e2e_s / 1e9
    h2d = 4 * (nv + 1) + 8 * ne
    d2h = 4 * nv * len(srcs)

    # ---- parity at the headline configuration: every source's distances
    # against the oracle's Dijkstra (exact: distances are unique), and against
    # the reference's own SSSPHostNaive for the sources the CPU baseline runs
    parity_fail = 0
    for s in srcs:
        parity_fail += int(not np.array_equal(gpu_dist[s], oracle_dijkstra(h, s)))
    cpu, ref_checked = None, 0
    if rank == 0 and world == 1:
        cpu = cpu_baseline(h, srcs)
        for s, d in cpu.pop("results").items():
            parity_fail += int(not np.array_equal(gpu_dist[s], d))
            ref_checked += 1
    parity_fail = int(sum_over_ranks(parity_fail))
    peak, peak_kind = peak_hbm()
    avg_launch_ms = float(np.mean(launch_ms))
    achieved = (step_bytes / len(srcs)) / (avg_launch_ms * 1e-3) / 1e9
    traffic = read_traffic("delta" if "priority" in tuned else "push")
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic",
        "config": config_of(nv, ne, len(srcs), world),
        "tuning": {"mode": best, "options": tuned, "autotune_ms_per_source": tuned_ms, "autotune_report": mode_ms,
                   "edges_reached_per_step": step_edges},
        "parity": {"sssp_rmat22_headline": parity_fail == 0,
                   "checked": f"{len(srcs) * world} sources' distances vs the oracle's Dijkstra (all ranks); "
                              f"{ref_checked} of them also vs the reference's SSSPHostNaive (rank 0), bit-exact",
                   "mismatched_sources": parity_fail},
        "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "what": "per step: pinned CSR+weights upload and device check into the graph arena the context kept from the previous step (sg_graph_destroy keeps it for reuse), 8 queries into pinned host distance arrays, graph released",
                "ms_per_step": {k: 1e3 * v / e2e_steps for k, v in parts.items()}},
        "gpu_launches": a.steps * len(srcs),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind, "kernel": "hybrid_engine_kernel<SSSP>",
                     "avg_launch_ms": avg_launch_ms,
                     "bytes": "4(V+1) + 8*E_reached + 4V per source"},
        "clocks": clk.summary(),
    }
    if cpu:
        line["cpu_baseline"] = cpu
    if world == 1 and not a.quick:
        extra = {}
        cache = {"rmat22": (h, G)}
        wanted = set(a.extras.split(","))
        for name, fn in (("per_algo", per_algo), ("batched", batched), ("ingest", ingest), ("served", served)):
            if name not in wanted:
                continue
            t0 = time.perf_counter()
            try:
                extra[name] = fn(ctx, cache, a)
            except Exception as e:  # an extra must not hide the headline line
                extra[name] = {"error": repr(e)}
            extra[name]["bench_seconds"] = round(time.perf_counter() - t0, 1)
        line["extra"] = extra
        for k, (_, g) in list(cache.items()):
            if k != "rmat22":
                g.close()
    if "extra" in line:
        for name, sec in line["extra"].items():
            for k, v in _parity_flags(sec, name):
                line["parity"][k] = v
    if rank == 0:
        print(json.dumps(line), flush=True)
    G.close()
    ctx.close()
    if dist:
        torch.distributed.destroy_process_group()
    if parity_fail:
        sys.exit(3)  # a fast wrong answer is not a result


def _parity_flags(sec, prefix):
    """(name, bool) for every parity boolean an extra section reports."""
    out = []
    if not isinstance(sec, dict):
        return out
    for k, v in sec.items():
        if isinstance(v, dict):
            out += _parity_flags(v, f"{prefix}.{k}")
        elif isinstance(v, bool) and ("parity" in k or "same" in k or "agree" in k or k.endswith("_ok")):
            out.append((f"{prefix}.{k}", v))
    return out


def oracle_dijkstra(h, s):
    import oracle

    return oracle.dijkstra(h.offsets, h.indices, h.weights, s)


def read_traffic(mode):
    """DRAM bytes per launch of the engine kernel from the committed ncu summary of the full-size
    headline launch (delta-stepping options); None for a mode it does not describe."""
    if not mode.startswith("delta"):
        return None
    name = "sssp_rmat22_delta_engine_kernel_traffic.md"
    try:
        for line in open(os.path.join(ROOT, "profiles", name)):
            if line.startswith("dram_bytes_per_launch_full_size:"):
                return float(line.split(":")[1].split()[0])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------- extras
def _median_ms(fn, reps, si=1, key="time_kernel_ms"):
    """Median device time over reps calls (the first dropped when reps > 2); fn()[si] is the sg_stats."""
    ts, out = [], None
    for _ in range(reps):
        out = fn()
        ts.append(getattr(out[si], key))
    return statistics.median(ts[1:] if reps > 2 else ts), out


def _cpu_time(fn, budget_s=20.0):
    """Seconds per call of a host function, repeated while under the budget (at least once)."""
    n, t0 = 0, time.perf_counter()
    while True:
        fn()
        n += 1
        if time.perf_counter() - t0 > budget_s / 4 or n >= 5:
            return (time.perf_counter() - t0) / n


def _roof(bytes_, ms, peak):
    gbs = bytes_ / (ms * 1e-3) / 1e9
    return {"GBs": gbs, "frac_hbm": gbs / peak, "frac_hbm_nominal_8TBs": gbs / 8000.0}


def per_algo(ctx, cache, a):
    """One entry per algorithm: GTEPS, device ms (median of 5 after a warm-up), HBM roofline fraction."""
    import oracle
    import sepgraph as sg

    peak = peak_hbm()[0]
    ref = oracle.ref_available()
    cpu_kind = "reference host code compiled from its sources, 1 thread" if ref else "oracle C port, 1 thread"
    res = {}
    # BFS RMAT-16 symmetric, source = max-degree vertex (the reference's host-checker case)
    h = sg.HostGraph.rmat(16, 16, symmetric=True, seed=1)
    G = ctx.graph(h, symmetric=True)
    src = h.max_degree_vertex()[0]
    t, (lv, st, _) = _median_ms(lambda: G.bfs(src), 6)
    ok = bool((lv == oracle.bfs(h.offsets, h.indices, src)).all())
    cpu_s = _cpu_time(lambda: oracle.ref_bfs(h.offsets, h.indices, src) if ref else oracle.bfs(h.offsets, h.indices, src))
    res["bfs_rmat16_sym"] = dict(
        GTEPS=st.edges_reached / t / 1e6, GTEPS_graph500_half_edges=st.edges_reached / 2 / t / 1e6, ms=t,
        rounds=st.rounds, parity_vs_oracle=ok, **_roof(bfs_bytes(h.nv, st.edges_reached), t, peak),
        cpu_GTEPS=st.edges_reached / cpu_s / 1e9, cpu_ms=1e3 * cpu_s, cpu=cpu_kind)
    G.close()

    # SSSP on the 4096x4096 grid, weights [1,1000), source 0: options from the autotuner
    h = sg.HostGraph.grid(4096, 4096).gen_weights(1, 1000, 2)
    G = ctx.graph(h, no_csc=True)
    src = 0
    tuned, _, report = G.autotune("sssp", [src], max_iteration=10000000)
    t, (d, st, _) = _median_ms(lambda: G.sssp(src, max_iteration=10000000, **tuned), 6)
    t0 = time.perf_counter()
    ok = bool(np.array_equal(d, oracle.dijkstra(h.offsets, h.indices, h.weights, src)))
    dij_s = time.perf_counter() - t0
    res["sssp_grid4096_w1-1000"] = dict(
        GTEPS=st.edges_reached / t / 1e6, ms=t, rounds=st.rounds, options=tuned,
        autotune_report=report, candidates_agree=not any(r["status"] == 10 for r in report),
        parity_vs_oracle=ok, parity_how="distances bit-exact vs the oracle's Dijkstra (unique shortest distances)",
        us_per_round=1e3 * t / max(1, st.rounds), **_roof(sssp_bytes(h.nv, st.edges_reached), t, peak),
        cpu="the reference's SSSPHostNaive needs about 4 minutes on one core for this graph (not timed); "
            f"the oracle's binary-heap Dijkstra took {dij_s:.1f} s on one core")
    G.close()
    del h, d

    # PageRank RMAT-23 directed, FP32, residual 1e-7: data-driven push vs topology-driven pull
    h = sg.HostGraph.rmat(23, 16, seed=1)
    G = ctx.graph(h)
    pr, ranks = {}, {}
    for v in ("async_push_dd", "sync_pull_td"):
        t, (r, st, _) = _median_ms(lambda: G.pagerank(variant=v, pr_error=1e-7, max_iteration=100000), 6)
        if v == "sync_pull_td":
            b = st.rounds * (4 * (h.nv + 1) + 4 * h.ne + 12 * h.nv)  # gathers assumed L2-served
            extra = {"bytes_pessimistic_with_gathers": b + st.rounds * 4 * h.ne}
        else:
            b = 4 * st.edges_processed + 16 * st.vertices_processed
            extra = {}
        pr[v] = dict(ms=t, rounds=st.rounds, edges_processed=st.edges_processed,
                     GTEPS=st.edges_processed / t / 1e6, **_roof(b, t, peak), **extra)
        ranks[v] = np.asarray(r, np.float64)
    p0, p1 = ranks["async_push_dd"], ranks["sync_pull_td"]
    pr["l1_push_vs_pull_normalised"] = float(np.abs(p0 / p0.sum() - p1 / p1.sum()).sum())
    # FP64 oracle: PageRankHost's fixed point by parallel Jacobi sweeps to a 1e-13 relative L1 change
    t0 = time.perf_counter()
    ref64, sweeps = oracle.pagerank_fixed_point_f64(h.offsets, h.indices, 1e-13)
    pr["oracle"] = {"sweeps": sweeps, "seconds": time.perf_counter() - t0, "threads": oracle.host_threads(),
                    "what": "FP64 fixed point of PageRankHost, Jacobi sweeps to a 1e-13 relative L1 change"}
    for v in ("async_push_dd", "sync_pull_td"):
        l1 = float(np.abs(ranks[v] / ranks[v].sum() - ref64 / ref64.sum()).sum())
        pr[v]["l1_vs_fp64_oracle"] = l1
        pr[v]["parity_vs_oracle"] = l1 <= 1e-6
    del ref64
    G.close()
    del h, ranks
    # CPU: PageRankHost at the same threshold on a bounded sample (RMAT-20, same generator)
    hs = sg.HostGraph.rmat(20, 16, seed=1)
    cpu_s = _cpu_time(lambda: oracle.ref_pagerank(hs.offsets, hs.indices, 1e-7) if ref
                      else oracle.pagerank_f32(hs.offsets, hs.indices, 1e-7), budget_s=30.0)
    Gs = ctx.graph(hs)
    _, sts, _ = Gs.pagerank(variant="async_push_dd", pr_error=1e-7, max_iteration=100000)
    pr["cpu"] = {"sample": "RMAT-20 directed (same generator), PageRankHost, 1e-7", "cpu_ms": 1e3 * cpu_s,
                 "cpu_G_edge_updates_per_s_est": sts.edges_processed / cpu_s / 1e9, "kind": cpu_kind}
    Gs.close()
    res["pagerank_rmat23"] = pr
    del hs

    # BFS and BC on RMAT-23 symmetrised, source = max-degree vertex
    h = sg.HostGraph.rmat(23, 16, symmetric=True, seed=1)
    G = ctx.graph(h, symmetric=True)
    src = h.max_degree_vertex()[0]
    t, (lv, st, _) = _median_ms(lambda: G.bfs(src), 6)
    t0 = time.perf_counter()
    ok = bool(np.array_equal(lv, oracle.bfs(h.offsets, h.indices, src)))
    cpu_s = time.perf_counter() - t0
    res["bfs_rmat23_sym"] = dict(
        GTEPS=st.edges_reached / t / 1e6, GTEPS_graph500_half_edges=st.edges_reached / 2 / t / 1e6, ms=t,
        rounds=st.rounds, rounds_by_variant=list(st.rounds_by_variant), edges_processed=st.edges_processed,
        parity_vs_oracle=ok, **_roof(bfs_bytes(h.nv, st.edges_reached), t, peak),
        cpu_GTEPS=st.edges_reached / cpu_s / 1e9, cpu_ms=1e3 * cpu_s, cpu="oracle BFSHost restatement, 1 thread")
    t, (bc, sig, st) = _median_ms(lambda: G.bc(src), 6, si=2, key="time_total_ms")
    e_r = st.edges_reached // 2  # sg_bc counts both traversals
    b = 2 * (4 * (h.nv + 1) + 4 * e_r) + 32 * h.nv
    cpu_s = _cpu_time(lambda: oracle.ref_bc(h.offsets, h.indices, src) if ref else oracle.bc_f32(h.offsets, h.indices, src),
                      budget_s=40.0)
    bc64, sig64, _ = oracle.bc_f64(h.offsets, h.indices, src)
    err = np.abs(bc.astype(np.float64) - bc64)
    ok_bc = bool(np.all(err <= 1e-4 * np.abs(bc64) + 1e-5))
    ok_sig = bool(np.array_equal(np.asarray(sig, np.float64), sig64))
    res["bc_rmat23_sym"] = dict(GTEPS=2 * e_r / t / 1e6, ms=t, rounds=st.rounds, **_roof(b, t, peak),
                                parity_vs_oracle=ok_bc and ok_sig,
                                parity_how="BC within 1e-4 relative + 1e-5 of the FP64 oracle, path counts exact",
                                max_rel_err_where_above_1=float(np.max(err[np.abs(bc64) > 1] / np.abs(bc64[np.abs(bc64) > 1]))
                                                                if np.any(np.abs(bc64) > 1) else 0.0),
                                cpu_GTEPS=2 * e_r / cpu_s / 1e9, cpu_ms=1e3 * cpu_s, cpu=cpu_kind)
    del bc64, sig64
    G.close()
    return res


def batched(ctx, cache, a):
    """Batched launches against one plain launch per query, same results required;
    a sample of the plain results is checked against the oracle."""
    import oracle
    import sepgraph as sg

    res = {}
    h = sg.HostGraph.rmat(22, 16, symmetric=True, seed=1)
    G = ctx.graph(h, symmetric=True)
    srcs = [int(s) for s in h.pick_sources(64, 11)]
    plain_ms, plain = 0.0, []
    for s in srcs:
        lv, st, _ = G.bfs(s)
        plain_ms += st.time_kernel_ms
        plain.append(lv)
    plain_ok = all(np.array_equal(plain[i], oracle.bfs(h.offsets, h.indices, srcs[i])) for i in range(4))
    ms_t, (outs, st_t, _) = _median_ms(lambda: ctx.bfs_batch([(G, s) for s in srcs]), 3)
    same_t = all((o == p).all() for o, p in zip(outs, plain))
    ms_m, (lv_m, st_m) = _median_ms(lambda: G.msbfs(srcs), 3)
    same_m = all((lv_m[i] == plain[i]).all() for i in range(len(srcs)))
    e = sum(reached_edges(h, p) for p in plain)
    res["bfs64_rmat22_sym"] = {
        "plain_ms": plain_ms, "plain_qps": 64 / (plain_ms * 1e-3), "plain_GTEPS": e / plain_ms / 1e6,
        "team_batch_ms": ms_t, "team_batch_qps": 64 / (ms_t * 1e-3), "team_batch_GTEPS": e / ms_t / 1e6,
        "team_blocks": st_t.vertices_reached, "teams": st_t.search_depth, "team_batch_same_results": same_t,
        "msbfs_ms": ms_m, "msbfs_qps": 64 / (ms_m * 1e-3), "msbfs_GTEPS": e / ms_m / 1e6, "msbfs_same_results": same_m,
        "plain_parity_vs_oracle_first4": plain_ok}
    del plain, outs, lv_m

    # the same on a high-diameter graph: 16 sources on the 4096x4096 grid
    hg = sg.HostGraph.grid(4096, 4096)
    Gg = ctx.graph(hg)
    gsrcs = [int(x) for x in hg.pick_sources(16, 12)]
    plain_g, plain_ms_g = [], 0.0
    for s_ in gsrcs:
        lv, st, _ = Gg.bfs(s_, max_iteration=1000000)
        plain_ms_g += st.time_kernel_ms
        plain_g.append(lv)
    ms_g, (lv_g, _) = _median_ms(lambda: Gg.msbfs(gsrcs, max_iteration=1000000), 3)
    res["bfs16_grid4096"] = {"plain_ms": plain_ms_g, "plain_qps": 16 / (plain_ms_g * 1e-3), "msbfs_ms": ms_g,
                             "msbfs_qps": 16 / (ms_g * 1e-3),
                             "msbfs_same_results": all((lv_g[i] == plain_g[i]).all() for i in range(16))}
    Gg.close()
    del hg, plain_g, lv_g

    srcs32 = srcs[:32]
    plain_ms, plain = 0.0, []
    for s in srcs32:
        bc, _, st = G.bc(s)
        plain_ms += st.time_total_ms
        plain.append(bc)
    bc_ok = True
    for i in range(2):
        bc64, _, _ = oracle.bc_f64(h.offsets, h.indices, srcs32[i])
        bc_ok &= bool(np.all(np.abs(plain[i] - bc64) <= 1e-4 * np.abs(bc64) + 1e-5))
    del bc64
    ms_b, (outs, st_b, _) = _median_ms(lambda: ctx.bc_batch([(G, s) for s in srcs32]), 3)
    same_b = all(np.allclose(o, p, rtol=1e-4, atol=1e-5) for o, p in zip(outs, plain))
    ms_mb, (rows_mb, _) = _median_ms(lambda: G.msbc(srcs32), 3)
    same_mb = all(np.allclose(rows_mb[i], plain[i], rtol=1e-4, atol=1e-5) for i in range(len(srcs32)))
    res["bc32_rmat22_sym"] = {"plain_ms": plain_ms, "plain_qps": 32 / (plain_ms * 1e-3), "batch_ms": ms_b,
                              "batch_qps": 32 / (ms_b * 1e-3), "same_results_rtol_1e-4": same_b,
                              "batch_GTEPS": st_b.edges_reached / ms_b / 1e6,
                              "msbc_ms": ms_mb, "msbc_qps": 32 / (ms_mb * 1e-3),
                              "msbc_same_results_rtol_1e-4": same_mb, "plain_parity_vs_oracle_first2": bc_ok}
    G.close()
    del h, plain, outs

    # 256 SSSP instances over RMAT scale 12-20 graphs (directed, weights [1,64))
    graphs = []
    for sc in range(12, 21):
        hh = sg.HostGraph.rmat(sc, 16, seed=100 + sc).gen_weights(1, 64, 200 + sc)
        graphs.append((hh, ctx.graph(hh, no_csc=True)))
    rng = random.Random(5)
    queries = []
    for k in range(256):
        hh, gg = graphs[k % len(graphs)]
        queries.append((gg, rng.randrange(hh.nv)))
    kw = dict(variant="async_push_dd", max_iteration=1000000)
    plain_ms, plain = 0.0, []
    for gg, s in queries:
        d, st, _ = gg.sssp(s, **kw)
        plain_ms += st.time_kernel_ms
        plain.append(d)
    sssp_ok = all(np.array_equal(plain[k], oracle.dijkstra(graphs[k % len(graphs)][0].offsets,
                                                         graphs[k % len(graphs)][0].indices,
                                                         graphs[k % len(graphs)][0].weights, queries[k][1]))
                  for k in range(0, 256, 16))
    ms_s, (outs, st_s, _) = _median_ms(lambda: ctx.sssp_batch(queries, **kw), 3)
    same_s = all((o == p).all() for o, p in zip(outs, plain))
    # the same batch planned once and replayed as a CUDA graph into device outputs
    import torch

    douts = [torch.empty(gg.nv, dtype=torch.int32, device="cuda") for gg, _ in queries]
    plan = ctx.batch_plan("sssp", queries, douts, **kw)
    plan_ms = []
    for _ in range(6):
        plan.launch()
        st_p, _ = plan.wait()
        plan_ms.append(st_p.time_kernel_ms)
    same_p = all((d.cpu().numpy().view(np.uint32) == p).all() for d, p in zip(douts, plain))
    captured = plan.captured
    plan.close()
    ms_p = statistics.median(plan_ms[1:])
    res["sssp256_rmat12-20"] = {"plain_ms": plain_ms, "plain_qps": 256 / (plain_ms * 1e-3), "batch_ms": ms_s,
                                "batch_qps": 256 / (ms_s * 1e-3), "same_results": same_s,
                                "batch_GTEPS": st_s.edges_reached / ms_s / 1e6, "teams": st_s.search_depth,
                                "team_blocks": st_s.vertices_reached, "plan_ms": ms_p,
                                "plan_qps": 256 / (ms_p * 1e-3), "plan_cuda_graph": captured,
                                "plan_same_results": same_p, "plain_parity_vs_oracle_every16th": sssp_ok}
    for _, gg in graphs:
        gg.close()
    return res


def _wall_ms(fn, reps=4):
    """Median wall ms of fn() between device synchronisations (the first call dropped);
    for host-orchestrated multi-kernel work such as graph construction."""
    import torch

    ts = []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        ts.append((time.perf_counter() - t0) * 1e3)
        if hasattr(r, "close"):
            r.close()
    return statistics.median(ts[1:])


def ingest(ctx, cache, a):
    """Graph construction on the device.  (1) sg_graph_create of a directed weighted
    RMAT-23 CSR already in HBM: validation plus the csr_tocsc transpose; algorithmic
    bytes = read CSR + write CSC = 2 * (4(V+1) + 8E).  (2) sg_graph_build of the RMAT-22
    raw edge stream (self-loops and duplicates kept, shuffled) under the converter's
    options.  CPU baseline: the reference's CSCGraph construction (csr_tocsc) on the
    RMAT-21 CSR, one thread; results checked against the oracle on smaller cases by the
    tests, and here against the host generator's CSR."""
    import oracle
    import sepgraph as sg
    import torch

    peak = peak_hbm()[0]
    res = {}
    h = sg.HostGraph.rmat(23, 16, seed=1).gen_weights(1, 64, 2)
    nv, ne = h.nv, len(h.indices)
    dev = [torch.from_numpy(x.view(np.int32)).cuda() for x in (h.offsets, h.indices, h.weights)]
    t_nocsc = _wall_ms(lambda: ctx.graph_from_csr(*dev, nv=nv, ne=ne, no_csc=True))
    t_csc = _wall_ms(lambda: ctx.graph_from_csr(*dev, nv=nv, ne=ne))
    t_tr = t_csc - t_nocsc
    tr_bytes = 2 * (4 * (nv + 1) + 8 * ne)
    res["transpose_rmat23_dir_w"] = dict(nv=nv, ne=ne, create_no_csc_ms=t_nocsc, create_with_csc_ms=t_csc,
                                         transpose_ms=t_tr, transpose_Gedges_s=ne / t_tr / 1e6,
                                         **_roof(tr_bytes, t_tr, peak))
    del dev, h
    hc = sg.HostGraph.rmat(21, 16, seed=1).gen_weights(1, 64, 2)
    if oracle.ref_available():
        cpu_s = _cpu_time(lambda: oracle.ref_csr_tocsc(hc.offsets, hc.indices, hc.weights), 20.0)
        kind = "reference CSCGraph (csr_tocsc) compiled from its sources, 1 thread"
    else:
        cpu_s = _cpu_time(lambda: oracle.csr_tocsc(hc.offsets, hc.indices, hc.weights), 20.0)
        kind = "oracle numpy port"
    res["transpose_rmat23_dir_w"].update(cpu_Gedges_s=len(hc.indices) / cpu_s / 1e9, cpu_sample="RMAT-21 directed weighted",
                                         cpu_ms=cpu_s * 1e3, cpu=kind)
    del hc

    raw = sg.HostGraph.rmat(22, 16, seed=1, keep_self_loops=True, keep_duplicates=True)
    s = np.repeat(np.arange(raw.nv, dtype=np.uint32), np.diff(raw.offsets.astype(np.int64)))
    d = raw.indices.copy()
    nv = raw.nv
    del raw
    p = np.random.default_rng(9).permutation(len(s))
    s, d = s[p], d[p]
    m = len(s)
    sd, dd = torch.from_numpy(s.view(np.int32)).cuda(), torch.from_numpy(d.view(np.int32)).cuda()
    del s, d, p
    out = {"edges_in": m}
    for name, kw in (("csr_input_order", dict(no_csc=True)), ("csr_sorted_rows", dict(sort_rows=True, no_csc=True)),
                     ("deself_dedup_sorted", dict(deself_cycle=True, deduplicate=True, sort_rows=True, no_csc=True)),
                     ("deself_d2ud", dict(deself_cycle=True, d2ud=True))):
        t = _wall_ms(lambda: ctx.build_graph(nv, sd, dd, m=m, **kw))
        out[name] = {"ms": t, "Medges_in_s": m / t / 1e3}
    G = ctx.build_graph(nv, sd, dd, m=m, deself_cycle=True, d2ud=True)
    off, idx, _ = G.copy_out()
    G.close()
    hs = sg.HostGraph.rmat(22, 16, symmetric=True, seed=1)
    out["d2ud_equals_host_symmetric_generator"] = bool(np.array_equal(off, hs.offsets) and np.array_equal(idx, hs.indices))
    res["build_rmat22_raw_shuffled"] = out
    return res


SERVED_MIX = (("bfs", 0.60), ("sssp", 0.25), ("pagerank", 0.10), ("bc", 0.05))


def served(ctx, cache, a):
    """Mixed query stream through the server: throughput when offered far above
    capacity, latency percentiles at 25 / 50 / 90 % of that capacity, and the plain
    one-query-per-launch path on a uniform sample of the stream (results compared)."""
    import sepgraph as sg
    import torch

    specs = [("rmat", sc) for sc in range(14, 23)] + [("grid", n) for n in (1024, 1448, 2048, 2560, 2896, 3584, 4096)]
    graphs = []
    for k, (kind, p) in enumerate(specs):
        if kind == "rmat" and p == 22 and "rmat22" in cache:
            hh, gg = cache["rmat22"]  # the headline graph (same generator and weights)
        elif kind == "rmat":
            hh = sg.HostGraph.rmat(p, 16, seed=300 + p).gen_weights(1, 64, 400 + p)
            gg = ctx.graph(hh)
            cache[f"served_rmat{p}"] = (hh, gg)
        else:
            hh = sg.HostGraph.grid(p, p).gen_weights(1, 64, 500 + p)
            gg = ctx.graph(hh)
            cache[f"served_grid{p}"] = (hh, gg)
        graphs.append((f"{kind}{p}", hh, gg))
    nq = a.served_queries
    rng = random.Random(17)
    names, probs = zip(*SERVED_MIX)
    queries = []
    n_rmat = sum(1 for kind, _ in specs if kind == "rmat")
    for _ in range(nq):
        algo = rng.choices(names, probs)[0]
        # BC draws from the RMAT graphs: shortest-path counts on a large grid
        # (C(2n, n) between opposite corners) exceed uint64 and any float type
        gid = rng.randrange(n_rmat if algo == "bc" else len(graphs))
        nv = graphs[gid][1].nv
        queries.append((algo, gid, rng.randrange(nv)))
    sample_every = 10
    sample = set(range(0, nq, sample_every))
    # outputs: sampled queries get their own arrays (compared below), the rest share per-graph sinks
    sinks = {}

    def pinned(n, dt):
        # result arrays in page-locked host memory, as a serving client keeps
        # them: device-to-host copies run at DMA speed (pageable copies are
        # staged through the driver and cost about 15 % of the served rate)
        return torch.zeros(n, dtype=torch.int32).pin_memory().numpy().view(dt)

    def out_for(i, algo, gid):
        dt = np.float32 if algo in ("pagerank", "bc") else np.uint32
        if i in sample:
            return pinned(graphs[gid][1].nv, dt)
        key = (gid, dt)
        if key not in sinks:
            sinks[key] = pinned(graphs[gid][1].nv, dt)
        return sinks[key]

    outs = [out_for(i, al, g) for i, (al, g, _) in enumerate(queries)]

    def stream(qs, rate, seed, **cfg):
        """Submits qs with Poisson arrivals at `rate` queries/s; returns statuses, wall seconds, server stats."""
        srv = sg.Server(0, **dict(dict(slots=a.served_slots, max_batch=256, blocks_per_sm=a.served_bps), **cfg))
        try:
            for _, _, gg in graphs:
                srv.add_graph(gg)
            tickets = [None] * len(qs)
            t_start = time.perf_counter()

            def producer():
                r = random.Random(seed)
                for i, (al, g, s) in enumerate(qs):
                    tickets[i] = srv.submit(al, g, s, outs[i])
                    time.sleep(r.expovariate(rate))

            th = threading.Thread(target=producer)
            th.start()
            th.join()
            sts = [srv.wait(t, 1800.0) for t in tickets]
            return sts, time.perf_counter() - t_start, srv.stats()
        finally:
            srv.close()

    rate = 5000.0  # offered load, queries/s (Poisson): far above capacity, measures throughput
    statuses, wall, st = stream(queries, rate, 23)
    failed = sum(1 for s_, _ in statuses if s_ != 0)
    capacity = nq / wall
    # the same overload with one graph per batch, shortest measured group first (the other policy)
    _, wall_one, _ = stream(queries, rate, 23, batch_graphs=1)
    # latency below capacity: Poisson streams offered at 25 / 50 / 90 % of the measured
    # throughput, each of about 12 s (at least 200 queries, at most the whole stream)
    loads = {}
    for f, bg in ((0.25, 0), (0.5, 0), (0.9, 0), (0.5, 1)):
        n = int(min(nq, max(200, 12.0 * f * capacity)))
        _, w, sl = stream(queries[:n], f * capacity, 29 + int(100 * f), batch_graphs=bg)
        key = f"{int(100 * f)}pct" + ("_one_graph_shortest_first" if bg == 1 else "")
        loads[key] = {"queries": n, "offered_qps": f * capacity, "served_qps": n / w,
                      "p50_ms": sl["p50_ms"], "p99_ms": sl["p99_ms"], "p999_ms": sl["p999_ms"]}

    # plain path: the sampled queries one at a time, results to host like the server's
    plain_lat, same, plain_failed, failed_plain = [], True, 0, set()
    mismatched, pr_l1_max = [], 0.0
    plain_out = {}  # pinned result arrays, as the served queries have
    for i in sorted(sample):
        al, g, s = queries[i]
        gg = graphs[g][2]
        key = (g, np.float32 if al in ("pagerank", "bc") else np.uint32)
        if key not in plain_out:
            plain_out[key] = pinned(graphs[g][1].nv, key[1])
        po = plain_out[key]
        t0 = time.perf_counter()
        try:
            if al == "bfs":
                o, _, _ = gg.bfs(s, out=po, max_iteration=1000000)
            elif al == "sssp":
                # the server's SSSP method (delta-stepping push, lookahead 4), one query per launch
                o, _, _ = gg.sssp(s, out=po, variant="async_push_dd", priority="low_high", local_depth=4,
                                  max_iteration=1000000)
            elif al == "pagerank":
                o, _, _ = gg.pagerank(out=po, pr_error=1e-7, max_iteration=100000)
            else:
                o, _, _ = gg.bc(s, out=po, max_iteration=1000000)
        except sg.SGError:
            plain_failed += 1
            failed_plain.add(i)
            same &= statuses[i][0] != 0  # the served query must have failed too
            continue
        plain_lat.append(1e3 * (time.perf_counter() - t0))
        if al in ("bfs", "sssp"):
            ok = bool((o == outs[i]).all())
        elif al == "pagerank":
            x, y = np.asarray(o, np.float64), np.asarray(outs[i], np.float64)
            l1 = float(np.abs(x / x.sum() - y / y.sum()).sum())
            pr_l1_max = max(pr_l1_max, l1)
            ok = l1 <= 2e-6  # each within 1e-6 of the fixed point, whichever variants the policy ran
        else:
            ok = bool(np.allclose(o, outs[i], rtol=1e-4, atol=1e-5))
        same &= ok
        if not ok:
            mismatched.append(f"{al}@{graphs[g][0]}")
    by_algo = {}
    for i, ms in zip([i for i in sorted(sample) if i not in failed_plain], plain_lat):
        al = queries[i][0]
        cnt, tot = by_algo.get(al, (0, 0.0))
        by_algo[al] = (cnt + 1, tot + ms)
    plain_lat_sorted = sorted(plain_lat)

    def pct(v, p):
        return v[min(len(v) - 1, int(p * (len(v) - 1) + 0.5))]

    plain_qps = len(plain_lat) / (sum(plain_lat) * 1e-3)
    served_qps = nq / wall
    return {
        "queries": nq, "offered_qps": rate, "mix": dict(SERVED_MIX), "graphs": [n for n, _, _ in graphs],
        "stream_note": f"{nq} queries of the 100k-query configuration (same mix, graphs and arrival process); "
                       f"the full 100k would take about {100000 / served_qps / 60:.0f} minutes at this rate",
        "served_qps": served_qps, "server_qps_first_to_last": st["qps"], "p50_ms": st["p50_ms"],
        "p99_ms": st["p99_ms"], "p999_ms": st["p999_ms"], "max_ms": st["max_ms"], "batches": st["batches"],
        "load_points": loads, "batch_graphs": "mixed-graph batches from the oldest query (default)",
        "slots": a.served_slots, "outputs": "pinned host arrays, served and plain alike",
        "one_graph_shortest_first_qps": nq / wall_one,
        "policies": "default: mixed-graph batches from the oldest query; compared: one graph per batch, "
                    "shortest measured (algorithm, graph) group first with a 500 ms aging bound",
        "failed": failed, "plain_failed": plain_failed, "hbm_peak_bytes": st["hbm_peak"],
        "hbm_budget_bytes": st["hbm_budget"], "sssp": "delta-stepping (push, two-level priority, lookahead 4), each graph's delta heuristic",
        "plain_sample": len(plain_lat), "plain_qps": plain_qps, "plain_p50_ms": pct(plain_lat_sorted, 0.5),
        "plain_p99_ms": pct(plain_lat_sorted, 0.99), "speedup_qps": served_qps / plain_qps,
        "sample_results_same": same, "mismatched": mismatched, "pagerank_l1_max": pr_l1_max,
        "plain_ms_by_algo": {k: {"queries": c, "mean_ms": t / c} for k, (c, t) in by_algo.items()},
        "note": "plain path = one blocking call per query on the sampled 1-in-10 queries, service time only "
                "(no queueing), each algorithm with the server's method (SSSP: delta-stepping push, "
                "lookahead 4); served latency includes queueing under the offered Poisson load",
    }


def main():
    a = args_parse()
    if a.profile:
        run_profile(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
