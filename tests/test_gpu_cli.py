"""The sample executables end to end on the GPU: each runs on a generated
graph with --check, --trace and --json, exits 0 (its check passed), and writes
a run record with the keys and value types of the reference's
Engine::SaveToJson (framework.cuh:205-257) plus the sample's own."""
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "sep-graph_b200", "bin")

TIME_KEYS = ["time_input_active_node", "time_output_active_node", "time_input_workload", "time_output_workload",
             "time_queue2bitmap", "time_bitmap2queue", "time_rebuild_worklist", "time_priority_sample",
             "time_sort_worklist", "time_unique_worklist", "time_kernel", "time_total", "time_per_round"]
STRING_KEYS = ["priority_type", "fused_kernel", "max_iteration_reached", "device", "dataset", "algo_type"]

SAMPLES = {
    "hybrid_bfs": (["--source_node=0"], "TRAVERSAL_SCHEME", {"non_atomic"}),
    "hybrid_sssp": (["--source_node=0", "--gen_weights", "--prio_delta=50"], "TRAVERSAL_SCHEME", {"priority_delta"}),
    "hybrid_pr": (["--error=1e-5", "--max_iteration=1000"], "ITERATIVE_SCHEME", {"error_tolerance"}),
    "hybrid_bc": (["--source_node=0"], "TRAVERSAL_SCHEME", {"time_stage2"}),
}


@pytest.mark.parametrize("sample", sorted(SAMPLES))
def test_sample_run_record(sample, tmp_path):
    exe = os.path.join(BIN, sample)
    if not os.path.exists(exe):
        pytest.fail(f"{exe} not built")
    extra, algo_type, own = SAMPLES[sample]
    out = tmp_path / "run.json"
    cmd = [exe, "--gen_graph", "--gen_method=4", "--gen_rmat_scale=12", "--gen_factor=8", "--check", "--trace",
           "--lb_push=fine", f"--json={out}"] + extra
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    rec = json.loads(out.read_text())
    for k in TIME_KEYS:
        assert isinstance(rec[k], (int, float)) and rec[k] >= 0, k
    for k in STRING_KEYS:
        assert isinstance(rec[k], str), k
    assert isinstance(rec["num_iteration"], int) and rec["num_iteration"] >= 1
    assert isinstance(rec["nnodes"], int) and rec["nnodes"] == 4096
    assert isinstance(rec["nedges"], int) and rec["nedges"] > 0
    assert rec["algo_type"] == algo_type
    assert rec["force_push_load_balancing"] == "FINE_GRAINED"
    assert rec["fused_kernel"] in ("YES", "NO") and rec["max_iteration_reached"] in ("YES", "NO")
    assert rec["priority_type"] == ("low_high" if sample == "hybrid_sssp" else "none")
    assert len(rec["round"]) == rec["num_iteration"]
    assert all(line.startswith("Round: ") for line in rec["round"])
    assert own <= set(rec), own - set(rec)
    assert list(rec) == sorted(rec)  # keys in the reference writer's (sorted) order
