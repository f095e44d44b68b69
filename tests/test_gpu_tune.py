"""Autotuner: every candidate reproduces the first one's result, the chosen
options are one of the candidates and give the oracle's result again."""
import numpy as np
import pytest

import oracle
import sepgraph as sg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = sg.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("algo", ["bfs", "sssp", "pagerank", "bc"])
def test_autotune_candidates_agree(ctx, algo):
    sym = algo in ("bfs", "bc")
    h = sg.HostGraph.rmat(12, 16, symmetric=sym, seed=4)
    if algo == "sssp":
        h.gen_weights(1, 64, 5)
    G = ctx.graph(h, symmetric=sym)
    srcs = h.pick_sources(2, 9)
    best, ms, report = G.autotune(algo, srcs, max_iteration=100000, pr_error=1e-7)
    assert report and all(r["status"] == 0 for r in report), report
    assert ms > 0 and ms == min(r["ms"] for r in report)
    s = int(srcs[0])
    if algo == "bfs":
        assert (G.bfs(s, max_iteration=100000, **best)[0] == oracle.bfs(h.offsets, h.indices, s)).all()
    elif algo == "sssp":
        got = G.sssp(s, max_iteration=100000, **best)[0]
        assert (got == oracle.sssp(h.offsets, h.indices, h.weights, s)).all()


def test_autotune_rejects_bad_input(ctx):
    h = sg.HostGraph.rmat(8, 8, seed=1)
    G = ctx.graph(h)
    with pytest.raises(sg.SGError):
        G.autotune("bfs", [])  # a source-based algorithm needs sources
    with pytest.raises(sg.SGError):
        G.autotune("sssp", [h.nv])
