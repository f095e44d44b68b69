"""A CPU model of the push-only multi-source BFS kernel's round
(`msbfs_fused_kernel` in sep-graph_b200/csrc/sg_batch.cu), run under random
interleavings of its threads' memory operations and with stale reads, to
check the argument its correctness rests on: levels equal single-source BFS
levels whatever a thread reads of a neighbour that another thread is settling.

Model of one round k with parity p (q = p ^ 1), one thread per listed vertex u:
  settle:  was = seen[u]; nx = next[p][u]; nb = nx & ~was; next[p][u] = 0;
           if nb: seen[u] = was | nb; levels[s][u] = k for each bit s of nb
  expand:  for each out-neighbour w: sn = seen[w]; nq = next[q][w];
           add = nb & ~sn; if add and (nq & add) != add:
               old = atomic_or(next[q][w], add); if old == 0: list w in T[q]
Plain reads (seen, the next pre-check) may return any value the location held
since the last barrier (the barrier orders everything before it); the
atomic OR is exact.  The threads' steps interleave at random.
"""
import random

import numpy as np
import pytest

import oracle

INF = 0xFFFFFFFF


class Loc:
    """A memory word whose plain reads may return any value written since the last barrier."""

    def __init__(self):
        self.hist = [0]

    def read(self, rng):
        return rng.choice(self.hist)

    def read_exact(self):
        return self.hist[-1]

    def write(self, v):
        self.hist.append(v)

    def barrier(self):
        self.hist = [self.hist[-1]]


def model_msbfs(nv, adj, sources, rng, max_rounds=10**6):
    seen = [Loc() for _ in range(nv)]
    nxt = [[Loc() for _ in range(nv)], [Loc() for _ in range(nv)]]
    levels = np.full((len(sources), nv), INF, np.uint32)
    lists = [[], []]
    for i, s in enumerate(sources):  # the sources' bits pending in next[0]
        old = nxt[0][s].read_exact()
        nxt[0][s].write(old | (1 << i))
        if old == 0:
            lists[0].append(s)
    k, p = 0, 0
    while True:
        q = p ^ 1
        expand = k < max_rounds
        appended = []

        def thread(u):
            was = seen[u].read(rng)
            yield
            nx = nxt[p][u].read_exact()  # only the settling thread touches next[p][u] this round
            nb = nx & ~was
            nxt[p][u].write(0)
            yield
            if not nb:
                return
            seen[u].write(was | nb)
            for s in range(len(sources)):
                if (nb >> s) & 1:
                    assert levels[s][u] == INF, "a (source, vertex) pair settled twice"
                    levels[s][u] = k
            yield
            if not expand:
                return
            for w in adj[u]:
                sn = seen[w].read(rng)
                nq = nxt[q][w].read(rng)
                yield
                add = nb & ~sn
                if add and (nq & add) != add:
                    old = nxt[q][w].read_exact()
                    nxt[q][w].write(old | add)
                    if old == 0:
                        appended.append(w)
                yield

        live = [thread(u) for u in lists[p]]
        while live:
            t = rng.randrange(len(live))
            try:
                next(live[t])
            except StopIteration:
                live.pop(t)
        assert len(appended) == len(set(appended)), "a vertex listed twice in one round"
        for loc in seen + nxt[0] + nxt[1]:
            loc.barrier()
        lists[p] = []
        lists[q] = appended
        k += 1
        if not appended or not expand:
            break
        p = q
    return levels


def _random_sparse(nv, rng):
    adj = [set() for _ in range(nv)]
    for v in range(nv - 1):  # a path keeps most vertices reachable
        adj[v].add(v + 1)
    for _ in range(2 * nv):
        a, b = rng.randrange(nv), rng.randrange(nv)
        if a != b:
            adj[a].add(b)
    adj = [sorted(x) for x in adj]
    off = np.zeros(nv + 1, np.uint32)
    off[1:] = np.cumsum([len(x) for x in adj])
    idx = np.array([w for x in adj for w in x], np.uint32)
    return adj, off, idx


@pytest.mark.parametrize("seed", range(12))
def test_model_levels_equal_bfs_under_any_interleaving(seed):
    rng = random.Random(seed)
    nv = rng.randrange(8, 40)
    adj, off, idx = _random_sparse(nv, rng)
    sources = [rng.randrange(nv) for _ in range(rng.randrange(1, 9))]
    sources.append(sources[0])  # a duplicate source
    for trial in range(6):
        lv = model_msbfs(nv, adj, sources, random.Random(1000 * seed + trial))
        for i, s in enumerate(sources):
            assert (lv[i] == oracle.bfs(off, idx, s)).all(), (seed, trial, i)


@pytest.mark.parametrize("max_rounds", [0, 1, 3])
def test_model_round_limit_settles_levels_up_to_it(max_rounds):
    rng = random.Random(7)
    adj, off, idx = _random_sparse(30, rng)
    sources = [0, 5, 17]
    lv = model_msbfs(30, adj, sources, random.Random(3), max_rounds=max_rounds)
    for i, s in enumerate(sources):
        full = oracle.bfs(off, idx, s)
        assert (lv[i] == np.where(full <= max_rounds, full, np.uint32(INF))).all()
