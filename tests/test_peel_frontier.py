"""The frontier rule of the k-truss peeling, restated on the host.

csrc/ktruss.cu removes, from its third round on (`k_truss`) or after the
first round of a level (truss decomposition), exactly the edges that the
previous round's peel brought below the threshold, instead of scanning every
alive edge. These restatements run both forms on small random graphs (with
self-loops and parallel edges) and require the same rounds, survivors and
trussness. The scanning form is the reference's round rule
(crates/grafeo-cuda-algos/src/k_truss.rs: remove every edge with support
< k - 2, self-loop terms in round 1 only); the frontier form is the device's.
"""
from __future__ import annotations

import random

import pytest


def build(n, pairs):
    adj = [set() for _ in range(n)]
    loops = [0] * n
    for a, b in pairs:
        if a == b:
            loops[a] = 1
        else:
            adj[a].add(b)
            adj[b].add(a)
    edges = sorted({(min(a, b), max(a, b)) for a, b in pairs if a != b})
    eid = {e: i for i, e in enumerate(edges)}
    support = [len(adj[a] & adj[b]) for a, b in edges]
    return adj, loops, edges, eid, support


def peel(adj, edges, eid, state, support, removed, rnd, threshold, crossed):
    """Every triangle of a removed edge that is alive at the start of round
    rnd is destroyed once (by its removed edge with the smallest id); its
    surviving edges lose one support. With `crossed`, an edge whose support
    falls from the threshold to below it is appended there."""
    for e in removed:
        a, b = edges[e]
        for w in adj[a] & adj[b]:
            e1 = eid[(min(a, w), max(a, w))]
            e2 = eid[(min(b, w), max(b, w))]
            s1, s2 = state[e1], state[e2]
            if (s1 != 0 and s1 != rnd) or (s2 != 0 and s2 != rnd):
                continue
            if (s1 == rnd and e1 < e) or (s2 == rnd and e2 < e):
                continue
            for ex, sx in ((e1, s1), (e2, s2)):
                if sx == 0:
                    old = support[ex]
                    support[ex] -= 1
                    if crossed is not None and old == threshold:
                        crossed.append(ex)


def below(edges, loops, state, support, threshold, rnd):
    extra = (lambda a, b: loops[a] + loops[b]) if rnd == 1 else (lambda a, b: 0)
    return [i for i, (a, b) in enumerate(edges)
            if state[i] == 0 and support[i] + extra(a, b) < threshold]


def k_truss_scanning(n, pairs, k):
    adj, loops, edges, eid, support = build(n, pairs)
    state = [0] * len(edges)
    rnd = 1
    while True:
        removed = below(edges, loops, state, support, k - 2, rnd)
        if not removed and not (rnd == 1 and any(loops)):
            break
        for e in removed:
            state[e] = rnd
        peel(adj, edges, eid, state, support, removed, rnd, k - 2, None)
        rnd += 1
    return rnd, [e for i, e in enumerate(edges) if state[i] == 0]


def k_truss_frontier(n, pairs, k):
    adj, loops, edges, eid, support = build(n, pairs)
    state = [0] * len(edges)
    rnd = 1
    crossed = []
    while True:
        if rnd == 1 or (rnd == 2 and any(loops)):
            removed = below(edges, loops, state, support, k - 2, rnd)
        else:
            removed = crossed
        for e in removed:
            state[e] = rnd
        if not removed and not (rnd == 1 and any(loops)):
            break
        crossed = []
        peel(adj, edges, eid, state, support, removed, rnd, k - 2, crossed)
        rnd += 1
    return rnd, [e for i, e in enumerate(edges) if state[i] == 0]


def decomposition(n, pairs, frontier):
    adj, loops, edges, eid, support = build(n, pairs)
    state = [0] * len(edges)
    truss = [0] * len(edges)
    alive = len(edges)
    rnd, k, top = 0, 3, (2 if alive else 0)
    level_start = True
    crossed = []
    while alive > 0:
        rnd += 1
        if level_start or not frontier:
            removed = below(edges, loops, state, support, k - 2, 0)
        else:
            removed = crossed
        for e in removed:
            state[e] = rnd
            truss[e] = k - 1
        if not removed:
            top, k, level_start = k, k + 1, True
            continue
        alive -= len(removed)
        crossed = []
        peel(adj, edges, eid, state, support, removed, rnd, k - 2, crossed)
        level_start = False
    return rnd, top, truss


@pytest.mark.parametrize("seed", range(4))
def test_frontier_rounds_match_scanning_rounds(seed):
    rng = random.Random(seed)
    for _ in range(100):
        n = rng.randint(2, 25)
        pairs = [(rng.randrange(n), rng.randrange(n)) for _ in range(rng.randint(0, n * 5))]
        for k in (2, 3, 4, 5, 6):
            assert k_truss_scanning(n, pairs, k) == k_truss_frontier(n, pairs, k), (pairs, k)
        plain = [(a, b) for a, b in pairs if a != b]
        assert decomposition(n, plain, False) == decomposition(n, plain, True), plain
