"""The triangle count's orientation and edge split, restated on the host.

csrc/triangle.cu counts the triangles of a symmetric CSR over a DAG oriented
by degree-class rank (classes of list length [2^(c-1), 2^c) in descending
order, ids ascending inside a class; an edge points at the lower rank), and
splits the DAG edges u -> v between two kernels: the tail side (the table
holds N+(u), N+(v) is streamed) when d+(v) <= d+(u) or d+(u) < 2, the head side
(the table holds N+(v), N+(u) is streamed) when 2 <= d+(u) < d+(v). Its CTA
kernels replace the table by a bitmap of the ranks below the owner's rank,
which holds the owner's whole out-list only because every out-neighbour ranks
below its owner. These restatements check, on random graphs and the golden
catalog, that the split covers every edge once and gives the oracle's count,
and that the ranking property holds.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O


def degree_class_rank(offsets: np.ndarray) -> np.ndarray:
    deg = np.diff(offsets.astype(np.int64))
    cls = np.zeros_like(deg)
    nz = deg > 0
    cls[nz] = np.floor(np.log2(deg[nz])).astype(np.int64) + 1
    order = np.lexsort((np.arange(len(deg)), -cls))  # class descending, id ascending
    rank = np.empty(len(deg), dtype=np.int64)
    rank[order] = np.arange(len(deg))
    return rank


def ranked_dag(offsets: np.ndarray, targets: np.ndarray):
    rank = degree_class_rank(offsets)
    n = len(offsets) - 1
    src = np.repeat(np.arange(n), np.diff(offsets.astype(np.int64)))
    keep = rank[targets] < rank[src]
    out = [set() for _ in range(n)]
    for u, v in zip(src[keep].tolist(), targets[keep].tolist()):
        out[u].add(v)
    return rank, out


def split_count(out) -> tuple[int, int, int]:
    dp = [len(x) for x in out]
    tail = head = covered = 0
    for u, nu in enumerate(out):
        for v in nu:
            covered += 1
            if dp[u] >= 2 and dp[u] < dp[v]:
                head += len(out[v] & nu)  # table N+(v), N+(u) streamed
            else:
                tail += len(nu & out[v])  # table N+(u), N+(v) streamed
    return tail, head, covered


def random_symmetric(rng, n: int, m: int):
    pairs = {(int(a), int(b)) for a, b in rng.integers(0, n, size=(m, 2)) if a != b}
    adj = [set() for _ in range(n)]
    for a, b in pairs:
        adj[a].add(b)
        adj[b].add(a)
    offsets = np.zeros(n + 1, dtype=np.uint32)
    offsets[1:] = np.cumsum([len(x) for x in adj])
    targets = np.array([w for x in adj for w in sorted(x)], dtype=np.uint32)
    return offsets, targets


def check(offsets, targets):
    offsets = np.asarray(offsets, dtype=np.uint32)
    targets = np.asarray(targets, dtype=np.int64)
    rank, out = ranked_dag(offsets, targets)
    for u, nu in enumerate(out):
        assert all(rank[v] < rank[u] for v in nu)  # the bitmap of ranks below rank[u] holds N+(u)
    tail, head, covered = split_count(out)
    src = np.repeat(np.arange(len(offsets) - 1), np.diff(offsets.astype(np.int64)))
    loops = int(np.sum(targets == src))
    assert covered * 2 == len(targets) - loops  # every undirected edge once
    assert tail + head == O.triangle_count(offsets, targets.astype(np.uint32))


@pytest.mark.parametrize("seed", range(3))
def test_ranked_split_counts_every_triangle_once(seed):
    rng = np.random.default_rng(seed)
    for _ in range(60):
        n = int(rng.integers(3, 80))
        offsets, targets = random_symmetric(rng, n, int(rng.integers(0, n * 8)))
        check(offsets, targets)


def test_ranked_split_on_golden_graphs(golden_graphs):
    for g in golden_graphs:
        o = np.asarray(g["offsets"], dtype=np.int64)
        t = np.asarray(g["targets"], dtype=np.int64)
        n = len(o) - 1
        src = np.repeat(np.arange(n), np.diff(o))
        sym = set(zip(src.tolist(), t.tolist()))
        if all((b, a) in sym for a, b in sym):
            check(o, t)
