"""Graph fixtures shared by the tests and tests/golden/make_golden.py.

They rebuild, in this project's own code, the graph families the reference's
GPU tests use:
  - the named catalog (crates/grafeo-cuda-algos/tests/correctness.rs:120-172),
  - the "messy" export case with self-loops, parallel edges and a deleted node
    (correctness.rs:174-210), reproduced through from_edge_pairs, whose dedup
    and self-loop rules equal the Grafeo export's (csr_export.rs:130-135),
  - the property-test strategy: n in [1, 16) nodes and up to 48 random pairs
    (correctness.rs:483-513), drawn here from a seeded numpy generator,
  - the roundtrip fixtures K4 / path5 (tests/roundtrip.rs:9-41) and the
    wide-frontier BFS regression graph (roundtrip.rs:186-222).
Every graph is returned as undirected edge pairs plus a node count; the
symmetric CSR is built with the library's from_edge_pairs or the oracle's.
"""
from __future__ import annotations

import numpy as np


def complete_edges(n: int) -> list[tuple[int, int]]:
    return [(i, j) for i in range(n) for j in range(i + 1, n)]


def path_edges(n: int) -> list[tuple[int, int]]:
    return [(i - 1, i) for i in range(1, n)]


def catalog() -> list[tuple[str, int, list[tuple[int, int]]]]:
    """(name, num_nodes, undirected edges) for the reference's named graphs."""
    # Petersen graph: outer 5-cycle, spokes, inner pentagram.
    petersen = [(i, (i + 1) % 5) for i in range(5)] + [(i, i + 5) for i in range(5)]
    petersen += [(5 + i, 5 + (i + 2) % 5) for i in range(5)]
    star = [(0, leaf) for leaf in range(1, 9)]
    wheel = [(0, i) for i in range(1, 7)] + [(i, i % 6 + 1) for i in range(1, 7)]
    two_k4 = complete_edges(4) + [(a + 4, b + 4) for a, b in complete_edges(4)] + [(3, 4)]
    k4_tail = complete_edges(4) + [(3, 4), (4, 5)]
    return [
        ("single node", 1, []),
        ("edgeless", 4, []),
        ("K4", 4, complete_edges(4)),
        ("K5", 5, complete_edges(5)),
        ("K7", 7, complete_edges(7)),
        ("path", 10, path_edges(10)),
        ("petersen", 10, petersen),
        ("star", 9, star),
        ("wheel", 7, wheel),
        ("diamond", 4, [(0, 1), (0, 2), (1, 2), (1, 3), (2, 3)]),
        ("bowtie", 5, [(0, 1), (0, 2), (1, 2), (0, 3), (0, 4), (3, 4)]),
        ("triangle, edge and isolated nodes", 7, [(0, 1), (1, 2), (0, 2), (3, 4)]),
        ("two K4 joined by a bridge", 8, two_k4),
        ("K4 with a tail", 6, k4_tail),
    ]


def messy(self_loops: bool = True, parallel_edges: bool = True) -> tuple[int, list[tuple[int, int]]]:
    """The messy export case after node 2 is deleted: 6 live nodes.

    Base graph on 7 nodes, optional self-loops at 0 and 4 and parallel copies
    of four edges; deleting node 2 drops its edges (detached or not, the
    export skips edges to deleted nodes) and renumbers 0,1,3,4,5,6 -> 0..5.
    """
    base = [(0, 1), (1, 3), (0, 3), (3, 4), (4, 5), (5, 3), (1, 2), (2, 6), (6, 0), (5, 6), (4, 6)]
    edges = list(base)
    if self_loops:
        edges += [(0, 0), (4, 4)]
    if parallel_edges:
        edges += [(0, 1), (4, 3), (5, 6), (6, 5)]
    live = [0, 1, 3, 4, 5, 6]
    remap = {old: new for new, old in enumerate(live)}
    kept = [(remap[a], remap[b]) for a, b in edges if a in remap and b in remap]
    return len(live), kept


def random_graphs(count: int = 48, seed: int = 20240531) -> list[tuple[int, list[tuple[int, int]]]]:
    """Property-test graphs: n in [1, 16), up to 48 pairs (self-loops and repeats allowed)."""
    rng = np.random.default_rng(seed)
    out = [(1, [])]  # the recorded shrink case (correctness.proptest-regressions:7)
    while len(out) < count:
        n = int(rng.integers(1, 16))
        m = int(rng.integers(0, 49))
        pairs = [(int(a), int(b)) for a, b in rng.integers(0, n, size=(m, 2))]
        out.append((n, pairs))
    return out


def wide_frontier(width: int = 500_000, depth: int = 4):
    """roundtrip.rs:186-222: 0 - 1, then 1 fans out to `width` chains of `depth` nodes."""
    num_nodes = 2 + depth * width
    chains = np.arange(width, dtype=np.uint32)
    parts = [np.array([[0, 1]], dtype=np.uint32)]
    first = 2 + chains
    parts.append(np.stack([np.ones(width, dtype=np.uint32), first], axis=1))
    for level in range(3, depth + 2):
        prev = 2 + (level - 3) * width + chains
        cur = 2 + (level - 2) * width + chains
        parts.append(np.stack([prev, cur], axis=1).astype(np.uint32))
    pairs = np.concatenate(parts)
    expected = np.concatenate(
        [np.array([0, 1], dtype=np.int32)] + [np.full(width, lvl, dtype=np.int32) for lvl in range(2, depth + 2)]
    )
    return num_nodes, pairs, expected


K4_CSR = ([0, 3, 6, 9, 12], [1, 2, 3, 0, 2, 3, 0, 1, 3, 0, 1, 2])
PATH5_CSR = ([0, 1, 3, 5, 7, 8], [1, 0, 2, 1, 3, 2, 4, 3])
