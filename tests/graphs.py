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


# ---------------------------------------------------------------- generator restatements
# numpy restatements of the device generators (csrc/build_csr.cu), used to
# check them pair for pair: SplitMix64 stream value n of `state` is
# mix(state + (n + 1) * gamma), state = mix(seed + gamma).

_C1, _C2 = np.uint64(0xBF58476D1CE4E5B9), np.uint64(0x94D049BB133111EB)
_GAMMA = np.uint64(0x9E3779B97F4A7C15)


def _mix(z: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * _C1
        z = (z ^ (z >> np.uint64(27))) * _C2
    return z ^ (z >> np.uint64(31))


def _state(seed: int) -> np.uint64:
    with np.errstate(over="ignore"):
        return _mix(np.array([np.uint64(seed) + _GAMMA], dtype=np.uint64))[0]


def _stream(state, idx: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        return _mix(np.uint64(state) + (idx.astype(np.uint64) + np.uint64(1)) * _GAMMA)


def _unit(r: np.ndarray) -> np.ndarray:
    return (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _scale_to(r: np.ndarray, n: int) -> np.ndarray:
    """floor(r * n / 2^64) for n < 2^32."""
    hi, lo = r >> np.uint64(32), r & np.uint64(0xFFFFFFFF)
    n = np.uint64(n)
    return ((hi * n + ((lo * n) >> np.uint64(32))) >> np.uint64(32)).astype(np.uint32)


def symmetric_csr(n: int, src: np.ndarray, dst: np.ndarray):
    """Symmetric, loop-free, deduplicated CSR of undirected pairs."""
    keep = src != dst
    s = np.concatenate([src[keep], dst[keep]]).astype(np.uint64)
    d = np.concatenate([dst[keep], src[keep]]).astype(np.uint64)
    keys = np.unique((s << np.uint64(32)) | d)
    offsets = np.zeros(n + 1, dtype=np.uint32)
    np.add.at(offsets, (keys >> np.uint64(32)).astype(np.int64) + 1, 1)
    return np.cumsum(offsets, dtype=np.uint64).astype(np.uint32), (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def rmat_pairs(scale: int, edge_factor: int, a: float, b: float, c: float, seed: int):
    """R-MAT pairs: pair i picks one quadrant per level (top bit first) from
    draw i * scale + level: below a (0, 0), below a + b (0, 1), below
    a + b + c (1, 0), else (1, 1)."""
    m = edge_factor << scale
    u = _unit(_stream(_state(seed), np.arange(m * scale, dtype=np.uint64))).reshape(m, scale)
    row = (u >= a + b).astype(np.uint32)
    col = (((u >= a) & (u < a + b)) | (u >= a + b + c)).astype(np.uint32)
    weights = (np.uint32(1) << np.arange(scale - 1, -1, -1, dtype=np.uint32))
    return (row * weights).sum(axis=1).astype(np.uint32), (col * weights).sum(axis=1).astype(np.uint32)


def grid_pairs(width: int, height: int, drop: float, seed: int):
    horizontal = height * (width - 1)
    e = np.arange(horizontal + (height - 1) * width, dtype=np.uint64)
    keep = _unit(_stream(_state(seed), e)) >= drop
    y, x = e // max(width - 1, 1), e % max(width - 1, 1)
    src = np.where(e < horizontal, y * width + x, e - horizontal)
    dst = np.where(e < horizontal, src + 1, src + width)
    return src[keep].astype(np.uint32), dst[keep].astype(np.uint32)


def watts_strogatz_pairs(n: int, k: int, p: float, seed: int):
    half = k // 2
    idx = np.arange(n * half, dtype=np.uint64)
    state = _state(seed)
    src = idx // np.uint64(half)
    j = idx - src * np.uint64(half) + np.uint64(1)
    dst = ((src + j) % np.uint64(n)).astype(np.uint32)
    rewire = _unit(_stream(state, 2 * idx)) < p
    dst = np.where(rewire, _scale_to(_stream(state, 2 * idx + np.uint64(1)), n), dst)
    return src.astype(np.uint32), dst.astype(np.uint32)


def geometric_pairs(n: int, avg_degree: float, seed: int):
    """All pairs within r, (n - 1) pi r^2 = avg_degree (O(n^2): small n)."""
    i = np.arange(n, dtype=np.uint64)
    state = _state(seed)
    x, y = _unit(_stream(state, 2 * i)), _unit(_stream(state, 2 * i + np.uint64(1)))
    r = np.sqrt(avg_degree / (np.pi * (n - 1))) if n > 1 else 1.0
    r2 = r * r
    dx = x[:, None] - x[None, :]
    dy = y[:, None] - y[None, :]
    a, b = np.nonzero(np.triu((dx * dx + dy * dy) <= r2, k=1))
    return a.astype(np.uint32), b.astype(np.uint32)
