"""Generates the golden fixtures in this directory.

Run from the repository root:  python tests/golden/make_golden.py

Two files:
  reference_pins.json  the literal known answers written in the reference's
                       own tests, each with the file:line it comes from;
  catalog.json         for every graph of tests/graphs.py (the reference's
                       catalog, the messy export case and 48 property-test
                       graphs): its symmetric CSR, built here in pure Python,
                       and triangle count, BFS levels from every source,
                       PageRank and the k-trusses for k = 3..8, all computed
                       by networkx (an independent implementation, imported,
                       never copied). PageRank runs to tol 1e-13 so the
                       fixed point is what gets pinned.
The oracle (oracle/oracle.c) is checked against both by tests/test_oracle.py.
"""
from __future__ import annotations

import json
import os
import sys

import networkx as nx

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import graphs  # noqa: E402


def symmetric_csr(n: int, edges) -> tuple[list[int], list[int]]:
    adj = [set() for _ in range(n)]
    for a, b in edges:
        adj[a].add(b)
        adj[b].add(a)
    offsets, targets = [0], []
    for v in range(n):
        targets.extend(sorted(adj[v]))
        offsets.append(len(targets))
    return offsets, targets


def record(name: str, n: int, edges) -> dict:
    g = nx.Graph()
    g.add_nodes_from(range(n))
    g.add_edges_from(edges)
    simple = g.copy()
    simple.remove_edges_from(list(nx.selfloop_edges(simple)))
    offsets, targets = symmetric_csr(n, edges)
    bfs = []
    for s in range(n):
        lengths = nx.single_source_shortest_path_length(g, s)
        dist = [lengths.get(v, -1) for v in range(n)]
        bfs.append({"source": s, "distances": dist, "reachable": len(lengths), "max_depth": max(lengths.values())})
    pr = nx.pagerank(g, alpha=0.85, tol=1e-13, max_iter=100000) if n else {}
    trusses = {}
    for k in range(3, 9):
        h = nx.k_truss(simple, k)
        trusses[str(k)] = sorted([min(a, b), max(a, b)] for a, b in h.edges())
    return {
        "name": name,
        "num_nodes": n,
        "edges": [list(e) for e in edges],
        "offsets": offsets,
        "targets": targets,
        "triangles": sum(nx.triangles(simple).values()) // 3,
        "bfs": bfs,
        "pagerank": [pr[v] for v in range(n)],
        "k_truss": trusses,
    }


def pins() -> dict:
    """Literal values from the reference's tests (paths inside grafeo-cuda)."""
    return {
        "triangles": [
            {"graph": "K4", "value": 4, "source": "crates/grafeo-cuda-algos/tests/roundtrip.rs:53-58"},
            {"graph": "K5", "value": 10, "source": "crates/grafeo-cuda-algos/tests/correctness.rs:344-352"},
            {"graph": "path5", "value": 0, "source": "crates/grafeo-cuda-algos/tests/roundtrip.rs:62-67"},
            {"graph": "K5 oriented", "value": 10, "source": "crates/grafeo-cuda-algos/tests/roundtrip.rs:228-236"},
        ],
        "bfs": [
            {"graph": "K4", "source": 0, "distances": [0, 1, 1, 1], "reachable": 4, "max_depth": 1,
             "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:71-82"},
            {"graph": "path5", "source": 0, "distances": [0, 1, 2, 3, 4], "reachable": 5, "max_depth": 4,
             "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:86-96"},
            {"graph": "path6", "source": 0, "reachable": 6, "max_depth": 5,
             "ref": "crates/grafeo-cuda-algos/tests/correctness.rs:356-363"},
            {"graph": "edgeless3", "source": 1, "distances": [-1, 0, -1], "reachable": 1, "max_depth": 0,
             "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:170-172"},
        ],
        "pagerank": [
            {"graph": "K4", "damping": 0.85, "max_iterations": 100, "tolerance": 1e-6, "value": 0.25,
             "abs_tol": 0.01, "converged": True, "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:100-114"},
            {"graph": "edgeless3", "damping": 0.85, "max_iterations": 50, "tolerance": 1e-7, "value": 1.0 / 3.0,
             "abs_tol": 1e-5, "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:175-178"},
            {"graph": "empty", "damping": 0.85, "max_iterations": 20, "tolerance": 1e-6, "ranks": [],
             "converged": True, "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:138-140"},
        ],
        "pagerank_vs_cpu": {"gpu": [0.85, 1000, 1e-7], "cpu": [0.85, 1000, 1e-12], "per_node_abs": 1e-4,
                            "sum_abs": 1e-3, "ref": "crates/grafeo-cuda-algos/tests/correctness.rs:286-303"},
        "k_truss": [
            {"graph": "K5", "k": 5, "edges": 10, "ref": "crates/grafeo-cuda-algos/tests/correctness.rs:377-386"},
            {"graph": "K5", "k": 6, "edges": 0, "ref": "crates/grafeo-cuda-algos/tests/correctness.rs:377-386"},
            {"graph": "empty", "k": 3, "edges": 0, "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:142-144"},
            {"graph": "edgeless4", "k": 3, "edges": 0, "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:165-168"},
        ],
        "errors": [
            {"call": "bfs", "graph": "empty", "arg": 0, "kind": "Kernel",
             "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:145"},
            {"call": "bfs", "graph": "K4", "arg": 4, "kind": "Kernel",
             "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:267"},
            {"call": "k_truss", "graph": "K4", "arg": 2, "kind": "Kernel",
             "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:268-271"},
        ],
        "invalid_csr": [
            {"offsets": [], "targets": [], "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:247"},
            {"offsets": [0, 5], "targets": [1], "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:248"},
            {"offsets": [0, 1, 2], "targets": [7, 0], "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:249"},
            {"offsets": [0, 2, 1, 2], "targets": [1, 2], "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:250"},
            {"offsets": [0, 2, 2], "targets": [1, 0], "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:251"},
        ],
        "validate_messages": [
            {"offsets": [], "targets": [], "contains": "empty"},
            {"offsets": [1, 1], "targets": [0], "contains": "offsets[0]"},
            {"offsets": [0, 2], "targets": [1], "contains": "offsets[1] is 2"},
            {"offsets": [0, 2, 1, 2], "targets": [1, 2], "contains": "decrease"},
            {"offsets": [0, 1, 1], "targets": [2], "contains": "only 2 nodes"},
            {"offsets": [0, 2, 2], "targets": [1, 0], "contains": "not strictly increasing"},
            {"offsets": [0, 2, 2], "targets": [1, 1], "contains": "not strictly increasing"},
        ],
        "validate_messages_ref": "crates/grafeo-cuda-core/tests/csr_export.rs:533-551",
        "validate_accepts": [
            {"offsets": [0], "targets": []},
            {"offsets": [0, 0, 0], "targets": []},
            {"offsets": [0, 3, 6, 9, 12], "targets": [1, 2, 3, 0, 2, 3, 0, 1, 3, 0, 1, 2]},
            {"offsets": [0, 2, 3], "targets": [0, 1, 0]},
        ],
        "validate_accepts_ref": "crates/grafeo-cuda-core/tests/csr_export.rs:533-540",
        "builders": [
            {"call": "from_edge_pairs", "edges": [[0, 1]], "num_nodes": 4, "symmetric": True,
             "offsets": [0, 1, 2, 2, 2], "targets": [1, 0],
             "ref": "crates/grafeo-cuda-core/tests/csr_export.rs:463-467"},
            {"call": "from_edge_pairs", "edges": [], "num_nodes": 0, "symmetric": True, "offsets": [0],
             "targets": [], "ref": "crates/grafeo-cuda-core/tests/csr_export.rs:469-474"},
            {"call": "from_edge_pairs_oriented", "edges": [], "num_nodes": 0, "offsets": [0], "targets": [],
             "ref": "crates/grafeo-cuda-core/tests/csr_export.rs:469-474"},
            {"call": "from_edge_pairs_oriented", "edges": [[2, 2]], "num_nodes": 3, "offsets": [0, 0, 0, 0],
             "targets": [], "ref": "crates/grafeo-cuda-core/tests/csr_export.rs:469-474"},
        ],
        "tsv": [
            {"text": "# comment\n% matrix-market style comment\n\n19\t88\t1.0\n88 3\nnot numbers\n19\n3\t19\n",
             "edges": [[0, 1], [1, 2], [2, 0]], "num_nodes": 3,
             "ref": "crates/grafeo-cuda-core/tests/csr_export.rs:495-505"},
            {"text": "18446744073709551615 0\n", "edges": [[0, 1]], "num_nodes": 2,
             "ref": "crates/grafeo-cuda-core/tests/csr_export.rs:507-516"},
            {"text": "# nothing here\n", "edges": [], "num_nodes": 0,
             "ref": "crates/grafeo-cuda-core/tests/csr_export.rs:507-516"},
        ],
        "wide_frontier": {"width": 500000, "depth": 4, "repeats": 5, "max_depth": 5,
                          "ref": "crates/grafeo-cuda-algos/tests/roundtrip.rs:186-222"},
    }


def directed_csr(n: int, edges) -> tuple[list[int], list[int]]:
    adj = [set() for _ in range(n)]
    for a, b in edges:
        adj[a].add(b)
    offsets, targets = [0], []
    for v in range(n):
        targets.extend(sorted(adj[v]))
        offsets.append(len(targets))
    return offsets, targets


def pagerank_variants() -> list[dict]:
    """Directed PageRank (out-edges = CSR lists) and personalised PageRank,
    networkx fixed points (tol 1e-13; dangling mass follows the teleport)."""
    import random

    out = []
    rnd = random.Random(77)
    cases = []
    for i in range(12):
        n = rnd.randint(2, 14)
        m = rnd.randint(0, 4 * n)
        cases.append((f"directed {i}", n, [(rnd.randrange(n), rnd.randrange(n)) for _ in range(m)]))
    cases.append(("directed chain with a sink", 5, [(0, 1), (1, 2), (2, 3), (3, 4)]))
    cases.append(("directed star out", 6, [(0, v) for v in range(1, 6)]))
    for name, n, edges in cases:
        dg = nx.DiGraph()
        dg.add_nodes_from(range(n))
        dg.add_edges_from(edges)
        offsets, targets = directed_csr(n, edges)
        pr = nx.pagerank(dg, alpha=0.85, tol=1e-13, max_iter=100000)
        seeds = sorted({rnd.randrange(n) for _ in range(2)})
        pers = {v: (1.0 / len(seeds) if v in seeds else 0.0) for v in range(n)}
        ppr = nx.pagerank(dg, alpha=0.85, personalization=pers, tol=1e-13, max_iter=100000)
        out.append({"name": name, "num_nodes": n, "directed": True, "offsets": offsets, "targets": targets,
                    "pagerank": [pr[v] for v in range(n)], "seeds": seeds, "ppr": [ppr[v] for v in range(n)]})
    for name, n, edges in graphs.catalog()[2:9]:
        g = nx.Graph()
        g.add_nodes_from(range(n))
        g.add_edges_from(edges)
        offsets, targets = symmetric_csr(n, edges)
        seeds = [0, n - 1]
        pers = {v: (0.5 if v in seeds else 0.0) for v in range(n)}
        ppr = nx.pagerank(g, alpha=0.85, personalization=pers, tol=1e-13, max_iter=100000)
        out.append({"name": name, "num_nodes": n, "directed": False, "offsets": offsets, "targets": targets,
                    "seeds": seeds, "ppr": [ppr[v] for v in range(n)]})
    return out


def main() -> None:
    with open(os.path.join(HERE, "pagerank_variants.json"), "w") as f:
        json.dump({"generator": "networkx " + nx.__version__, "graphs": pagerank_variants()}, f,
                  separators=(",", ":"))
    recs = [record(name, n, e) for name, n, e in graphs.catalog()]
    n, e = graphs.messy(True, True)
    recs.append(record("messy", n, e))
    n, e = graphs.messy(True, False)
    recs.append(record("messy without parallel edges", n, e))
    for i, (n, e) in enumerate(graphs.random_graphs()):
        recs.append(record(f"random {i}", n, e))
    with open(os.path.join(HERE, "catalog.json"), "w") as f:
        json.dump({"generator": "networkx " + nx.__version__, "graphs": recs}, f, separators=(",", ":"))
    with open(os.path.join(HERE, "reference_pins.json"), "w") as f:
        json.dump(pins(), f, indent=1)
    print(f"wrote {len(recs)} graphs")


if __name__ == "__main__":
    main()
