"""Pins the oracle before anything is compared with it (CPU only).

The oracle (oracle/oracle.c) must reproduce the literal answers written in
the reference's tests and networkx's results on the reference's catalog, the
messy export case and the property-test graphs (tests/golden/).
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O

import graphs


def csr(g):
    return np.asarray(g["offsets"], dtype=np.uint32), np.asarray(g["targets"], dtype=np.uint32)


def test_oracle_triangles_match_networkx(golden_graphs):
    for g in golden_graphs:
        o, t = csr(g)
        assert O.triangle_count(o, t) == g["triangles"], g["name"]
        # Same graph through the degree-oriented builder (correctness.rs:240-257).
        pairs = [(u, v) for u in range(g["num_nodes"]) for v in t[o[u]:o[u + 1]] if v > u]
        oo, ot = O.from_edge_pairs_oriented(pairs, g["num_nodes"])
        assert O.triangle_count_oriented(oo, ot) == g["triangles"], g["name"]


def test_oracle_bfs_matches_networkx_from_every_source(golden_graphs):
    for g in golden_graphs:
        o, t = csr(g)
        for rec in g["bfs"]:
            r = O.bfs(o, t, rec["source"])
            assert r["distances"].tolist() == rec["distances"], (g["name"], rec["source"])
            assert r["reachable"] == rec["reachable"]
            assert r["max_depth"] == rec["max_depth"]


def test_oracle_pagerank_matches_networkx_fixed_point(golden_graphs):
    for g in golden_graphs:
        if g["num_nodes"] == 0:
            continue
        o, t = csr(g)
        r = O.pagerank(o, t, 0.85, 100000, 1e-15, rule="max")
        assert r["converged"], g["name"]
        np.testing.assert_allclose(r["ranks"], g["pagerank"], atol=1e-10, rtol=0, err_msg=g["name"])
        assert abs(r["ranks"].sum() - 1.0) < 1e-12


def test_oracle_k_truss_matches_networkx(golden_graphs):
    for g in golden_graphs:
        o, t = csr(g)
        for k in range(3, 9):
            r = O.k_truss(o, t, k)
            got = sorted(map(tuple, r["edges"].tolist()))
            assert len(set(got)) == len(got), (g["name"], k)
            assert got == [tuple(e) for e in g["k_truss"][str(k)]], (g["name"], k)


def test_oracle_reproduces_reference_literal_answers(pins):
    k4o, k4t = graphs.K4_CSR
    p5o, p5t = graphs.PATH5_CSR
    lookup = {"K4": (k4o, k4t), "path5": (p5o, p5t)}
    k5o, k5t = O.from_edge_pairs(graphs.complete_edges(5), 5, True)
    lookup["K5"] = (k5o, k5t)
    for pin in pins["triangles"]:
        if pin["graph"] == "K5 oriented":
            oo, ot = O.from_edge_pairs_oriented(graphs.complete_edges(5), 5)
            assert O.triangle_count_oriented(oo, ot) == pin["value"]
        else:
            assert O.triangle_count(*lookup[pin["graph"]]) == pin["value"], pin
    p6 = O.from_edge_pairs(graphs.path_edges(6), 6, True)
    lookup["path6"] = p6
    lookup["edgeless3"] = ([0, 0, 0, 0], [])
    for pin in pins["bfs"]:
        r = O.bfs(*lookup[pin["graph"]], pin["source"])
        if "distances" in pin:
            assert r["distances"].tolist() == pin["distances"]
        assert r["reachable"] == pin["reachable"] and r["max_depth"] == pin["max_depth"], pin
    lookup["empty"] = ([0], [])
    for pin in pins["pagerank"]:
        r = O.pagerank(*lookup[pin["graph"]], pin["damping"], pin["max_iterations"], pin["tolerance"])
        if "value" in pin:
            assert np.all(np.abs(r["ranks"] - pin["value"]) < pin["abs_tol"]), pin
        if "ranks" in pin:
            assert r["ranks"].tolist() == pin["ranks"]
        if "converged" in pin:
            assert r["converged"] == pin["converged"]
    lookup["edgeless4"] = ([0, 0, 0, 0, 0], [])
    for pin in pins["k_truss"]:
        assert len(O.k_truss(*lookup[pin["graph"]], pin["k"])["edges"]) == pin["edges"], pin


def test_oracle_builders_match_reference_examples(pins):
    for b in pins["builders"]:
        if b["call"] == "from_edge_pairs":
            o, t = O.from_edge_pairs(b["edges"], b["num_nodes"], b["symmetric"])
        else:
            o, t = O.from_edge_pairs_oriented(b["edges"], b["num_nodes"])
        assert o.tolist() == b["offsets"] and t.tolist() == b["targets"], b


@pytest.mark.parametrize("seed", range(8))
def test_oracle_oriented_builder_rules(seed):
    """csr_export.rs(tests):402-458: each edge once, lower (degree, id) -> higher,
    and the oriented count equals a brute-force triangle count."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 14))
    raw = rng.integers(0, n, size=(int(rng.integers(0, 60)), 2))
    o, t = O.from_edge_pairs_oriented(raw, n)
    und = {(min(a, b), max(a, b)) for a, b in raw.tolist() if a != b}
    assert len(t) == len(und)
    deg = np.zeros(n, dtype=int)
    for a, b in und:
        deg[a] += 1
        deg[b] += 1
    seen = set()
    for u in range(n):
        for v in t[o[u]:o[u + 1]].tolist():
            assert deg[u] < deg[v] or (deg[u] == deg[v] and u < v)
            assert (min(u, v), max(u, v)) not in seen
            seen.add((min(u, v), max(u, v)))
    assert seen == und
    brute = sum(
        1
        for a in range(n)
        for b in range(a + 1, n)
        for c in range(b + 1, n)
        if (a, b) in und and (b, c) in und and (a, c) in und
    )
    assert O.triangle_count_oriented(o, t) == brute


def test_oracle_directed_and_personalized_pagerank_match_networkx(pagerank_variants):
    for g in pagerank_variants:
        o, t = csr(g)
        n = g["num_nodes"]
        tele = O.seed_vector(n, g["seeds"])
        if g["directed"]:
            r = O.pagerank_directed(o, t, 0.85, 100000, 1e-15, rule="max")
            assert r["converged"]
            np.testing.assert_allclose(r["ranks"], g["pagerank"], atol=1e-10, rtol=0, err_msg=g["name"])
            r = O.pagerank_directed(o, t, 0.85, 100000, 1e-15, rule="max", tele=tele)
        else:
            r = O.pagerank(o, t, 0.85, 100000, 1e-15, rule="max", tele=tele)
        assert r["converged"]
        np.testing.assert_allclose(r["ranks"], g["ppr"], atol=1e-10, rtol=0, err_msg=g["name"])
        assert abs(r["ranks"].sum() - 1.0) < 1e-12


def test_oracle_truss_decomposition_matches_networkx_trusses(golden_graphs):
    for g in golden_graphs:
        o, t = csr(g)
        r = O.truss_decomposition(o, t)
        src = np.repeat(np.arange(g["num_nodes"]), np.diff(o))
        upper = [(int(a), int(b), int(x)) for a, b, x in zip(src, t, r["trussness"]) if a < b]
        for k in range(3, 9):
            got = sorted((a, b) for a, b, x in upper if x >= k)
            assert got == [tuple(e) for e in g["k_truss"][str(k)]], (g["name"], k)
        assert all(x == 0 for a, b, x in zip(src, t, r["trussness"]) if a == b)


def test_oracle_transpose():
    o, t = O.transpose([0, 2, 3, 3, 4], [1, 3, 2, 0])
    assert o.tolist() == [0, 1, 2, 3, 4] and t.tolist() == [3, 0, 1, 0]


def test_schedule_oracle_gradient_matches_central_differences():
    """The FP64 schedule-network oracle's analytic gradient (against which the
    GPU gradient kernel is checked) equals central differences of its loss."""
    from oracle import schedule_mlp as M

    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, M.PARAMS)
    x = rng.uniform(-1, 2, (50, 12))
    y = rng.normal(3, 2, (50, 3))
    m = rng.random((50, 3)) < 0.7
    _, g = M.loss_and_grad(p, x, y, m)
    h = 1e-6
    for i in rng.choice(M.PARAMS, 60, replace=False):
        e = np.zeros(M.PARAMS)
        e[i] = h
        num = (M.loss_and_grad(p + e, x, y, m)[0] - M.loss_and_grad(p - e, x, y, m)[0]) / (2 * h)
        assert abs(num - g[i]) <= 1e-6 * max(1.0, abs(g[i]))
    # BF16 rounding is round-to-nearest-even.
    assert M.bf16_bits(np.array([1.0, 1.00390625, 1.005859375, -2.5], np.float32)).tolist() == [
        0x3F80, 0x3F80, 0x3F81, 0xC020]


def test_oracle_k_truss_round_semantics_on_self_loops():
    """A self-loop inflates first-round support (the reference merges raw lists,
    kernels/k_truss.cu:59-92); the fixpoint is still the maximal k-truss."""
    # Triangle 0-1-2 plus a pendant edge 2-3 with a self-loop at 3 and at 2.
    o, t = O.from_edge_pairs([(0, 1), (1, 2), (0, 2), (2, 3), (3, 3), (2, 2)], 4, True)
    r = O.k_truss(o, t, 3)
    assert sorted(map(tuple, r["edges"].tolist())) == [(0, 1), (0, 2), (1, 2)]
    # Edge 2-3 is kept in round 1 (self-loops at 2 and 3 count as common
    # neighbours), loses the self-loops in round 1, and goes in round 2.
    assert r["iterations"] == 3


# ---------------------------------------------------------------- the oracle at scale (oracle_scale.c)


def _simple(g) -> bool:
    o, t = csr(g)
    src = np.repeat(np.arange(g["num_nodes"]), np.diff(o))
    return not np.any(src == t)


@pytest.mark.parametrize("scale,seed", [(1, 1), (6, 7), (11, 2), (14, 1)])
def test_oracle_rmat_generator_matches_library_and_numpy(scale, seed):
    """The oracle's radix-sort R-MAT builder equals the library's host
    generator (bucket sort) entry for entry, and the numpy restatement of the
    pair draws in tests/graphs.py."""
    import grafeo_cuda as G

    a = O.generate_rmat(scale, 16, 0.57, 0.19, 0.19, seed)
    b = G.generate_rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed)
    assert np.array_equal(a.offsets, b.offsets) and np.array_equal(a.targets, b.targets)
    if scale <= 11:
        s, d = graphs.rmat_pairs(scale, 16, 0.57, 0.19, 0.19, seed)
        o, t = O.from_edge_pairs(np.stack([s, d], axis=1)[s != d], 1 << scale, True)
        assert np.array_equal(a.offsets, o) and np.array_equal(a.targets, t)


@pytest.mark.parametrize("n,pairs,seed", [(0, 0, 1), (1, 5, 1), (1000, 16000, 3), (70000, 1 << 20, 3)])
def test_oracle_erdos_renyi_generator_matches_library(n, pairs, seed):
    import grafeo_cuda as G

    a = O.generate_erdos_renyi(n, pairs, seed)
    b = G.generate_erdos_renyi(n, pairs, seed=seed)
    assert np.array_equal(a.offsets, b.offsets) and np.array_equal(a.targets, b.targets)


def test_oracle_sorted_transpose_matches_serial_transpose():
    rng = np.random.default_rng(5)
    for n in (1, 7, 300, 5000):
        pairs = rng.integers(0, n, size=(4 * n, 2))
        o, t = O.from_edge_pairs(pairs, n, False)
        x, y = O.transpose(o, t), O.transpose_sorted(o, t)
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])
    c = O.generate_rmat(13, 16, 0.57, 0.19, 0.19, 4)
    x, y = O.transpose(c.offsets, c.targets), O.transpose_sorted(c.offsets, c.targets)
    assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])


def test_oracle_edge_support_counts_triangles(golden_graphs):
    for g in golden_graphs:
        if not _simple(g):
            continue
        o, t = csr(g)
        s = O.edge_support(o, t)
        assert int(s.sum()) == 6 * g["triangles"], g["name"]
    c = O.generate_rmat(14, 16, 0.57, 0.19, 0.19, 1)
    assert int(O.edge_support(c.offsets, c.targets).sum()) == 6 * O.triangle_count(c.offsets, c.targets)
    with pytest.raises(ValueError):
        O.edge_support([0, 1, 1], [1])  # not symmetric
    with pytest.raises(ValueError):
        O.edge_support([0, 1], [0])  # self-loop


def test_oracle_peeling_k_truss_matches_full_recomputation(golden_graphs):
    """The incremental peel gives orc_k_truss's edges and round counts (the
    reference's round rule) on the catalog, the property-test graphs without
    self-loops and random R-MAT / Erdos-Renyi graphs."""
    cases = [csr(g) for g in golden_graphs if _simple(g)]
    for scale, seed in ((9, 1), (11, 3), (12, 2)):
        c = O.generate_rmat(scale, 16, 0.57, 0.19, 0.19, seed)
        cases.append((c.offsets, c.targets))
    c = O.generate_erdos_renyi(3000, 3000 * 12, 9)
    cases.append((c.offsets, c.targets))
    for o, t in cases:
        sup = O.edge_support(o, t) if len(t) else None
        for k in (2, 3, 4, 5, 6, 8, 11):
            a, b = O.k_truss(o, t, k), O.k_truss_peel(o, t, k, sup)
            assert np.array_equal(a["edges"], b["edges"]), k
            assert a["iterations"] == b["iterations"], k


def test_oracle_peeling_decomposition_matches_definition_and_round_rule(golden_graphs):
    """Trussness from the peel equals the definition-based decomposition;
    rounds equal the host restatement of the device's level-by-level rule."""
    import random

    import test_peel_frontier as PF

    for g in golden_graphs:
        if not _simple(g):
            continue
        o, t = csr(g)
        a, b = O.truss_decomposition(o, t), O.truss_decomposition_peel(o, t)
        assert np.array_equal(a["trussness"], b["trussness"]) and a["max_trussness"] == b["max_trussness"], g["name"]
    rng = random.Random(11)
    for _ in range(60):
        n = rng.randint(2, 30)
        pairs = [(rng.randrange(n), rng.randrange(n)) for _ in range(rng.randint(0, n * 6))]
        pairs = [(x, y) for x, y in pairs if x != y]
        o, t = O.from_edge_pairs(pairs, n, True)
        rounds, top, truss = PF.decomposition(n, pairs, True)
        b = O.truss_decomposition_peel(o, t)
        assert b["rounds"] == rounds and b["max_trussness"] == top, pairs
        src = np.repeat(np.arange(n), np.diff(o))
        edges = sorted({(min(x, y), max(x, y)) for x, y in pairs})
        by_edge = dict(zip(edges, truss))
        assert [by_edge[(min(x, y), max(x, y))] for x, y in zip(src, t)] == b["trussness"].tolist(), pairs
    c = O.generate_rmat(12, 16, 0.57, 0.19, 0.19, 6)
    a, b = O.truss_decomposition(c.offsets, c.targets), O.truss_decomposition_peel(c.offsets, c.targets)
    assert np.array_equal(a["trussness"], b["trussness"]) and a["max_trussness"] == b["max_trussness"]
