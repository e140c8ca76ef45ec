"""GPU parity: the sm_100a paths against the oracle and the reference's pins.

Ports crates/grafeo-cuda-algos/tests/roundtrip.rs and correctness.rs: literal
known answers, the catalog from every BFS source, the messy export case, the
property-test graphs, the wide-frontier regression, invalid CSR and argument
errors. Beyond the reference: bit-exact comparisons with the oracle at
R-MAT/Erdos-Renyi sizes the oracle finishes in seconds, the exact k-truss
round count, and PageRank L1 error against the FP64 oracle.

Tolerances: triangle counts, BFS distances/reachable/max_depth and k-truss
edge lists are bit-exact. PageRank: per node < 1e-4 and sum within 1e-3 of 1
against the converged CPU result (correctness.rs:286-303), and L1 <= 1e-6
against the FP64 oracle run for the same number of iterations.
"""
from __future__ import annotations

import numpy as np
import pytest

import grafeo_cuda as G
from grafeo_cuda import GrafeoCudaError
from oracle import oracle as O

import graphs

pytestmark = pytest.mark.gpu

PR_L1_TOL = 1e-6


def upload(device, offsets, targets):
    return G.GpuGraph.from_csr(np.asarray(offsets, dtype=np.uint32), np.asarray(targets, dtype=np.uint32), device)


def edge_set(edges) -> list[tuple[int, int]]:
    return [tuple(map(int, e)) for e in np.asarray(edges).reshape(-1, 2).tolist()]


# ---------------------------------------------------------------- roundtrip.rs


def test_triangle_count_k4_and_path(device):
    assert upload(device, *graphs.K4_CSR).triangle_count()["total_triangles"] == 4
    assert upload(device, *graphs.PATH5_CSR).triangle_count()["total_triangles"] == 0


def test_bfs_k4_and_path(device):
    r = upload(device, *graphs.K4_CSR).bfs(0)
    assert (r["reachable"], r["max_depth"]) == (4, 1)
    assert r["distances"] == [0, 1, 1, 1]
    r = upload(device, *graphs.PATH5_CSR).bfs(0)
    assert (r["reachable"], r["max_depth"]) == (5, 4)
    assert r["distances"] == [0, 1, 2, 3, 4]


def test_pagerank_k4(device):
    r = upload(device, *graphs.K4_CSR).pagerank(0.85, 100, 1e-6)
    assert r["converged"]
    assert all(abs(x - 0.25) < 0.01 for x in r["ranks"])


def test_empty_graph(device):
    g = upload(device, [0], [])
    assert (g.num_nodes, g.num_edges) == (0, 0)
    assert g.triangle_count()["total_triangles"] == 0
    assert g.triangle_count_oriented()["total_triangles"] == 0
    r = g.pagerank(0.85, 20, 1e-6)
    assert r["ranks"] == [] and r["converged"]
    assert g.k_truss(3)["edges"] == []
    with pytest.raises(GrafeoCudaError) as e:
        g.bfs(0)
    assert e.value.status == G.ERR_KERNEL


def test_edgeless_graph(device):
    g = upload(device, [0, 0, 0, 0], [])
    assert g.triangle_count()["total_triangles"] == 0
    assert g.triangle_count_oriented()["total_triangles"] == 0
    assert g.k_truss(3)["edges"] == []
    r = g.bfs(1)
    assert r["distances"] == [-1, 0, -1] and (r["reachable"], r["max_depth"]) == (1, 0)
    r = g.pagerank(0.85, 50, 1e-7)
    assert all(abs(x - 1.0 / 3.0) < 1e-5 for x in r["ranks"])


def test_bfs_wide_frontier_after_first_level(device):
    n, pairs, expected = graphs.wide_frontier(500_000, 4)
    csr = G.from_edge_pairs(pairs, n, True)
    g = G.GpuGraph.from_csr_arrays(csr, device)
    for run in range(5):
        r = g.bfs_array(0)
        wrong = int(np.count_nonzero(r["distances"] != expected))
        assert wrong == 0, f"run {run}: {wrong} nodes have a wrong distance"
        assert r["reachable"] == n and r["max_depth"] == 5


def test_triangle_count_oriented_k5(device):
    csr = G.from_edge_pairs_oriented(graphs.complete_edges(5), 5)
    assert G.GpuGraph.from_csr_arrays(csr, device).triangle_count_oriented()["total_triangles"] == 10


def test_invalid_csr_is_rejected(device, pins):
    for case in pins["invalid_csr"]:
        with pytest.raises(GrafeoCudaError) as e:
            G.GpuGraph.from_csr(case["offsets"], case["targets"], device)
        assert e.value.status == G.ERR_INVALID_CSR, case


def test_invalid_csr_messages_match_host_validation(device):
    rng = np.random.default_rng(5)
    for _ in range(40):
        n = int(rng.integers(1, 12))
        deg = rng.integers(0, 5, size=n)
        offsets = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
        targets = rng.integers(0, n + 1, size=int(offsets[-1]))
        if rng.random() < 0.3 and n > 1:
            i = int(rng.integers(1, n))
            offsets[i] = offsets[i] + 1 if offsets[i] < offsets[-1] else offsets[i]
        try:
            G.validate_csr(offsets, targets)
            host = None
        except GrafeoCudaError as e:
            host = str(e)
        try:
            G.GpuGraph.from_csr(offsets, targets, device)
            dev = None
        except GrafeoCudaError as e:
            dev = str(e)
        assert host == dev, (offsets.tolist(), targets.tolist())


def test_chunked_upload_checks_every_chunk(device):
    """from_csr copies the targets in 16M-entry chunks and checks each chunk
    as it lands: a violation in the third chunk, at a chunk boundary, or in
    the first entry of a chunk is reported like the host validator does, and
    a valid graph of several chunks comes back entry for entry."""
    n, deg = 1 << 20, 40  # 41,943,040 entries: three chunks
    offsets = np.arange(n + 1, dtype=np.uint32) * deg
    base = (np.arange(n, dtype=np.uint64)[:, None] * 7 + np.arange(deg, dtype=np.uint64)[None, :] * 26_000)
    targets = (base % n).astype(np.uint32)
    targets.sort(axis=1)
    targets = np.ascontiguousarray(targets.reshape(-1))
    g = G.GpuGraph.from_csr(offsets, targets, device)
    back = g.to_csr()
    assert np.array_equal(back.offsets, offsets) and np.array_equal(back.targets, targets)
    del g
    chunk = 1 << 24
    for j in (36_000_000, chunk, 2 * chunk - 1, 2 * chunk):
        bad = targets.copy()
        row = j // deg
        bad[j] = bad[j - 1] if j % deg else n  # a repeat inside the list, or past the end at a list start
        with pytest.raises(GrafeoCudaError) as host:
            G.validate_csr(offsets, bad)
        with pytest.raises(GrafeoCudaError) as dev:
            G.GpuGraph.from_csr(offsets, bad, device)
        assert str(dev.value) == str(host.value), (j, row)


def test_argument_errors(device):
    g = upload(device, *graphs.K4_CSR)
    with pytest.raises(GrafeoCudaError) as e:
        g.bfs(4)
    assert e.value.status == G.ERR_KERNEL and "out of range" in str(e.value)
    with pytest.raises(GrafeoCudaError) as e:
        g.k_truss(2)
    assert e.value.status == G.ERR_KERNEL and "k must be >= 3" in str(e.value)


def test_device_properties(device):
    assert "B200" in device.name or device.name
    assert device.total_memory > 100 * 2**30
    assert device.sm_count >= 100


# ---------------------------------------------------------------- correctness.rs


def check_graph(device, g: dict, pr_vs_cpu: bool = True):
    offsets, targets = g["offsets"], g["targets"]
    gg = upload(device, offsets, targets)
    name = g["name"]
    # triangles, both paths
    assert gg.triangle_count()["total_triangles"] == g["triangles"], name
    n = g["num_nodes"]
    pairs = [(u, v) for u in range(n) for v in targets[offsets[u]:offsets[u + 1]] if v > u]
    oriented = G.GpuGraph.from_csr_arrays(G.from_edge_pairs_oriented(pairs, n), device)
    assert oriented.triangle_count_oriented()["total_triangles"] == g["triangles"], name
    # BFS from every source
    for rec in g["bfs"]:
        r = gg.bfs(rec["source"])
        assert r["distances"] == rec["distances"], (name, rec["source"])
        assert (r["reachable"], r["max_depth"]) == (rec["reachable"], rec["max_depth"]), (name, rec["source"])
    # PageRank against the converged CPU fixed point
    if pr_vs_cpu and n:
        r = gg.pagerank(0.85, 1000, 1e-7)
        assert len(r["ranks"]) == n
        ranks = np.asarray(r["ranks"], dtype=np.float64)
        assert np.all(np.abs(ranks - np.asarray(g["pagerank"])) < 1e-4), name
        assert abs(ranks.sum() - 1.0) < 1e-3, name
        ref = O.pagerank(offsets, targets, 0.85, r["iterations"], 0.0)
        assert np.abs(ranks - ref["ranks"]).sum() <= PR_L1_TOL, name
    # k-truss for k = 3..8, exact edges (CSR order) and exact round count
    for k in range(3, 9):
        r = gg.k_truss(k)
        ref = O.k_truss(offsets, targets, k)
        assert edge_set(r["edges"]) == edge_set(ref["edges"]), (name, k)
        assert sorted(edge_set(r["edges"])) == [tuple(e) for e in g["k_truss"][str(k)]], (name, k)
        assert r["iterations"] == ref["iterations"], (name, k)
        assert r["k"] == k


def test_catalog_matches_cpu(device, golden_graphs):
    for g in golden_graphs:
        if not g["name"].startswith("random") and not g["name"].startswith("messy"):
            check_graph(device, g)


def test_messy_graph_matches_cpu(device, golden_graphs):
    for g in golden_graphs:
        if g["name"].startswith("messy"):
            assert g["num_nodes"] == 6
            check_graph(device, g)


def test_random_graphs_match_cpu(device, golden_graphs):
    for g in golden_graphs:
        if g["name"].startswith("random"):
            check_graph(device, g)


# ---------------------------------------------------------------- beyond the reference


def directed_csr(rng, n, m):
    pairs = rng.integers(0, n, size=(m, 2))
    c = G.from_edge_pairs(pairs, n, False)
    return c.offsets, c.targets


def test_non_symmetric_csr_follows_reference_formulas(device):
    """A directed CSR: BFS follows the lists, TC uses the reference's v > u
    formula, k-truss keeps the reference's per-entry rules."""
    rng = np.random.default_rng(11)
    for _ in range(30):
        n = int(rng.integers(2, 40))
        o, t = directed_csr(rng, n, int(rng.integers(0, 6 * n)))
        g = upload(device, o, t)
        assert g.triangle_count()["total_triangles"] == O.triangle_count(o, t)
        assert g.triangle_count_oriented()["total_triangles"] == O.triangle_count_oriented(o, t)
        for s in range(0, n, max(1, n // 5)):
            r = g.bfs_array(s)
            ref = O.bfs(o, t, s)
            assert np.array_equal(r["distances"], ref["distances"])
            assert (r["reachable"], r["max_depth"]) == (ref["reachable"], ref["max_depth"])
        for k in (3, 4):
            r = g.k_truss_array(k)
            ref = O.k_truss(o, t, k)
            assert edge_set(r["edges"]) == edge_set(ref["edges"]) and r["iterations"] == ref["iterations"]


def test_k_truss_with_self_loops_matches_oracle(device):
    """Self-loops inflate first-round support in the reference (k_truss.cu:59-92);
    the incremental peel must reproduce the edges and the round count."""
    base = G.generate_rmat(12, 8, 0.57, 0.19, 0.19, seed=9)
    rng = np.random.default_rng(9)
    src = np.repeat(np.arange(base.num_nodes, dtype=np.uint32), np.diff(base.offsets))
    pairs = np.stack([src, base.targets], axis=1)
    loops = rng.choice(base.num_nodes, size=base.num_nodes // 10, replace=False).astype(np.uint32)
    pairs = np.concatenate([pairs, np.stack([loops, loops], axis=1)])
    csr = G.from_edge_pairs(pairs, base.num_nodes, True)
    g = G.GpuGraph.from_csr_arrays(csr, device)
    for k in (3, 4, 5, 7):
        r = g.k_truss_array(k)
        ref = O.k_truss(csr.offsets, csr.targets, k)
        assert np.array_equal(r["edges"], ref["edges"]), k
        assert r["iterations"] == ref["iterations"], k


def compare_with_oracle(device, csr, sources, pr_iterations, ks, label):
    o, t = csr.offsets, csr.targets
    g = G.GpuGraph.from_csr_arrays(csr, device)
    assert g.triangle_count()["total_triangles"] == O.triangle_count(o, t), label
    for s in sources:
        r = g.bfs_array(int(s))
        ref = O.bfs(o, t, int(s))
        assert np.array_equal(r["distances"], ref["distances"]), (label, s)
        assert (r["reachable"], r["max_depth"]) == (ref["reachable"], ref["max_depth"]), (label, s)
    r = g.pagerank_array(0.85, pr_iterations, 1e-30)
    ref = O.pagerank(o, t, 0.85, r["iterations"], 0.0)
    assert r["iterations"] == pr_iterations
    l1 = float(np.abs(r["ranks"].astype(np.float64) - ref["ranks"]).sum())
    assert l1 <= PR_L1_TOL, (label, l1)
    for k in ks:
        r = g.k_truss_array(k)
        ref = O.k_truss(o, t, k)
        assert np.array_equal(r["edges"], ref["edges"]), (label, k)
        assert r["iterations"] == ref["iterations"], (label, k)


def test_rmat_scale14_config(device):
    """The small config: R-MAT scale 14, seed 1; TC, BFS from 0, PR 20
    iterations at tol 1e-6, k-truss k = 4, all against the oracle."""
    csr = G.generate_rmat(14, 16, 0.57, 0.19, 0.19, seed=1)
    g = G.GpuGraph.from_csr_arrays(csr, device)
    o, t = csr.offsets, csr.targets
    assert g.triangle_count()["total_triangles"] == O.triangle_count(o, t)
    r = g.bfs_array(0)
    ref = O.bfs(o, t, 0)
    assert np.array_equal(r["distances"], ref["distances"])
    assert (r["reachable"], r["max_depth"]) == (ref["reachable"], ref["max_depth"])
    r = g.pagerank_array(0.85, 20, 1e-6)
    ref = O.pagerank(o, t, 0.85, 20, 1e-6)
    assert (r["iterations"], r["converged"]) == (ref["iterations"], ref["converged"])
    assert float(np.abs(r["ranks"] - ref["ranks"]).sum()) <= PR_L1_TOL
    r = g.k_truss_array(4)
    ref = O.k_truss(o, t, 4)
    assert np.array_equal(r["edges"], ref["edges"]) and r["iterations"] == ref["iterations"]


@pytest.mark.parametrize("scale,seed", [(12, 3), (16, 2)])
def test_rmat_matches_oracle(device, scale, seed):
    csr = G.generate_rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed)
    rng = np.random.default_rng(seed)
    deg = np.diff(csr.offsets)
    sources = rng.choice(np.flatnonzero(deg > 0), size=4, replace=False)
    compare_with_oracle(device, csr, [0, *sources], 50, (3, 5, 8) if scale <= 12 else (3, 6), f"rmat{scale}")


def test_erdos_renyi_matches_oracle(device):
    csr = G.generate_erdos_renyi(1 << 15, 16 << 15, seed=3)
    compare_with_oracle(device, csr, [0, 7, 12345], 50, (3, 4), "er15")


def test_bfs_and_pagerank_scale20_properties(device):
    """At a size where every oracle pass still takes seconds: BFS distances
    equal the oracle's from 3 sources; PageRank L1 against the FP64 oracle at
    50 iterations; ranks sum to 1."""
    csr = G.generate_rmat(20, 16, 0.57, 0.19, 0.19, seed=2)
    g = G.GpuGraph.from_csr_arrays(csr, device)
    o, t = csr.offsets, csr.targets
    for s in (0, 1, 977):
        r = g.bfs_array(s)
        ref = O.bfs(o, t, s)
        assert np.array_equal(r["distances"], ref["distances"])
        assert (r["reachable"], r["max_depth"]) == (ref["reachable"], ref["max_depth"])
    r = g.pagerank_array(0.85, 50, 1e-30)
    ref = O.pagerank(o, t, 0.85, 50, 0.0)
    l1 = float(np.abs(r["ranks"].astype(np.float64) - ref["ranks"]).sum())
    assert l1 <= PR_L1_TOL, l1
    assert abs(float(r["ranks"].astype(np.float64).sum()) - 1.0) < 1e-5
    assert g.triangle_count()["total_triangles"] == O.triangle_count(o, t)
