"""GPU parity for the PageRank extensions: directed PageRank (pull over a
device-built transpose) and personalised PageRank.

The reference has neither (its PageRank pulls over the CSR lists, right only
for symmetric graphs, pagerank.rs:10); the large-graph config asks for a
directed copy of R-MAT with 3% of the vertices left without out-edges, and
the batched config for personalised PageRank from seed vertices. Tolerances:
per node < 1e-4 and sum within 1e-3 of 1 against networkx's fixed point (the
reference's CPU comparison, correctness.rs:286-303), and L1 <= 1e-6 against
the FP64 oracle run for the same number of iterations.
"""
from __future__ import annotations

import numpy as np
import pytest

import grafeo_cuda as G
from grafeo_cuda import GrafeoCudaError
from oracle import oracle as O

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6


def upload(device, offsets, targets):
    return G.GpuGraph.from_csr(np.asarray(offsets, dtype=np.uint32), np.asarray(targets, dtype=np.uint32), device)


def test_variants_match_networkx_and_oracle(device, pagerank_variants):
    for g in pagerank_variants:
        o, t = np.asarray(g["offsets"], dtype=np.uint32), np.asarray(g["targets"], dtype=np.uint32)
        n = g["num_nodes"]
        gg = upload(device, o, t)
        tele = O.seed_vector(n, g["seeds"])
        if g["directed"]:
            r = gg.pagerank_directed(0.85, 1000, 1e-7)
            assert np.all(np.abs(r["ranks"] - np.asarray(g["pagerank"])) < 1e-4), g["name"]
            assert abs(float(r["ranks"].astype(np.float64).sum()) - 1.0) < 1e-3
            ref = O.pagerank_directed(o, t, 0.85, r["iterations"], 0.0)
            assert np.abs(r["ranks"] - ref["ranks"]).sum() <= L1_TOL, g["name"]
        r = gg.personalized_pagerank(g["seeds"], 0.85, 1000, 1e-7, directed=g["directed"])
        assert np.all(np.abs(r["ranks"] - np.asarray(g["ppr"])) < 1e-4), g["name"]
        assert abs(float(r["ranks"].astype(np.float64).sum()) - 1.0) < 1e-3
        if g["directed"]:
            ref = O.pagerank_directed(o, t, 0.85, r["iterations"], 0.0, tele=tele)
        else:
            ref = O.pagerank(o, t, 0.85, r["iterations"], 0.0, tele=tele)
        assert np.abs(r["ranks"] - ref["ranks"]).sum() <= L1_TOL, g["name"]


def dangling_copy(csr, fraction: float, seed: int):
    """Directed copy of a symmetric CSR with `fraction` of the vertices' out-edges removed."""
    rng = np.random.default_rng(seed)
    n = csr.num_nodes
    dangling = rng.choice(n, size=int(round(fraction * n)), replace=False)
    keep = np.ones(n, dtype=bool)
    keep[dangling] = False
    src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(csr.offsets))
    mask = keep[src]
    pairs = np.stack([src[mask], csr.targets[mask]], axis=1)
    return G.from_edge_pairs(pairs, n, False)


def test_directed_rmat_with_dangling_vertices_matches_fp64_oracle(device):
    """The large-graph config in miniature: R-MAT with 3% of the vertices'
    out-edges removed, up to 100 iterations at tol 1e-7; L1 and Linf error."""
    base = G.generate_rmat(16, 16, 0.57, 0.19, 0.19, seed=5)
    d = dangling_copy(base, 0.03, 5)
    g = G.GpuGraph.from_csr_arrays(d, device)
    r = g.pagerank_directed(0.85, 100, 1e-7)
    ref = O.pagerank_directed(d.offsets, d.targets, 0.85, r["iterations"], 0.0)
    err = np.abs(r["ranks"].astype(np.float64) - ref["ranks"])
    assert err.sum() <= L1_TOL, err.sum()
    assert err.max() <= 1e-7
    assert abs(float(r["ranks"].astype(np.float64).sum()) - 1.0) < 1e-5
    # Same stopping decision as the FP64 oracle with the reference's L1 rule.
    ref_full = O.pagerank_directed(d.offsets, d.targets, 0.85, 100, 1e-7)
    assert abs(r["iterations"] - ref_full["iterations"]) <= 1


def test_symmetric_graph_directed_pagerank_equals_pagerank(device):
    """On a symmetric CSR the transpose is the graph itself."""
    csr = G.generate_rmat(12, 16, 0.57, 0.19, 0.19, seed=3)
    g = G.GpuGraph.from_csr_arrays(csr, device)
    a = g.pagerank_array(0.85, 30, 0.0)
    b = g.pagerank_directed(0.85, 30, 0.0)
    assert np.abs(a["ranks"] - b["ranks"]).sum() <= 1e-6


def test_personalized_pagerank_on_rmat(device):
    csr = G.generate_rmat(14, 16, 0.57, 0.19, 0.19, seed=1)
    g = G.GpuGraph.from_csr_arrays(csr, device)
    seeds = [3, 17, 17, 1000, 4095, 8191, 12000, 16383]
    r = g.personalized_pagerank(seeds, 0.85, 100, 1e-6)
    ref = O.pagerank(csr.offsets, csr.targets, 0.85, r["iterations"], 0.0, tele=O.seed_vector(csr.num_nodes, seeds))
    assert np.abs(r["ranks"] - ref["ranks"]).sum() <= L1_TOL
    assert r["converged"]


def test_personalized_pagerank_argument_errors(device):
    g = upload(device, [0, 1, 2], [1, 0])
    with pytest.raises(GrafeoCudaError) as e:
        g.personalized_pagerank([])
    assert e.value.status == G.ERR_KERNEL
    with pytest.raises(GrafeoCudaError) as e:
        g.personalized_pagerank([2])
    assert e.value.status == G.ERR_KERNEL and "out of range" in str(e.value)


def test_gather_probe_times_the_plan_and_leaves_results_alone(device):
    """The diagnostic gather probe runs over the PageRank plan (built on
    demand, directed or not), returns a positive device time, and later
    PageRank calls give the same ranks bit for bit."""
    g = G.GpuGraph.generate_rmat(device, 14, 16, 0.57, 0.19, 0.19, seed=1)
    before = g.pagerank_array(0.85, 30, 0.0)["ranks"]
    ms = g.pagerank_gather_probe(False, 5)
    assert np.isfinite(ms) and ms > 0
    assert np.array_equal(g.pagerank_array(0.85, 30, 0.0)["ranks"], before)
    directed_before = g.pagerank_directed(0.85, 30, 0.0)["ranks"]
    assert g.pagerank_gather_probe(True, 3) > 0
    assert np.array_equal(g.pagerank_directed(0.85, 30, 0.0)["ranks"], directed_before)
    assert g.pagerank_gather_probe(False, 0) == 0.0
