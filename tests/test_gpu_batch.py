"""GPU parity of the batched form (many graphs packed into one CSR).

Per graph, the batched triangle counts and BFS (S sources at once) are
bit-exact with the oracle, and the batched personalised PageRank is within
L1 1e-6 of the FP64 oracle run for the same number of iterations, on batches
built from the catalog / random graphs and on a generated R-MAT /
Watts-Strogatz batch; the captured CUDA-graph replay reproduces the direct
calls; the per-graph plain calls on `member(i)` agree.
"""
from __future__ import annotations

import numpy as np
import pytest

import grafeo_cuda as G
from grafeo_cuda import GrafeoCudaError
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PPR_L1 = 1e-6


def check_batch(device, b, csrs, S=16, K=8, seed=0):
    rng = np.random.default_rng(seed)
    sizes = [len(o) - 1 for o, _ in csrs]
    sources = np.array([rng.integers(0, max(n, 1), size=S) for n in sizes], dtype=np.uint32)
    seeds = np.array([rng.integers(0, max(n, 1), size=K) for n in sizes], dtype=np.uint32)
    tri = b.triangle_count()["total_triangles"]
    b.set_bfs_sources(sources)
    bfs = b.bfs()
    b.set_pagerank_seeds(seeds, 0.85, 100, 1e-6)
    ppr = b.personalized_pagerank()
    vb = b.vertex_base
    for g, (o, t) in enumerate(csrs):
        n = sizes[g]
        assert int(tri[g]) == O.triangle_count(o, t), g
        for k in range(S):
            ref = O.bfs(o, t, int(sources[g, k]))
            assert np.array_equal(bfs["distances"][k, vb[g]:vb[g + 1]], ref["distances"]), (g, k)
            assert bfs["reachable"][g, k] == ref["reachable"] and bfs["max_depth"][g, k] == ref["max_depth"], (g, k)
        it = int(ppr["iterations"][g])
        ref = O.pagerank(o, t, 0.85, it, 0.0, tele=O.seed_vector(n, seeds[g]))
        err = np.abs(ppr["ranks"][vb[g]:vb[g + 1]].astype(np.float64) - ref["ranks"]).sum()
        assert err <= PPR_L1, (g, err)
        assert ppr["converged"][g] == (it < 100 or bool(ppr["converged"][g]))
    return sources, seeds, tri, bfs, ppr


def test_batch_of_catalog_and_random_graphs(device, golden_graphs):
    csrs = [(np.asarray(g["offsets"], np.uint32), np.asarray(g["targets"], np.uint32))
            for g in golden_graphs if len(g["offsets"]) > 1]
    for scale, seed in ((9, 1), (11, 2)):
        c = G.generate_rmat(scale, 16, seed=seed)
        csrs.append((c.offsets, c.targets))
    b = G.GpuBatch.from_graphs(csrs, device)
    assert b.num_graphs == len(csrs)
    check_batch(device, b, csrs, S=5, K=3)


def test_generated_batch_members_and_replay(device):
    b = G.GpuBatch.generate(device, 24, seed=4)
    csr = b.to_csr()
    vb = b.vertex_base
    csrs = []
    for g in range(b.num_graphs):
        o = csr.offsets[vb[g]:vb[g + 1] + 1] - csr.offsets[vb[g]]
        t = csr.targets[csr.offsets[vb[g]]:csr.offsets[vb[g + 1]]] - vb[g]
        m = b.member(g).to_csr()
        assert np.array_equal(m.offsets, o) and np.array_equal(m.targets, t), g
        csrs.append((o, t))
    sources, seeds, tri, bfs, ppr = check_batch(device, b, csrs)
    b.capture()
    for _ in range(2):
        b.replay()
        r = b.results()
        assert np.array_equal(r["total_triangles"], tri)
        assert np.array_equal(r["distances"], bfs["distances"])
        assert np.array_equal(r["reachable"], bfs["reachable"]) and np.array_equal(r["max_depth"], bfs["max_depth"])
        assert np.array_equal(r["iterations"], ppr["iterations"])
        assert np.abs(r["ranks"] - ppr["ranks"]).max() <= 1e-6
    tuning = b.tuning()
    assert tuning["bfs_threads"]["chosen"] in (256, 512, 1024)
    # The per-graph plain calls agree.
    for g in (0, 5, 23):
        m = b.member(g)
        assert m.triangle_count()["total_triangles"] == int(tri[g])
        assert np.array_equal(m.bfs_array(int(sources[g, 0]))["distances"], bfs["distances"][0, vb[g]:vb[g + 1]])
        p = m.personalized_pagerank(seeds[g], 0.85, 100, 1e-6)
        assert np.abs(p["ranks"] - ppr["ranks"][vb[g]:vb[g + 1]]).sum() <= 2 * PPR_L1


def test_batch_errors(device):
    with pytest.raises(GrafeoCudaError) as e:  # edge 1 -> 2 crosses from graph 0 into graph 1
        G.GpuBatch.from_csr([0, 2, 3], [0, 1, 2, 3], [1, 2, 1], device)
    assert "leaves its graph" in str(e.value)
    with pytest.raises(GrafeoCudaError) as e:
        G.GpuBatch.from_csr([0, 1, 2], [0, 2, 1], [1], device)  # offsets decrease: invalid CSR first
    assert e.value.status == G.ERR_INVALID_CSR
    b = G.GpuBatch.from_graphs([([0, 1, 2], [1, 0]), ([0, 0], [])], device)
    with pytest.raises(GrafeoCudaError):
        b.set_bfs_sources([[0], [1]])  # graph 1 has one node
    with pytest.raises(GrafeoCudaError):
        b.capture()  # nothing set yet
    b.set_bfs_sources([[0], [0]])
    r = b.bfs()
    assert r["reachable"].tolist() == [[2], [1]] and r["max_depth"].tolist() == [[1], [0]]


def test_new_sources_drop_the_capture(device):
    """A capture reads the source, seed and result buffers by address:
    setting new sources or seeds drops it, replay refuses until the next
    capture, and the recaptured replay gives oracle-correct results for the
    new sources (here with a different S, so the buffers change size)."""
    b = G.GpuBatch.generate(device, 6, seed=9)
    csr = b.to_csr()
    vb = b.vertex_base
    csrs = []
    for g in range(b.num_graphs):
        csrs.append((csr.offsets[vb[g]:vb[g + 1] + 1] - csr.offsets[vb[g]],
                     csr.targets[csr.offsets[vb[g]]:csr.offsets[vb[g + 1]]] - vb[g]))
    rng = np.random.default_rng(3)
    n = [vb[g + 1] - vb[g] for g in range(b.num_graphs)]
    b.set_bfs_sources(np.array([rng.integers(0, x, 4) for x in n], dtype=np.uint32))
    b.set_pagerank_seeds(np.array([rng.integers(0, x, 2) for x in n], dtype=np.uint32))
    b.capture()
    b.replay()
    b.results()
    src = np.array([rng.integers(0, x, 9) for x in n], dtype=np.uint32)
    b.set_bfs_sources(src)
    with pytest.raises(GrafeoCudaError) as e:
        b.replay()
    assert "no captured graph" in str(e.value)
    seeds = np.array([rng.integers(0, x, 5) for x in n], dtype=np.uint32)
    b.capture()
    b.set_pagerank_seeds(seeds)
    with pytest.raises(GrafeoCudaError):
        b.replay()
    b.capture()
    b.replay()
    r = b.results()
    for g, (o, t) in enumerate(csrs):
        for k in range(9):
            ref = O.bfs(o, t, int(src[g, k]))
            assert np.array_equal(r["distances"][k, vb[g]:vb[g + 1]], ref["distances"]), (g, k)
        ref = O.pagerank(o, t, 0.85, int(r["iterations"][g]), 0.0, tele=O.seed_vector(len(o) - 1, seeds[g]))
        assert np.abs(r["ranks"][vb[g]:vb[g + 1]].astype(np.float64) - ref["ranks"]).sum() <= PPR_L1
