"""GPU parity for the device CSR builder and the device generators.

from_edge_pairs / from_edge_pairs_oriented on the device must give the CSR
(and the errors) of the host builders, which restate csr_export.rs:202-239 and
:299-350 and are pinned in test_oracle.py against the reference's examples.
The device generators must draw exactly the pairs of their restatements (the
host R-MAT / Erdos-Renyi generators, numpy for grid, Watts-Strogatz and
random geometric graphs).
"""
from __future__ import annotations

import numpy as np
import pytest

import grafeo_cuda as G
from grafeo_cuda import GrafeoCudaError
from oracle import oracle as O

import graphs

pytestmark = pytest.mark.gpu


def csr_equal(g, offsets, targets, label):
    c = g.to_csr()
    assert np.array_equal(c.offsets, np.asarray(offsets, dtype=np.uint32)), label
    assert np.array_equal(c.targets, np.asarray(targets, dtype=np.uint32)), label


def random_pairs(rng, n, m, loops=True):
    p = rng.integers(0, n, size=(m, 2)).astype(np.uint32)
    if not loops:
        p = p[p[:, 0] != p[:, 1]]
    return p


@pytest.mark.parametrize("seed", range(6))
def test_device_from_edge_pairs_matches_host_builders(device, seed):
    rng = np.random.default_rng(seed)
    for n, m in ((1, 0), (1, 3), (7, 30), (300, 5000), (5000, 200_000)):
        p = random_pairs(rng, n, m)
        for sym in (False, True):
            h = G.from_edge_pairs(p, n, sym)
            csr_equal(G.GpuGraph.from_edge_pairs(p, n, sym, device), h.offsets, h.targets, (n, m, sym))
        h = G.from_edge_pairs_oriented(p, n)
        g = G.GpuGraph.from_edge_pairs_oriented(p, n, device)
        csr_equal(g, h.offsets, h.targets, (n, m, "oriented"))
        assert g.triangle_count_oriented()["total_triangles"] == O.triangle_count_oriented(h.offsets, h.targets)


def test_device_from_edge_pairs_reference_examples_and_errors(device, pins):
    for b in pins["builders"]:
        if b["call"] == "from_edge_pairs":
            g = G.GpuGraph.from_edge_pairs(b["edges"], b["num_nodes"], b["symmetric"], device)
        else:
            g = G.GpuGraph.from_edge_pairs_oriented(b["edges"], b["num_nodes"], device)
        csr_equal(g, b["offsets"], b["targets"], b)
    g = G.GpuGraph.from_edge_pairs([], 0, True, device)
    assert g.num_nodes == 0 and g.num_edges == 0
    g = G.GpuGraph.from_edge_pairs([], 5, False, device)
    csr_equal(g, [0] * 6, [], "edgeless")
    # The first offending pair in input order is the one reported.
    bad = [(0, 1), (1, 9), (7, 0), (1, 2)]
    for sym in (True, False):
        with pytest.raises(GrafeoCudaError) as dev_err:
            G.GpuGraph.from_edge_pairs(bad, 5, sym, device) if sym else G.GpuGraph.from_edge_pairs(
                [(0, 1), (7, 0)], 5, False, device)
        with pytest.raises(GrafeoCudaError) as host_err:
            G.from_edge_pairs(bad, 5, sym) if sym else G.from_edge_pairs([(0, 1), (7, 0)], 5, False)
        assert dev_err.value.status == G.ERR_EXPORT and str(dev_err.value) == str(host_err.value)
    with pytest.raises(GrafeoCudaError) as dev_err:
        G.GpuGraph.from_edge_pairs_oriented(bad, 5, device)
    with pytest.raises(GrafeoCudaError) as host_err:
        G.from_edge_pairs_oriented(bad, 5)
    assert str(dev_err.value) == str(host_err.value)
    # A directed target >= num_nodes passes the builder and fails validation.
    host = G.from_edge_pairs([(0, 1), (1, 9), (2, 0)], 4, False)
    with pytest.raises(GrafeoCudaError) as host_err:
        G.GpuGraph.from_csr(host.offsets, host.targets, device)
    with pytest.raises(GrafeoCudaError) as dev_err:
        G.GpuGraph.from_edge_pairs([(0, 1), (1, 9), (2, 0)], 4, False, device)
    assert dev_err.value.status == G.ERR_INVALID_CSR and str(dev_err.value) == str(host_err.value)


@pytest.mark.parametrize("scale,ef,seed", [(1, 4, 0), (8, 16, 1), (12, 16, 2), (14, 8, 9)])
def test_device_rmat_equals_host_rmat(device, scale, ef, seed):
    h = G.generate_rmat(scale, ef, 0.57, 0.19, 0.19, seed=seed)
    g = G.GpuGraph.generate_rmat(device, scale, ef, 0.57, 0.19, 0.19, seed=seed)
    csr_equal(g, h.offsets, h.targets, (scale, ef, seed))
    h = G.generate_rmat(scale, ef, 0.45, 0.25, 0.25, seed=seed)
    csr_equal(G.GpuGraph.generate_rmat(device, scale, ef, 0.45, 0.25, 0.25, seed=seed), h.offsets, h.targets, "a=.45")


@pytest.mark.parametrize("n,m,seed", [(0, 10, 1), (1, 10, 1), (1000, 16000, 3), (70000, 600000, 4)])
def test_device_erdos_renyi_equals_host(device, n, m, seed):
    h = G.generate_erdos_renyi(n, m, seed=seed)
    csr_equal(G.GpuGraph.generate_erdos_renyi(device, n, m, seed=seed), h.offsets, h.targets, (n, m))


@pytest.mark.parametrize("w,h,drop,seed", [(1, 1, 0.05, 0), (1, 9, 0.0, 1), (7, 1, 0.5, 2), (40, 31, 0.05, 3),
                                           (300, 200, 0.05, 4)])
def test_device_grid(device, w, h, drop, seed):
    o, t = graphs.symmetric_csr(w * h, *graphs.grid_pairs(w, h, drop, seed))
    csr_equal(G.GpuGraph.generate_grid(device, w, h, drop, seed), o, t, (w, h))


@pytest.mark.parametrize("n,k,p,seed", [(1, 10, 0.1, 0), (11, 10, 0.1, 1), (256, 10, 0.1, 2), (5000, 10, 0.3, 3)])
def test_device_watts_strogatz(device, n, k, p, seed):
    o, t = graphs.symmetric_csr(n, *graphs.watts_strogatz_pairs(n, k, p, seed))
    csr_equal(G.GpuGraph.generate_watts_strogatz(device, n, k, p, seed), o, t, (n, k, p))


@pytest.mark.parametrize("n,deg,seed", [(1, 8, 0), (2, 8, 1), (500, 8, 2), (3000, 64, 3), (3000, 8, 4)])
def test_device_geometric(device, n, deg, seed):
    o, t = graphs.symmetric_csr(n, *graphs.geometric_pairs(n, deg, seed))
    g = G.GpuGraph.generate_geometric(device, n, deg, seed)
    csr_equal(g, o, t, (n, deg))


def test_device_generated_graph_runs_the_algorithms(device):
    g = G.GpuGraph.generate_rmat(device, 11, 16, seed=7)
    c = g.to_csr()
    assert g.triangle_count()["total_triangles"] == O.triangle_count(c.offsets, c.targets)
    d = g.bfs_array(0)["distances"]
    assert np.array_equal(d, O.bfs(c.offsets, c.targets, 0)["distances"])
