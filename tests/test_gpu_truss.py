"""GPU parity for the truss decomposition (per-edge trussness).

Bit-exact against the oracle, which derives trussness from the definition by
running k_truss for k = 3, 4, ... (the reference's tests sweep k = 3..8,
correctness.rs:305-326); and consistent with gcu_k_truss: for every k the
entries with u < v and trussness >= k are exactly k_truss(k)'s edges.
"""
from __future__ import annotations

import numpy as np
import pytest

import grafeo_cuda as G
from grafeo_cuda import GrafeoCudaError
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def check(device, offsets, targets, label, ks=None):
    o, t = np.asarray(offsets, dtype=np.uint32), np.asarray(targets, dtype=np.uint32)
    g = G.GpuGraph.from_csr(o, t, device)
    r = g.truss_decomposition()
    ref = O.truss_decomposition(o, t)
    assert np.array_equal(r["trussness"], ref["trussness"]), label
    assert r["max_trussness"] == ref["max_trussness"], label
    src = np.repeat(np.arange(len(o) - 1, dtype=np.uint32), np.diff(o))
    for k in ks or range(3, ref["max_trussness"] + 2):
        sel = (src < t) & (r["trussness"] >= k)
        expected = np.stack([src[sel], t[sel]], axis=1)
        assert np.array_equal(g.k_truss_array(k)["edges"], expected), (label, k)


def test_truss_decomposition_on_catalog_messy_and_random(device, golden_graphs):
    for gg in golden_graphs:
        check(device, gg["offsets"], gg["targets"], gg["name"])


@pytest.mark.parametrize("scale,seed", [(10, 1), (13, 4)])
def test_truss_decomposition_on_rmat(device, scale, seed):
    csr = G.generate_rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed)
    check(device, csr.offsets, csr.targets, f"rmat{scale}", ks=(3, 4, 6, 9))


def test_truss_decomposition_edge_cases(device):
    g = G.GpuGraph.from_csr([0, 0, 0], [], device)
    r = g.truss_decomposition()
    assert r["max_trussness"] == 0 and len(r["trussness"]) == 0
    g = G.GpuGraph.from_csr([0, 1, 1], [1], device)  # not symmetric
    with pytest.raises(GrafeoCudaError) as e:
        g.truss_decomposition()
    assert e.value.status == G.ERR_KERNEL
