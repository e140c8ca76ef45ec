"""The allocation-free oriented triangle count, through the C ABI.

This entry point serves callers that cannot allocate device memory when they
need a count (their memory pool owns the device, or their framework forbids
side allocations): they pass a CSR already on the device and get the count,
with the library's fixed internal array as the only working memory. The tests
put degree-oriented CSRs on the device with torch (the caller's memory), call
the entry point twice in a row on the same stream, and check both results
against the regular gcu_triangle_count_oriented and the oracle, which must
agree exactly (integer counts). The graphs cover both kernels the count runs:
short out-lists (a warp per vertex) and out-lists longer than 2,048 entries
(a CTA with a binary search of the list), and a graph at the 2^20-vertex
limit. This file is named to be collected last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import grafeo_cuda as G
from grafeo_cuda import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def count_noalloc(offsets, targets, stream_ptr) -> int:
    total = C.c_uint64()
    _lib.check(
        _lib.lib.gcu_triangle_count_oriented_noalloc(
            C.c_void_p(offsets.data_ptr()), C.c_void_p(targets.data_ptr()), offsets.numel() - 1, targets.numel(),
            C.c_void_p(stream_ptr), C.byref(total),
        )
    )
    return int(total.value)


def oriented_of(num_nodes: int, offsets: np.ndarray, targets: np.ndarray):
    src = np.repeat(np.arange(num_nodes, dtype=np.uint32), np.diff(offsets))
    return G.from_edge_pairs_oriented(np.stack([src, targets], axis=1), num_nodes)


def bipartite_with_right_edges(side: int, right_pairs: int, seed: int):
    """K_{side,side} plus random edges among the right side: every right
    vertex has a higher degree than every left vertex, so each left vertex's
    oriented out-list holds all `side` right vertices."""
    left = np.repeat(np.arange(side, dtype=np.uint32), side)
    right = np.tile(np.arange(side, 2 * side, dtype=np.uint32), side)
    rng = np.random.default_rng(seed)
    extra = rng.integers(side, 2 * side, size=(right_pairs, 2), dtype=np.uint32)
    pairs = np.concatenate([np.stack([left, right], axis=1), extra])
    return G.from_edge_pairs(pairs, 2 * side, True)


def check_twice(oriented, expected: int):
    import torch

    dev = G.GpuDevice(0)
    regular = G.GpuGraph.from_csr_arrays(oriented, dev).triangle_count_oriented()["total_triangles"]
    assert regular == expected
    offsets = torch.from_numpy(oriented.offsets.astype(np.int32)).cuda()
    targets = torch.from_numpy(oriented.targets.astype(np.int32)).cuda()
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    first = count_noalloc(offsets, targets, stream.cuda_stream)
    second = count_noalloc(offsets, targets, stream.cuda_stream)
    assert first == expected
    assert second == expected


@pytest.mark.parametrize("scale,seed", [(12, 5), (16, 2)])
def test_noalloc_matches_regular_entry_point_and_oracle_twice(scale, seed):
    csr = G.generate_rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed)
    oriented = oriented_of(csr.num_nodes, csr.offsets, csr.targets)
    expected = O.triangle_count_oriented(oriented.offsets, oriented.targets)
    assert expected > 0
    check_twice(oriented, expected)


def test_noalloc_out_lists_over_2048_entries():
    sym = bipartite_with_right_edges(2100, 30000, seed=8)
    oriented = oriented_of(sym.num_nodes, sym.offsets, sym.targets)
    assert np.diff(oriented.offsets).max() > 2048
    expected = O.triangle_count_oriented(oriented.offsets, oriented.targets)
    assert expected == O.triangle_count(sym.offsets, sym.targets) > 0
    check_twice(oriented, expected)


def test_noalloc_at_its_vertex_limit():
    csr = G.generate_rmat(20, 16, 0.57, 0.19, 0.19, seed=3)
    assert csr.num_nodes == 1 << 20
    oriented = oriented_of(csr.num_nodes, csr.offsets, csr.targets)
    expected = int(O.edge_support(csr.offsets, csr.targets).sum(dtype=np.uint64)) // 6
    check_twice(oriented, expected)


def test_noalloc_rejects_graphs_over_its_limit():
    import torch

    n = (1 << 20) + 1
    offsets = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    targets = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(G.GrafeoCudaError) as e:
        count_noalloc(offsets, targets, 0)
    assert e.value.status == G.ERR_KERNEL
    assert "at most 1048576" in str(e.value)
