"""The allocation-free oriented triangle count, through the C ABI.

This entry point serves callers that cannot allocate device memory when they
need a count (their memory pool owns the device, or their framework forbids
side allocations): they pass a CSR already on the device and get the count,
with the library's fixed internal array as the only working memory. The test
puts a degree-oriented CSR on the device with torch (the caller's memory), calls
the entry point twice in a row on the same stream, and checks both results
against the regular gcu_triangle_count_oriented, which must agree exactly
(integer counts). This file is named to be collected last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import grafeo_cuda as G
from grafeo_cuda import _lib

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


@pytest.mark.parametrize("scale,seed", [(12, 5), (16, 2)])
def test_noalloc_matches_the_regular_entry_point_twice(scale, seed):
    import torch

    csr = G.generate_rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed)
    src = np.repeat(np.arange(csr.num_nodes, dtype=np.uint32), np.diff(csr.offsets))
    oriented = G.from_edge_pairs_oriented(np.stack([src, csr.targets], axis=1), csr.num_nodes)

    dev = G.GpuDevice(0)
    expected = G.GpuGraph.from_csr_arrays(oriented, dev).triangle_count_oriented()["total_triangles"]
    assert expected > 0

    offsets = torch.from_numpy(oriented.offsets.astype(np.int32)).cuda()
    targets = torch.from_numpy(oriented.targets.astype(np.int32)).cuda()
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    first = count_noalloc(offsets, targets, stream.cuda_stream)
    second = count_noalloc(offsets, targets, stream.cuda_stream)
    assert first == expected
    assert second == expected


def test_noalloc_rejects_graphs_over_its_limit():
    import torch

    n = (1 << 20) + 1
    offsets = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    targets = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(G.GrafeoCudaError) as e:
        count_noalloc(offsets, targets, 0)
    assert e.value.status == G.ERR_KERNEL
    assert "at most 1048576" in str(e.value)
