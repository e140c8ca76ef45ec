"""The reference's own CUDA kernels, compiled for sm_100a (oracle/_ref, see
oracle/ref_gpu.cu), as a second oracle and as the speed to beat on this GPU.

* Parity: triangle counts and BFS distances equal the reference kernels' on
  the catalog, messy and random graphs and R-MAT 12/14; PageRank ranks after
  the same number of iterations agree within 1e-5 L1 (both are FP32; the
  reference sums with float atomics, so its own last bits vary run to run);
  k-truss edge sets and round counts for k = 3..8 equal the reference
  kernels' (crates/grafeo-cuda-algos/kernels/k_truss.cu driven as in
  src/k_truss.rs:42-161) on the same graphs, self-loop cases included.
* Speed: PageRank, BFS and triangle counting at R-MAT scale 18 and PageRank and
  BFS at scale 22, and the k-truss sweep at R-MAT 13, device time of the
  reference's launch sequence against ours (printed; ours must not be slower).
"""
from __future__ import annotations

import numpy as np
import pytest

import grafeo_cuda as G
from oracle import ref_gpu as R

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="reference kernels not built")]


def small_graphs(golden_graphs):
    out = [(g["name"], np.asarray(g["offsets"], np.uint32), np.asarray(g["targets"], np.uint32))
           for g in golden_graphs if len(g["offsets"]) > 1]
    for scale, seed in ((12, 1), (14, 1)):
        c = G.generate_rmat(scale, 16, seed=seed)
        out.append((f"rmat{scale}", c.offsets, c.targets))
    return out


def test_results_equal_the_reference_kernels(device, golden_graphs):
    for name, o, t in small_graphs(golden_graphs):
        g = G.GpuGraph.from_csr(o, t, device)
        ref = R.triangle_count(o, t)
        assert ref is not None and g.triangle_count()["total_triangles"] == ref["total_triangles"], name
        n = len(o) - 1
        for s in sorted({0, n // 2, n - 1}):
            r = R.bfs(o, t, s)
            mine = g.bfs_array(s)
            assert np.array_equal(mine["distances"], r["distances"]), (name, s)
            assert mine["reachable"] == r["reachable"] and mine["max_depth"] == r["max_depth"], (name, s)
        r = R.pagerank(o, t, 0.85, 20, 0.0)
        mine = g.pagerank_array(0.85, 20, 0.0)
        assert r["iterations"] == mine["iterations"] == 20
        assert np.abs(mine["ranks"].astype(np.float64) - r["ranks"]).sum() <= 1e-5, name


def test_k_truss_equals_the_reference_kernels(device, golden_graphs):
    cases = small_graphs(golden_graphs)
    # Self-loops: the reference's first round counts them as common neighbours.
    sl = G.from_edge_pairs([(0, 1), (1, 2), (0, 2), (2, 3), (3, 3), (2, 2), (1, 1)], 4, True)
    cases.append(("self-loops", sl.offsets, sl.targets))
    for name, o, t in cases:
        g = G.GpuGraph.from_csr(o, t, device)
        for k in range(3, 9):
            r = R.k_truss(o, t, k)
            mine = g.k_truss_array(k)
            assert np.array_equal(mine["edges"], r["edges"]), (name, k)
            assert mine["iterations"] == r["iterations"], (name, k)
    with pytest.raises(ValueError):
        R.k_truss(cases[0][1], cases[0][2], 2)


def _device_ms(device, fn):
    device.synchronize()
    device.timer_start()
    fn()
    return device.timer_stop()


@pytest.mark.parametrize("scale", [18, 22])
def test_faster_than_the_reference_kernels(device, scale):
    csr = G.generate_rmat(scale, 16, seed=2)
    o, t = csr.offsets, csr.targets
    g = G.GpuGraph.from_csr_arrays(csr, device)
    deg = np.diff(o)
    src = int(np.flatnonzero(deg > 0)[0])
    rows = {}
    g.pagerank_array(0.85, 20, 0.0, copy_result=False)
    ref = R.pagerank(o, t, 0.85, 20, 0.0)
    rows["pagerank_20_iterations"] = (ref["device_ms"], _device_ms(device, lambda: g.pagerank_array(0.85, 20, 0.0)))
    g.bfs_array(src, copy_result=False)
    ref = R.bfs(o, t, src)
    rows["bfs"] = (ref["device_ms"], _device_ms(device, lambda: g.bfs_array(src)))
    if scale <= 18:
        g.triangle_count()
        ref = R.triangle_count(o, t)
        rows["triangle_count"] = (ref["device_ms"], _device_ms(device, g.triangle_count))
    for k, (r_ms, m_ms) in rows.items():
        print(f"R-MAT {scale} {k}: reference kernels {r_ms:.3f} ms, ours {m_ms:.3f} ms, {r_ms / m_ms:.1f}x")
        assert m_ms <= r_ms, k


def test_k_truss_faster_than_the_reference_kernels(device):
    # R-MAT 13: the reference recomputes every support every round with one
    # thread per node, which takes minutes from R-MAT 16 on.
    csr = G.generate_rmat(13, 16, seed=2)
    o, t = csr.offsets, csr.targets
    ref_ms, mine_ms = 0.0, 0.0
    for k in range(3, 9):
        g = G.GpuGraph.from_csr_arrays(csr, device)  # a fresh graph: no cached support
        ref = R.k_truss(o, t, k)
        ms = _device_ms(device, lambda: g.k_truss_array(k))
        assert ms > 0
        ref_ms += ref["device_ms"]
        mine_ms += ms
    print(f"R-MAT 13 k-truss k = 3..8: reference kernels {ref_ms:.1f} ms, ours {mine_ms:.1f} ms, "
          f"{ref_ms / mine_ms:.1f}x")
    assert mine_ms <= ref_ms
