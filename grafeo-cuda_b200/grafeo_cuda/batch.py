"""Batched form: many graphs packed into one CSR (the gcu_batch_* C ABI).

    b = GpuBatch.generate(device, 4096, seed=4)       # R-MAT / Watts-Strogatz corpus
    tri = b.triangle_count()                           # per-graph totals
    b.set_bfs_sources(sources)                         # [num_graphs, S] local ids
    r = b.bfs()                                        # distances [S, num_nodes], reachable/max_depth [G, S]
    b.set_pagerank_seeds(seeds)                        # [num_graphs, K] local ids
    p = b.personalized_pagerank()                      # ranks [num_nodes], iterations/converged [G]
    b.capture(); b.replay(); b.results()               # all three as one CUDA graph

Graph i owns the union vertices [vertex_base[i], vertex_base[i + 1]);
`member(i)` copies it out as a plain GpuGraph with local ids, for the
per-graph loop the batch replaces.
"""
from __future__ import annotations

import ctypes as C
import json

import numpy as np

from . import CsrArrays, GpuDevice, GpuGraph, _ptr, _u32_array
from ._lib import check, lib


class GpuBatch:
    def __init__(self, handle: C.c_void_p, device: GpuDevice):
        self._h = handle
        self._device = device
        self.num_graphs = int(lib.gcu_batch_num_graphs(handle))
        self.num_nodes = int(lib.gcu_batch_num_nodes(handle))
        self.num_edges = int(lib.gcu_batch_num_edges(handle))
        vb = np.zeros(self.num_graphs + 1, dtype=np.uint32)
        check(lib.gcu_batch_vertex_base(handle, _ptr(vb)))
        self.vertex_base = vb
        self.S = 0
        self.K = 0
        self._keep = True

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.gcu_batch_destroy(h)
            self._h = None

    @staticmethod
    def generate(device: GpuDevice, num_graphs: int, seed: int = 4) -> "GpuBatch":
        h = C.c_void_p()
        check(lib.gcu_batch_generate(device._h, int(num_graphs), int(seed), C.byref(h)))
        return GpuBatch(h, device)

    @staticmethod
    def from_csr(vertex_base, offsets, targets, device: GpuDevice) -> "GpuBatch":
        vb = _u32_array(vertex_base, "vertex_base")
        o = _u32_array(offsets, "offsets")
        t = _u32_array(targets, "targets")
        h = C.c_void_p()
        check(lib.gcu_batch_from_csr(device._h, _ptr(vb), vb.size - 1, _ptr(o), o.size, _ptr(t), t.size,
                                     C.byref(h)))
        return GpuBatch(h, device)

    @staticmethod
    def from_graphs(csrs, device: GpuDevice) -> "GpuBatch":
        """Packs host CSRs ((offsets, targets) pairs, local ids) into a batch."""
        vb, offs, tgts, nb, eb = [0], [np.zeros(1, np.uint32)], [], 0, 0
        for o, t in csrs:
            o = np.asarray(o, dtype=np.uint64)
            t = np.asarray(t, dtype=np.uint64)
            offs.append((o[1:] + eb).astype(np.uint32))
            tgts.append((t + nb).astype(np.uint32))
            nb += len(o) - 1
            eb += len(t)
            vb.append(nb)
        return GpuBatch.from_csr(vb, np.concatenate(offs), np.concatenate(tgts) if tgts else [], device)

    def to_csr(self) -> CsrArrays:
        o = np.empty(self.num_nodes + 1, dtype=np.uint32)
        t = np.empty(max(self.num_edges, 1), dtype=np.uint32)
        check(lib.gcu_batch_copy_csr(self._h, _ptr(o), _ptr(t)))
        return CsrArrays(o, t[: self.num_edges], self.num_nodes, self.num_edges)

    def member(self, index: int) -> GpuGraph:
        h = C.c_void_p()
        check(lib.gcu_batch_member(self._h, int(index), C.byref(h)))
        return GpuGraph(h, self._device)

    def triangle_count(self) -> dict:
        tot = np.zeros(max(self.num_graphs, 1), dtype=np.uint64)
        secs = C.c_double()
        check(lib.gcu_batch_triangle_count(self._h, tot.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(secs)))
        return {"total_triangles": tot[: self.num_graphs], "time_seconds": float(secs.value)}

    def set_bfs_sources(self, sources, keep_distances: bool = True) -> None:
        s = np.ascontiguousarray(np.asarray(sources, dtype=np.uint32).reshape(self.num_graphs, -1))
        check(lib.gcu_batch_set_bfs_sources(self._h, _ptr(s), s.shape[1], 1 if keep_distances else 0))
        self.S = s.shape[1]
        self._keep = keep_distances

    def _bfs_arrays(self):
        d = np.empty((self.S, self.num_nodes), dtype=np.int32) if self._keep else None
        r = np.empty((self.num_graphs, self.S), dtype=np.uint32)
        m = np.empty((self.num_graphs, self.S), dtype=np.int32)
        return d, r, m

    def bfs(self) -> dict:
        d, r, m = self._bfs_arrays()
        secs = C.c_double()
        check(lib.gcu_batch_bfs(self._h, None if d is None else _ptr(d, C.c_int32), _ptr(r), _ptr(m, C.c_int32),
                                C.byref(secs)))
        return {"distances": d, "reachable": r, "max_depth": m, "time_seconds": float(secs.value)}

    def set_pagerank_seeds(self, seeds, damping: float = 0.85, max_iterations: int = 100,
                           tolerance: float = 1e-6) -> None:
        s = np.ascontiguousarray(np.asarray(seeds, dtype=np.uint32).reshape(self.num_graphs, -1))
        check(lib.gcu_batch_set_pagerank_seeds(self._h, _ptr(s), s.shape[1], float(damping), int(max_iterations),
                                               float(tolerance)))
        self.K = s.shape[1]

    def _ppr_arrays(self):
        return (np.empty(self.num_nodes, dtype=np.float32), np.empty(self.num_graphs, dtype=np.uint32),
                np.empty(self.num_graphs, dtype=np.uint8))

    def personalized_pagerank(self) -> dict:
        ranks, it, conv = self._ppr_arrays()
        secs = C.c_double()
        check(lib.gcu_batch_personalized_pagerank(self._h, _ptr(ranks, C.c_float), _ptr(it), _ptr(conv, C.c_uint8),
                                                  C.byref(secs)))
        return {"ranks": ranks, "iterations": it, "converged": conv.astype(bool), "time_seconds": float(secs.value)}

    def capture(self) -> None:
        check(lib.gcu_batch_capture(self._h))

    def replay(self) -> None:
        check(lib.gcu_batch_replay(self._h))

    def results(self, distances: bool = True) -> dict:
        tri = np.zeros(max(self.num_graphs, 1), dtype=np.uint64)
        d, r, m = self._bfs_arrays()
        if not distances:
            d = None
        ranks, it, conv = self._ppr_arrays()
        check(lib.gcu_batch_results(self._h, tri.ctypes.data_as(C.POINTER(C.c_uint64)),
                                    None if d is None else _ptr(d, C.c_int32), _ptr(r), _ptr(m, C.c_int32),
                                    _ptr(ranks, C.c_float), _ptr(it), _ptr(conv, C.c_uint8)))
        return {"total_triangles": tri[: self.num_graphs], "distances": d, "reachable": r, "max_depth": m,
                "ranks": ranks, "iterations": it, "converged": conv.astype(bool)}

    def tuning(self) -> dict:
        n = lib.gcu_batch_tuning(self._h, None, 0)
        buf = C.create_string_buffer(int(n))
        lib.gcu_batch_tuning(self._h, buf, n)
        return json.loads(buf.value.decode())


# ---------------------------------------------------------------- benchmark


def _sources(batch: GpuBatch, per_graph: int, seed: int) -> np.ndarray:
    """Seeded random sources per graph, drawn among vertices with edges where
    the graph has any."""
    rng = np.random.default_rng(seed)
    csr = batch.to_csr()
    deg = np.diff(csr.offsets)
    vb = batch.vertex_base
    out = np.zeros((batch.num_graphs, per_graph), dtype=np.uint32)
    for g in range(batch.num_graphs):
        live = np.nonzero(deg[vb[g]:vb[g + 1]])[0]
        pool = live if len(live) else np.arange(vb[g + 1] - vb[g])
        out[g] = pool[rng.integers(0, len(pool), size=per_graph)]
    return out


def benchmark(num_graphs: int = 4096, seed: int = 4, sources: int = 16, seeds: int = 8, replays: int = 5,
              loop_graphs: int | None = None, device: GpuDevice | None = None, log=print) -> dict:
    """Batched replay against the per-graph plain loop on the same work:
    triangle counts, BFS from `sources` random sources per graph and
    personalised PageRank from `seeds` seeds per graph (0.85, tol 1e-6)."""
    import time

    dev = device or GpuDevice(0)
    t0 = time.perf_counter()
    b = GpuBatch.generate(dev, num_graphs, seed)
    dev.synchronize()
    gen_s = time.perf_counter() - t0
    src = _sources(b, sources, seed + 1)
    sd = _sources(b, seeds, seed + 2)
    b.set_bfs_sources(src, keep_distances=True)
    b.set_pagerank_seeds(sd, 0.85, 100, 1e-6)
    t0 = time.perf_counter()
    b.capture()
    dev.synchronize()
    plan_s = time.perf_counter() - t0
    b.replay()
    dev.synchronize()
    times = []
    for _ in range(replays):
        dev.timer_start()
        b.replay()
        times.append(dev.timer_stop())
    t0 = time.perf_counter()
    b.replay()
    res = b.results(distances=False)
    e2e_s = time.perf_counter() - t0
    batched_ms = float(np.median(times))
    # Per-graph plain loop over the same graphs, sources and seeds (wall time,
    # the way a caller of the single-graph API runs it).
    n_loop = num_graphs if loop_graphs is None else min(loop_graphs, num_graphs)
    members = [b.member(g) for g in range(n_loop)]
    dev.synchronize()
    mismatches = {"triangles": 0, "bfs_reachable": 0, "pagerank_iterations": []}
    t0 = time.perf_counter()
    for g, m in enumerate(members):
        tri = m.triangle_count()["total_triangles"]
        for k in range(sources):
            r = m.bfs_array(int(src[g, k]), copy_result=False)
            mismatches["bfs_reachable"] += int(r["reachable"] != res["reachable"][g, k])
        p = m.personalized_pagerank(sd[g], 0.85, 100, 1e-6, copy_result=False)
        mismatches["triangles"] += int(tri != res["total_triangles"][g])
        if p["iterations"] != res["iterations"][g]:
            mismatches["pagerank_iterations"].append(g)
    loop_s = time.perf_counter() - t0
    # The two PageRank codes sum in different orders, so a graph whose L1
    # change crosses the tolerance within rounding can stop one iteration
    # apart; report how far apart the ranks are for those graphs.
    vb = b.vertex_base
    for i, g in enumerate(mismatches["pagerank_iterations"]):
        p = members[g].personalized_pagerank(sd[g], 0.85, 100, 1e-6)
        mismatches["pagerank_iterations"][i] = {
            "graph": int(g), "loop": int(p["iterations"]), "batch": int(res["iterations"][g]),
            "ranks_l1_apart": float(np.abs(p["ranks"].astype(np.float64) - res["ranks"][vb[g]:vb[g + 1]]).sum())}
    loop_full_s = loop_s * num_graphs / max(n_loop, 1)
    out = {
        "graphs": num_graphs, "vertices": b.num_nodes, "csr_entries": b.num_edges,
        "bfs_sources_per_graph": sources, "ppr_seeds_per_graph": seeds,
        "generate_s": round(gen_s, 3), "plan_and_capture_s": round(plan_s, 3),
        "batched_replay_ms": round(batched_ms, 3), "batched_e2e_ms": round(1000 * e2e_s, 3),
        "loop_graphs_timed": n_loop, "per_graph_loop_s": round(loop_full_s, 3),
        "speedup_device": round(1000 * loop_full_s / batched_ms, 1),
        "speedup_e2e": round(loop_full_s / e2e_s, 1),
        "loop_mismatches": mismatches, "tuning": b.tuning(),
    }
    log(json.dumps(out, indent=1))
    return out


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description="batched replay vs per-graph plain loop")
    ap.add_argument("--graphs", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--replays", type=int, default=5)
    ap.add_argument("--loop-graphs", type=int, default=None, help="time the plain loop on this many graphs and scale")
    a = ap.parse_args()
    benchmark(a.graphs, a.seed, replays=a.replays, loop_graphs=a.loop_graphs)
