"""Oracle — TEST INFRASTRUCTURE ONLY (ctypes wrapper of liboracle.so).

Loads the C restatement in oracle.c (building it with `make` when the shared
library is missing). Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg import this module; the product never does. See oracle.h for
what each function restates and how the oracle is pinned.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

u32p = C.POINTER(C.c_uint32)


def build(force: bool = False) -> str:
    newest = max(os.path.getmtime(os.path.join(HERE, f)) for f in ("oracle.c", "oracle_scale.c", "oracle.h"))
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < newest:
        subprocess.run(["make", "-B", "-C", HERE], check=True, capture_output=True)
    return LIB_PATH


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    lib.orc_triangle_count.restype = C.c_uint64
    lib.orc_triangle_count.argtypes = [u32p, u32p, C.c_uint32]
    lib.orc_triangle_count_oriented.restype = C.c_uint64
    lib.orc_triangle_count_oriented.argtypes = [u32p, u32p, C.c_uint32]
    lib.orc_bfs.restype = None
    lib.orc_bfs.argtypes = [u32p, u32p, C.c_uint32, C.c_uint32, C.POINTER(C.c_int32), u32p, C.POINTER(C.c_int32)]
    lib.orc_pagerank.restype = None
    lib.orc_pagerank.argtypes = [
        u32p, u32p, C.c_uint32, u32p, C.c_double, C.c_uint32, C.c_double, C.c_int,
        C.POINTER(C.c_double), u32p, C.POINTER(C.c_int),
    ]
    lib.orc_pagerank_tele.restype = None
    lib.orc_pagerank_tele.argtypes = [
        u32p, u32p, C.c_uint32, u32p, C.POINTER(C.c_double), C.c_double, C.c_uint32, C.c_double, C.c_int,
        C.POINTER(C.c_double), u32p, C.POINTER(C.c_int),
    ]
    lib.orc_transpose.restype = C.c_size_t
    lib.orc_transpose.argtypes = [u32p, u32p, C.c_uint32, u32p, u32p]
    lib.orc_k_truss.restype = C.c_size_t
    lib.orc_k_truss.argtypes = [u32p, u32p, C.c_uint32, C.c_uint32, u32p, u32p]
    lib.orc_from_edge_pairs.restype = C.c_size_t
    lib.orc_from_edge_pairs.argtypes = [u32p, C.c_size_t, C.c_uint32, C.c_int, u32p, u32p]
    lib.orc_from_edge_pairs_oriented.restype = C.c_size_t
    lib.orc_from_edge_pairs_oriented.argtypes = [u32p, C.c_size_t, C.c_uint32, u32p, u32p]
    lib.orc_num_threads.restype = C.c_int
    lib.orc_num_threads.argtypes = []
    lib.orc_generate_rmat.restype = C.c_size_t
    lib.orc_generate_rmat.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                      u32p, u32p]
    lib.orc_generate_erdos_renyi.restype = C.c_size_t
    lib.orc_generate_erdos_renyi.argtypes = [C.c_uint32, C.c_uint64, C.c_uint64, u32p, u32p]
    lib.orc_transpose_sorted.restype = C.c_size_t
    lib.orc_transpose_sorted.argtypes = [u32p, u32p, C.c_uint32, u32p, u32p]
    lib.orc_edge_support.restype = C.c_int
    lib.orc_edge_support.argtypes = [u32p, u32p, C.c_uint32, u32p]
    lib.orc_k_truss_peel.restype = C.c_size_t
    lib.orc_k_truss_peel.argtypes = [u32p, u32p, C.c_uint32, C.c_uint32, u32p, u32p, u32p]
    lib.orc_truss_decomposition_peel.restype = C.c_int
    lib.orc_truss_decomposition_peel.argtypes = [u32p, u32p, C.c_uint32, u32p, u32p, u32p, u32p]
    return lib


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def _p(a: np.ndarray, t=C.c_uint32):
    return a.ctypes.data_as(C.POINTER(t))


def num_threads() -> int:
    return int(lib().orc_num_threads())


def triangle_count(offsets, targets) -> int:
    o, t = _u32(offsets), _u32(targets)
    return int(lib().orc_triangle_count(_p(o), _p(t), len(o) - 1))


def triangle_count_oriented(offsets, targets) -> int:
    o, t = _u32(offsets), _u32(targets)
    return int(lib().orc_triangle_count_oriented(_p(o), _p(t), len(o) - 1))


def bfs(offsets, targets, source: int) -> dict:
    o, t = _u32(offsets), _u32(targets)
    n = len(o) - 1
    dist = np.empty(max(n, 1), dtype=np.int32)
    reach = C.c_uint32()
    depth = C.c_int32()
    lib().orc_bfs(_p(o), _p(t), n, int(source), _p(dist, C.c_int32), C.byref(reach), C.byref(depth))
    return {"distances": dist[:n], "reachable": int(reach.value), "max_depth": int(depth.value)}


def pagerank(offsets, targets, damping=0.85, max_iterations=100, tolerance=1e-6, rule="l1",
             out_degree=None, tele=None) -> dict:
    """rule 'l1': the reference GPU stopping rule; 'max': Grafeo's. The CSR
    holds the pulled (in-)lists; out_degree defaults to their lengths; tele is
    an optional personalisation vector."""
    o, t = _u32(offsets), _u32(targets)
    n = len(o) - 1
    ranks = np.zeros(max(n, 1), dtype=np.float64)
    it = C.c_uint32()
    conv = C.c_int()
    od = None if out_degree is None else _u32(out_degree)
    tv = None if tele is None else np.ascontiguousarray(np.asarray(tele, dtype=np.float64))
    lib().orc_pagerank_tele(
        _p(o), _p(t), n, None if od is None else _p(od), None if tv is None else _p(tv, C.c_double),
        float(damping), int(max_iterations), float(tolerance), 0 if rule == "l1" else 1, _p(ranks, C.c_double),
        C.byref(it), C.byref(conv),
    )
    return {"ranks": ranks[:n], "iterations": int(it.value), "converged": bool(conv.value)}


def transpose(offsets, targets):
    o, t = _u32(offsets), _u32(targets)
    n = len(o) - 1
    to = np.zeros(n + 1, dtype=np.uint32)
    tt = np.zeros(max(len(t), 1), dtype=np.uint32)
    lib().orc_transpose(_p(o), _p(t), n, _p(to), _p(tt))
    return to, tt[: len(t)]


def transpose_sorted(offsets, targets):
    """transpose() by the parallel radix sort (for graphs at scale)."""
    o, t = _u32(offsets), _u32(targets)
    n = len(o) - 1
    to = np.zeros(n + 1, dtype=np.uint32)
    tt = np.zeros(max(len(t), 1), dtype=np.uint32)
    lib().orc_transpose_sorted(_p(o), _p(t), n, _p(to), _p(tt))
    return to, tt[: len(t)]


def pagerank_directed(offsets, targets, damping=0.85, max_iterations=100, tolerance=1e-6, rule="l1",
                      tele=None) -> dict:
    """PageRank of the directed graph whose out-edges are the CSR lists."""
    o = _u32(offsets)
    to, tt = transpose_sorted(offsets, targets) if len(o) > (1 << 16) else transpose(offsets, targets)
    return pagerank(to, tt, damping, max_iterations, tolerance, rule, out_degree=np.diff(o), tele=tele)


def seed_vector(n: int, seeds) -> np.ndarray:
    """Personalisation vector of the seeds: 1/len(seeds) each, repeats add up."""
    p = np.zeros(n, dtype=np.float64)
    for s in seeds:
        p[int(s)] += 1.0 / len(seeds)
    return p


def k_truss(offsets, targets, k: int) -> dict:
    o, t = _u32(offsets), _u32(targets)
    n = len(o) - 1
    out = np.zeros(max(2 * len(t), 2), dtype=np.uint32)
    it = C.c_uint32()
    m = int(lib().orc_k_truss(_p(o), _p(t), n, int(k), _p(out), C.byref(it)))
    return {"edges": out[: 2 * m].reshape(m, 2), "iterations": int(it.value)}


def truss_decomposition(offsets, targets) -> dict:
    """Trussness per CSR entry from the definition: the largest k whose
    k-truss (k_truss above, k = 3, 4, ...) holds the edge; 2 for the other
    edges, 0 for self-loops. Symmetric CSR."""
    o, t = _u32(offsets), _u32(targets)
    n = len(o) - 1
    src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(o))
    truss = np.where(src == t, 0, 2).astype(np.uint32)
    key = (src.astype(np.uint64) << np.uint64(32)) | t.astype(np.uint64)  # sorted: CSR order
    k, top = 3, (2 if np.any(src != t) else 0)
    while True:
        edges = k_truss(o, t, k)["edges"]
        if len(edges) == 0:
            break
        u, v = edges[:, 0].astype(np.uint64), edges[:, 1].astype(np.uint64)
        for a, b in ((u, v), (v, u)):
            truss[np.searchsorted(key, (a << np.uint64(32)) | b)] = k
        top = k
        k += 1
    return {"trussness": truss, "max_trussness": top}


def from_edge_pairs(edges, num_nodes: int, symmetric: bool):
    p = _u32(edges).reshape(-1)
    offsets = np.zeros(num_nodes + 1, dtype=np.uint32)
    targets = np.zeros(max(len(p), 1), dtype=np.uint32)
    m = lib().orc_from_edge_pairs(_p(p), len(p) // 2, num_nodes, 1 if symmetric else 0, _p(offsets), _p(targets))
    if m == C.c_size_t(-1).value:
        raise ValueError("edge references a node >= num_nodes")
    return offsets, targets[:m]


def from_edge_pairs_oriented(edges, num_nodes: int):
    p = _u32(edges).reshape(-1)
    offsets = np.zeros(num_nodes + 1, dtype=np.uint32)
    targets = np.zeros(max(len(p) // 2, 1), dtype=np.uint32)
    m = lib().orc_from_edge_pairs_oriented(_p(p), len(p) // 2, num_nodes, _p(offsets), _p(targets))
    if m == C.c_size_t(-1).value:
        raise ValueError("edge references a node >= num_nodes")
    return offsets, targets[:m]


# ---------------------------------------------------------------- at scale (oracle_scale.c)


class Csr:
    """A CSR built by the oracle's generators (same fields as the library's)."""

    def __init__(self, offsets: np.ndarray, targets: np.ndarray):
        self.offsets, self.targets = offsets, targets
        self.num_nodes, self.num_edges = len(offsets) - 1, len(targets)


def generate_rmat(scale: int, edge_factor: int, a: float, b: float, c: float, seed: int) -> Csr:
    n = 1 << scale
    offsets = np.zeros(n + 1, dtype=np.uint32)
    targets = np.empty(max(2 * (edge_factor << scale), 1), dtype=np.uint32)
    m = lib().orc_generate_rmat(scale, edge_factor, a, b, c, seed, _p(offsets), _p(targets))
    if m == C.c_size_t(-1).value:
        raise ValueError("R-MAT scale must be in 1..=31")
    return Csr(offsets, targets[:m].copy())


def generate_erdos_renyi(n: int, num_pairs: int, seed: int) -> Csr:
    offsets = np.zeros(n + 1, dtype=np.uint32)
    targets = np.empty(max(2 * num_pairs, 1), dtype=np.uint32)
    m = lib().orc_generate_erdos_renyi(n, num_pairs, seed, _p(offsets), _p(targets))
    return Csr(offsets, targets[:m].copy())


def edge_support(offsets, targets) -> np.ndarray:
    """Triangles through the edge of every entry (simple symmetric CSR)."""
    o, t = _u32(offsets), _u32(targets)
    s = np.zeros(max(len(t), 1), dtype=np.uint32)
    if lib().orc_edge_support(_p(o), _p(t), len(o) - 1, _p(s)) != 0:
        raise ValueError("edge_support needs a simple symmetric CSR")
    return s[: len(t)]


def k_truss_peel(offsets, targets, k: int, support=None) -> dict:
    """k_truss() for a simple symmetric CSR by incremental peeling."""
    o, t = _u32(offsets), _u32(targets)
    out = np.zeros(max(len(t), 2), dtype=np.uint32)
    it = C.c_uint32()
    sp = None if support is None else _p(_u32(support))
    m = lib().orc_k_truss_peel(_p(o), _p(t), len(o) - 1, int(k), sp, _p(out), C.byref(it))
    if m == C.c_size_t(-1).value:
        raise ValueError("k_truss_peel needs a simple symmetric CSR")
    return {"edges": out[: 2 * m].reshape(m, 2), "iterations": int(it.value)}


def truss_decomposition_peel(offsets, targets, support=None) -> dict:
    """truss_decomposition() for a simple symmetric CSR by peeling, with the
    synchronous round count."""
    o, t = _u32(offsets), _u32(targets)
    tr = np.zeros(max(len(t), 1), dtype=np.uint32)
    top, rounds = C.c_uint32(), C.c_uint32()
    sp = None if support is None else _p(_u32(support))
    if lib().orc_truss_decomposition_peel(_p(o), _p(t), len(o) - 1, sp, _p(tr), C.byref(top), C.byref(rounds)) != 0:
        raise ValueError("truss_decomposition_peel needs a simple symmetric CSR")
    return {"trussness": tr[: len(t)], "max_trussness": int(top.value), "rounds": int(rounds.value)}
