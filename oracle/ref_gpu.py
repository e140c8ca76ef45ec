"""The reference's own CUDA kernels on this GPU — TEST INFRASTRUCTURE ONLY.

ctypes wrapper of oracle/_ref/libref_gpu.so (built by `make -C oracle ref`
from the reference checkout's kernels and oracle/ref_gpu.cu, which restates
the Rust launch sequences). Only tests/ use it: as a second oracle and to time
the reference kernels beside ours on the same device.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libref_gpu.so")
u32p = C.POINTER(C.c_uint32)


def available() -> bool:
    return os.path.exists(LIB_PATH)


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = C.CDLL(LIB_PATH)
        _lib.ref_pagerank.argtypes = [u32p, u32p, C.c_uint32, C.c_uint32, C.c_float, C.c_uint32, C.c_float,
                                      C.POINTER(C.c_float), u32p, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        _lib.ref_bfs.argtypes = [u32p, u32p, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_int32), u32p,
                                 C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        _lib.ref_triangle_count.argtypes = [u32p, u32p, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint64),
                                            C.POINTER(C.c_double)]
        _lib.ref_k_truss.argtypes = [u32p, u32p, C.c_uint32, C.c_uint32, C.c_uint32, u32p, C.POINTER(C.c_uint64),
                                     u32p, C.POINTER(C.c_double)]
        for f in (_lib.ref_pagerank, _lib.ref_bfs, _lib.ref_triangle_count, _lib.ref_k_truss):
            f.restype = C.c_int
    return _lib


def _csr(offsets, targets):
    o = np.ascontiguousarray(np.asarray(offsets, dtype=np.uint32))
    t = np.ascontiguousarray(np.asarray(targets, dtype=np.uint32))
    if t.size == 0:
        t = np.zeros(1, dtype=np.uint32)
    return o, t, len(o) - 1, int(o[-1])


def pagerank(offsets, targets, damping=0.85, max_iterations=100, tolerance=1e-6) -> dict:
    o, t, n, m = _csr(offsets, targets)
    ranks = np.zeros(max(n, 1), dtype=np.float32)
    it, conv, ms = C.c_uint32(), C.c_int(), C.c_double()
    rc = lib().ref_pagerank(o.ctypes.data_as(u32p), t.ctypes.data_as(u32p), n, m, damping, max_iterations,
                            tolerance, ranks.ctypes.data_as(C.POINTER(C.c_float)), C.byref(it), C.byref(conv),
                            C.byref(ms))
    assert rc == 0, rc
    return {"ranks": ranks[:n], "iterations": int(it.value), "converged": bool(conv.value), "device_ms": ms.value}


def bfs(offsets, targets, source: int) -> dict:
    o, t, n, m = _csr(offsets, targets)
    dist = np.zeros(max(n, 1), dtype=np.int32)
    reach, depth, ms = C.c_uint32(), C.c_int32(), C.c_double()
    rc = lib().ref_bfs(o.ctypes.data_as(u32p), t.ctypes.data_as(u32p), n, m, int(source),
                       dist.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(reach), C.byref(depth), C.byref(ms))
    assert rc == 0, rc
    return {"distances": dist[:n], "reachable": int(reach.value), "max_depth": int(depth.value),
            "device_ms": ms.value}


def triangle_count(offsets, targets) -> dict:
    """{'total_triangles', 'device_ms'}, or None where the reference refuses
    the size (more than 134,217,727 forward edges)."""
    o, t, n, m = _csr(offsets, targets)
    total, ms = C.c_uint64(), C.c_double()
    rc = lib().ref_triangle_count(o.ctypes.data_as(u32p), t.ctypes.data_as(u32p), n, m, C.byref(total),
                                  C.byref(ms))
    if rc == 2:
        return None
    assert rc == 0, rc
    return {"total_triangles": int(total.value), "device_ms": ms.value}


def k_truss(offsets, targets, k: int) -> dict:
    """{'edges' (m x 2, u < v, CSR order), 'iterations', 'device_ms'}; k < 3
    raises ValueError (the reference's Kernel error)."""
    o, t, n, m = _csr(offsets, targets)
    out = np.zeros(max(m, 2), dtype=np.uint32)
    count, it, ms = C.c_uint64(), C.c_uint32(), C.c_double()
    rc = lib().ref_k_truss(o.ctypes.data_as(u32p), t.ctypes.data_as(u32p), n, m, int(k), out.ctypes.data_as(u32p),
                           C.byref(count), C.byref(it), C.byref(ms))
    if rc == 3:
        raise ValueError("k must be >= 3 for k-truss decomposition")
    assert rc == 0, rc
    e = int(count.value)
    return {"edges": out[: 2 * e].reshape(e, 2), "iterations": int(it.value), "device_ms": ms.value}
