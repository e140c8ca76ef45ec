"""grafeo_cuda — B200 (sm_100a) graph hot paths behind grafeo-cuda's API.

Mirrors the reference's Python module `grafeo_cuda`
(crates/bindings/python/src/gpu_graph.rs:11-155): `GpuDevice(ordinal=0)` with
`.name` / `.total_memory`, and `GpuGraph.from_csr(offsets, targets, device)`
with `.num_nodes`, `.num_edges`, `.triangle_count()`, `.pagerank(damping=0.85,
max_iterations=100, tolerance=1e-6)`, `.bfs(source)` and `.k_truss(k)`, each
returning a dict with the reference's keys. Failures raise RuntimeError with
the reference's CudaError text (GrafeoCudaError is a RuntimeError subclass
that also carries the status code).

It also exposes the core crate's CSR helpers (crates/grafeo-cuda-core/src/
csr_export.rs): `CsrArrays`, `validate_csr`, `from_edge_pairs`,
`from_edge_pairs_oriented`, `parse_tsv_to_edges`, plus the synthetic graph
generators used by the tests and the benchmark.

Everything runs through the C ABI of libgrafeo_cuda.so; there is no CPU
fallback for any algorithm.
"""
from __future__ import annotations

import ctypes as C
import json
from dataclasses import dataclass

import numpy as np

from ._lib import (  # noqa: F401
    ERR_DRIVER,
    ERR_EXPORT,
    ERR_INVALID_CSR,
    ERR_KERNEL,
    ERR_NO_DEVICE,
    ERR_OUT_OF_MEMORY,
    LIB_PATH,
    OK,
    GrafeoCudaError,
    check,
    lib,
)

__all__ = [
    "GpuDevice",
    "GpuGraph",
    "CsrArrays",
    "GrafeoCudaError",
    "validate_csr",
    "from_edge_pairs",
    "from_edge_pairs_oriented",
    "parse_tsv_to_edges",
    "generate_rmat",
    "generate_erdos_renyi",
    "device_count",
    "version",
]


SCHEDULE_FEATURES = 12
SCHEDULE_OUTPUTS = 3
SCHEDULE_PARAMS = 1571


def version() -> str:
    return lib.gcu_version().decode()


def device_count() -> int:
    return int(lib.gcu_device_count())


def _u32_array(values, what: str) -> np.ndarray:
    """Converts a list or array to contiguous u32, refusing values outside u32
    (PyO3's Vec<u32> extraction raises OverflowError for those)."""
    if isinstance(values, np.ndarray) and values.dtype == np.uint32:
        return np.ascontiguousarray(values)
    arr = np.asarray(values)
    if arr.size == 0:
        return np.zeros(0, dtype=np.uint32)
    if arr.dtype.kind not in "iu":
        if arr.dtype.kind == "f" or arr.dtype == object:
            arr = np.asarray(values, dtype=np.int64)
        else:
            raise TypeError(f"{what} must be a sequence of integers")
    if arr.dtype.kind == "i" and arr.min() < 0 or arr.max() > 0xFFFFFFFF:
        raise OverflowError(f"{what} holds a value outside u32")
    return np.ascontiguousarray(arr, dtype=np.uint32)


def _ptr(arr: np.ndarray, ctype=C.c_uint32):
    return arr.ctypes.data_as(C.POINTER(ctype))


# ---------------------------------------------------------------- device


class GpuDevice:
    """A CUDA GPU device (device.rs:22-66): one stream, calls are synchronous."""

    def __init__(self, ordinal: int = 0):
        h = C.c_void_p()
        check(lib.gcu_device_create(int(ordinal), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.gcu_device_destroy(h)
            self._h = None

    @property
    def name(self) -> str:
        return lib.gcu_device_name(self._h).decode()

    @property
    def total_memory(self) -> int:
        return int(lib.gcu_device_total_memory(self._h))

    @property
    def ordinal(self) -> int:
        return int(lib.gcu_device_ordinal(self._h))

    @property
    def sm_count(self) -> int:
        return int(lib.gcu_device_sm_count(self._h))

    # -- measurement helpers (CUDA events on the device stream)
    def synchronize(self) -> None:
        check(lib.gcu_device_synchronize(self._h))

    def timer_start(self) -> None:
        check(lib.gcu_device_timer_start(self._h))

    def timer_stop(self) -> float:
        ms = C.c_float()
        check(lib.gcu_device_timer_stop(self._h, C.byref(ms)))
        return float(ms.value)

    @property
    def launch_count(self) -> int:
        return int(lib.gcu_device_launch_count(self._h))

    def set_kernel_timing(self, on: bool) -> None:
        lib.gcu_device_set_kernel_timing(self._h, 1 if on else 0)

    def set_bfs_device_loop(self, on: bool) -> None:
        """BFS level loop on the device (default) or driven from the host;
        the host drives it whenever per-kernel timing is on."""
        lib.gcu_device_set_bfs_device_loop(self._h, 1 if on else 0)

    def kernel_stats(self) -> dict:
        n = lib.gcu_device_kernel_stats(self._h, None, 0)
        buf = C.create_string_buffer(int(n))
        lib.gcu_device_kernel_stats(self._h, buf, n)
        return {k: (int(v[0]), float(v[1])) for k, v in json.loads(buf.value.decode()).items()}

    def reset_stats(self) -> None:
        lib.gcu_device_reset_stats(self._h)

    # -- learned schedule (grafeo_cuda.schedule trains and loads it)
    def set_schedule(self, weights) -> None:
        """Installs a schedule network (GCU_SCHEDULE_PARAMS BF16 bit patterns as
        uint16) for bfs and triangle_count; None restores the fixed rules."""
        if weights is None:
            check(lib.gcu_device_set_schedule(self._h, None))
            return
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.uint16))
        if w.size != SCHEDULE_PARAMS:
            raise ValueError(f"a schedule network has {SCHEDULE_PARAMS} parameters, got {w.size}")
        check(lib.gcu_device_set_schedule(self._h, _ptr(w, C.c_uint16)))


# ---------------------------------------------------------------- host CSR


@dataclass
class CsrArrays:
    """CSR arrays in host memory (csr_export.rs:16-30)."""

    offsets: np.ndarray
    targets: np.ndarray
    num_nodes: int
    num_edges: int

    def validate(self) -> None:
        """CsrArrays::validate (csr_export.rs:37-54)."""
        validate_csr(self.offsets, self.targets)
        nodes = len(self.offsets) - 1
        if self.num_nodes != nodes:
            raise GrafeoCudaError(
                ERR_INVALID_CSR,
                f"invalid CSR: num_nodes is {self.num_nodes} but offsets describe {nodes} nodes",
            )
        if self.num_edges != len(self.targets):
            raise GrafeoCudaError(
                ERR_INVALID_CSR,
                f"invalid CSR: num_edges is {self.num_edges} but targets has {len(self.targets)} entries",
            )


def _take_csr(handle: C.c_void_p) -> CsrArrays:
    try:
        n = int(lib.gcu_csr_num_nodes(handle))
        m = int(lib.gcu_csr_num_edges(handle))
        offsets = np.ctypeslib.as_array(lib.gcu_csr_offsets(handle), shape=(n + 1,)).copy()
        if m:
            targets = np.ctypeslib.as_array(lib.gcu_csr_targets(handle), shape=(m,)).copy()
        else:
            targets = np.zeros(0, dtype=np.uint32)
        return CsrArrays(offsets, targets, n, m)
    finally:
        lib.gcu_csr_free(handle)


def validate_csr(offsets, targets) -> None:
    """validate_csr (csr_export.rs:71-120); raises GrafeoCudaError(INVALID_CSR)."""
    o = _u32_array(offsets, "offsets")
    t = _u32_array(targets, "targets")
    check(lib.gcu_validate_csr(_ptr(o), o.size, _ptr(t), t.size))


def _pairs(edges) -> np.ndarray:
    arr = _u32_array(edges, "edges")
    return np.ascontiguousarray(arr.reshape(-1, 2)) if arr.size else np.zeros((0, 2), dtype=np.uint32)


def from_edge_pairs(edges, num_nodes: int, symmetric: bool) -> CsrArrays:
    """from_edge_pairs (csr_export.rs:202-239)."""
    p = _pairs(edges)
    h = C.c_void_p()
    check(lib.gcu_csr_from_edge_pairs(_ptr(p), p.shape[0], int(num_nodes), 1 if symmetric else 0, C.byref(h)))
    return _take_csr(h)


def from_edge_pairs_oriented(edges, num_nodes: int) -> CsrArrays:
    """from_edge_pairs_oriented (csr_export.rs:299-350)."""
    p = _pairs(edges)
    h = C.c_void_p()
    check(lib.gcu_csr_from_edge_pairs_oriented(_ptr(p), p.shape[0], int(num_nodes), C.byref(h)))
    return _take_csr(h)


def parse_tsv_to_edges(path) -> tuple[list[tuple[int, int]], int]:
    """parse_tsv_to_edges (csr_export.rs:246-287): (edge pairs, num_nodes)."""
    pp = C.POINTER(C.c_uint32)()
    n_pairs = C.c_size_t()
    nodes = C.c_uint32()
    check(lib.gcu_parse_tsv_to_edges(str(path).encode(), C.byref(pp), C.byref(n_pairs), C.byref(nodes)))
    try:
        m = int(n_pairs.value)
        flat = np.ctypeslib.as_array(pp, shape=(2 * m,)).copy() if m else np.zeros(0, dtype=np.uint32)
    finally:
        lib.gcu_free_pairs(pp)
    edges = [(int(flat[2 * i]), int(flat[2 * i + 1])) for i in range(m)]
    return edges, int(nodes.value)


def generate_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
                  seed: int = 1) -> CsrArrays:
    """Symmetric R-MAT graph without self-loops or duplicates (SplitMix64 stream)."""
    h = C.c_void_p()
    check(lib.gcu_generate_rmat(int(scale), int(edge_factor), float(a), float(b), float(c), int(seed), C.byref(h)))
    return _take_csr(h)


def generate_erdos_renyi(num_nodes: int, num_pairs: int, seed: int = 3) -> CsrArrays:
    """Symmetric G(n, m) graph from num_pairs uniform pairs, loops and repeats dropped."""
    h = C.c_void_p()
    check(lib.gcu_generate_erdos_renyi(int(num_nodes), int(num_pairs), int(seed), C.byref(h)))
    return _take_csr(h)


# ---------------------------------------------------------------- device graph


class GpuGraph:
    """A graph stored in GPU memory as CSR (gpu_graph.rs:15-26)."""

    def __init__(self, handle: C.c_void_p, device: GpuDevice):
        self._h = handle
        self._device = device  # keeps the Python device object alive too

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.gcu_graph_destroy(h)
            self._h = None

    @staticmethod
    def from_csr(offsets, targets, device: GpuDevice) -> "GpuGraph":
        """GpuGraph.from_csr(offsets, targets, device) (python/src/gpu_graph.rs:54-59)."""
        o = _u32_array(offsets, "offsets")
        t = _u32_array(targets, "targets")
        h = C.c_void_p()
        check(lib.gcu_graph_from_csr(device._h, _ptr(o), o.size, _ptr(t), t.size, C.byref(h)))
        return GpuGraph(h, device)

    @staticmethod
    def from_csr_arrays(csr: CsrArrays, device: GpuDevice) -> "GpuGraph":
        """GpuGraph::from_csr_arrays (gpu_graph.rs:46-60): validates the declared counts too."""
        nodes = len(csr.offsets) - 1
        if csr.num_nodes != nodes or csr.num_edges != len(csr.targets):
            csr.validate()
        return GpuGraph.from_csr(csr.offsets, csr.targets, device)

    @staticmethod
    def _built(call, device: GpuDevice, *args) -> "GpuGraph":
        h = C.c_void_p()
        check(call(device._h, *args, C.byref(h)))
        return GpuGraph(h, device)

    @staticmethod
    def from_edge_pairs(edges, num_nodes: int, symmetric: bool, device: GpuDevice) -> "GpuGraph":
        """from_edge_pairs + from_csr_arrays (csr_export.rs:202-239), sorted and
        deduplicated on the device."""
        p = _pairs(edges)
        return GpuGraph._built(lib.gcu_graph_from_edge_pairs, device, _ptr(p), p.shape[0], int(num_nodes),
                               1 if symmetric else 0)

    @staticmethod
    def from_edge_pairs_oriented(edges, num_nodes: int, device: GpuDevice) -> "GpuGraph":
        """from_edge_pairs_oriented (csr_export.rs:299-350) on the device."""
        p = _pairs(edges)
        return GpuGraph._built(lib.gcu_graph_from_edge_pairs_oriented, device, _ptr(p), p.shape[0], int(num_nodes))

    @staticmethod
    def generate_rmat(device: GpuDevice, scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
                      c: float = 0.19, seed: int = 1) -> "GpuGraph":
        """generate_rmat drawn on the device (the same CSR)."""
        return GpuGraph._built(lib.gcu_graph_generate_rmat, device, int(scale), int(edge_factor), float(a), float(b),
                               float(c), int(seed))

    @staticmethod
    def generate_erdos_renyi(device: GpuDevice, num_nodes: int, num_pairs: int, seed: int = 3) -> "GpuGraph":
        return GpuGraph._built(lib.gcu_graph_generate_erdos_renyi, device, int(num_nodes), int(num_pairs), int(seed))

    @staticmethod
    def generate_grid(device: GpuDevice, width: int, height: int, drop: float = 0.05, seed: int = 0) -> "GpuGraph":
        return GpuGraph._built(lib.gcu_graph_generate_grid, device, int(width), int(height), float(drop), int(seed))

    @staticmethod
    def generate_watts_strogatz(device: GpuDevice, num_nodes: int, k: int = 10, p: float = 0.1,
                                seed: int = 0) -> "GpuGraph":
        return GpuGraph._built(lib.gcu_graph_generate_watts_strogatz, device, int(num_nodes), int(k), float(p),
                               int(seed))

    @staticmethod
    def generate_geometric(device: GpuDevice, num_nodes: int, avg_degree: float, seed: int = 0) -> "GpuGraph":
        return GpuGraph._built(lib.gcu_graph_generate_geometric, device, int(num_nodes), float(avg_degree),
                               int(seed))

    def to_csr(self) -> CsrArrays:
        """The device CSR copied back to host arrays."""
        o = np.empty(self.num_nodes + 1, dtype=np.uint32)
        t = np.empty(max(self.num_edges, 1), dtype=np.uint32)
        check(lib.gcu_graph_copy_csr(self._h, _ptr(o), _ptr(t)))
        return CsrArrays(o, t[: self.num_edges], self.num_nodes, self.num_edges)

    @property
    def num_nodes(self) -> int:
        return int(lib.gcu_graph_num_nodes(self._h))

    @property
    def num_edges(self) -> int:
        return int(lib.gcu_graph_num_edges(self._h))

    @property
    def device(self) -> GpuDevice:
        return self._device

    # -- reference methods (dicts with the PyO3 keys)

    def triangle_count(self) -> dict:
        total = C.c_uint64()
        secs = C.c_double()
        check(lib.gcu_triangle_count(self._h, C.byref(total), C.byref(secs)))
        return {"total_triangles": int(total.value), "time_seconds": float(secs.value)}

    def triangle_count_oriented(self) -> dict:
        total = C.c_uint64()
        secs = C.c_double()
        check(lib.gcu_triangle_count_oriented(self._h, C.byref(total), C.byref(secs)))
        return {"total_triangles": int(total.value), "time_seconds": float(secs.value)}

    def pagerank(self, damping: float = 0.85, max_iterations: int = 100, tolerance: float = 1e-6) -> dict:
        r = self.pagerank_array(damping, max_iterations, tolerance)
        r["ranks"] = r["ranks"].tolist()
        return r

    def bfs(self, source: int) -> dict:
        r = self.bfs_array(source)
        r["distances"] = r["distances"].tolist()
        return r

    def k_truss(self, k: int) -> dict:
        r = self.k_truss_array(k)
        r["edges"] = [(int(u), int(v)) for u, v in r["edges"]]
        return r

    # -- the same calls returning numpy arrays (or nothing, with copy_result=False)

    def _check_u32(self, x: int, what: str) -> int:
        if x < 0 or x > 0xFFFFFFFF:
            raise OverflowError(f"{what} out of range for u32")
        return int(x)

    def bfs_array(self, source: int, copy_result: bool = True) -> dict:
        source = self._check_u32(source, "source")
        n = self.num_nodes
        dist = np.empty(n, dtype=np.int32) if copy_result else None
        reach = C.c_uint32()
        depth = C.c_int32()
        secs = C.c_double()
        ptr = dist.ctypes.data_as(C.POINTER(C.c_int32)) if copy_result and n else None
        check(lib.gcu_bfs(self._h, source, ptr, C.byref(reach), C.byref(depth), C.byref(secs)))
        return {
            "distances": dist,
            "reachable": int(reach.value),
            "max_depth": int(depth.value),
            "time_seconds": float(secs.value),
        }

    def pagerank_array(self, damping: float = 0.85, max_iterations: int = 100, tolerance: float = 1e-6,
                       copy_result: bool = True) -> dict:
        max_iterations = self._check_u32(max_iterations, "max_iterations")
        n = self.num_nodes
        ranks = np.empty(n, dtype=np.float32) if copy_result else None
        it = C.c_uint32()
        conv = C.c_int()
        secs = C.c_double()
        ptr = ranks.ctypes.data_as(C.POINTER(C.c_float)) if copy_result and n else None
        check(
            lib.gcu_pagerank(
                self._h, float(damping), max_iterations, float(tolerance), ptr, C.byref(it), C.byref(conv),
                C.byref(secs),
            )
        )
        return {
            "ranks": ranks,
            "iterations": int(it.value),
            "converged": bool(conv.value),
            "time_seconds": float(secs.value),
        }

    def _pagerank_result(self, call, copy_result: bool) -> dict:
        n = self.num_nodes
        ranks = np.empty(n, dtype=np.float32) if copy_result else None
        it = C.c_uint32()
        conv = C.c_int()
        secs = C.c_double()
        ptr = ranks.ctypes.data_as(C.POINTER(C.c_float)) if copy_result and n else None
        check(call(ptr, C.byref(it), C.byref(conv), C.byref(secs)))
        return {
            "ranks": ranks,
            "iterations": int(it.value),
            "converged": bool(conv.value),
            "time_seconds": float(secs.value),
        }

    def pagerank_directed(self, damping: float = 0.85, max_iterations: int = 100, tolerance: float = 1e-6,
                          copy_result: bool = True) -> dict:
        """PageRank of the directed graph whose out-edges are the CSR lists
        (pulls over a transpose built on the device)."""
        max_iterations = self._check_u32(max_iterations, "max_iterations")
        return self._pagerank_result(
            lambda *a: lib.gcu_pagerank_directed(self._h, float(damping), max_iterations, float(tolerance), *a),
            copy_result,
        )

    def pagerank_gather_probe(self, directed: bool = False, passes: int = 20) -> float:
        """Device ms per launch of the gather probe over this graph's PageRank
        plan (the target stream and contribution gathers alone): the floor of
        a pull SpMV on that layout. A diagnostic; builds the plan if needed."""
        passes = self._check_u32(passes, "passes")
        ms = C.c_double()
        check(lib.gcu_pagerank_gather_probe(self._h, 1 if directed else 0, passes, C.byref(ms)))
        return ms.value

    def personalized_pagerank(self, seeds, damping: float = 0.85, max_iterations: int = 100,
                              tolerance: float = 1e-6, directed: bool = False, copy_result: bool = True) -> dict:
        """PageRank whose teleport and dangling mass go to `seeds` uniformly."""
        max_iterations = self._check_u32(max_iterations, "max_iterations")
        s = _u32_array(seeds, "seeds")
        return self._pagerank_result(
            lambda *a: lib.gcu_personalized_pagerank(
                self._h, _ptr(s), s.size, 1 if directed else 0, float(damping), max_iterations, float(tolerance), *a
            ),
            copy_result,
        )

    def truss_decomposition(self, copy_result: bool = True) -> dict:
        """Trussness of every CSR entry's edge (symmetric CSR): the largest k
        whose k-truss holds the edge (2: in no triangle, 0: self-loop)."""
        n = self.num_edges
        truss = np.empty(n, dtype=np.uint32) if copy_result else None
        top = C.c_uint32()
        rounds = C.c_uint32()
        secs = C.c_double()
        ptr = truss.ctypes.data_as(C.POINTER(C.c_uint32)) if copy_result and n else None
        check(lib.gcu_truss_decomposition(self._h, ptr, C.byref(top), C.byref(rounds), C.byref(secs)))
        return {"trussness": truss, "max_trussness": int(top.value), "rounds": int(rounds.value),
                "time_seconds": float(secs.value)}

    def k_truss_array(self, k: int) -> dict:
        k = self._check_u32(k, "k")
        h = C.c_void_p()
        it = C.c_uint32()
        secs = C.c_double()
        check(lib.gcu_k_truss(self._h, k, C.byref(h), C.byref(it), C.byref(secs)))
        try:
            m = int(lib.gcu_edge_list_len(h))
            if m:
                edges = np.ctypeslib.as_array(lib.gcu_edge_list_data(h), shape=(2 * m,)).copy().reshape(m, 2)
            else:
                edges = np.zeros((0, 2), dtype=np.uint32)
        finally:
            lib.gcu_edge_list_free(h)
        return {"edges": edges, "k": k, "iterations": int(it.value), "time_seconds": float(secs.value)}

    def bfs_trace(self, source: int, explore_seed: int = 0, capacity: int = 65536) -> dict:
        """Per-level trace of every BFS step variant (gcu_bfs_trace): features
        [levels, 12], times_us [levels, 3] (NaN where a variant is not valid),
        valid masks, the alpha/beta rule's picks and the variants taken."""
        source = self._check_u32(source, "source")
        cap = int(max(1, capacity))
        f = np.zeros((cap, SCHEDULE_FEATURES), dtype=np.float32)
        t = np.zeros((cap, SCHEDULE_OUTPUTS), dtype=np.float32)
        valid = np.zeros(cap, dtype=np.uint8)
        fixed = np.zeros(cap, dtype=np.uint8)
        taken = np.zeros(cap, dtype=np.uint8)
        n = C.c_size_t()
        check(lib.gcu_bfs_trace(self._h, source, int(explore_seed), _ptr(f, C.c_float), _ptr(t, C.c_float),
                                _ptr(valid, C.c_uint8), _ptr(fixed, C.c_uint8), _ptr(taken, C.c_uint8), cap,
                                C.byref(n)))
        m = min(int(n.value), cap)
        return {"features": f[:m], "times_us": t[:m], "valid": valid[:m], "fixed_rule": fixed[:m],
                "taken": taken[:m], "levels": int(n.value)}

    def triangle_trace(self) -> dict:
        """Per out-degree bucket trace of every intersection variant
        (gcu_triangle_trace), plus the triangle count they all reproduce."""
        cap = 33
        f = np.zeros((cap, SCHEDULE_FEATURES), dtype=np.float32)
        t = np.zeros((cap, SCHEDULE_OUTPUTS), dtype=np.float32)
        valid = np.zeros(cap, dtype=np.uint8)
        fixed = np.zeros(cap, dtype=np.uint8)
        n = C.c_size_t()
        total = C.c_uint64()
        check(lib.gcu_triangle_trace(self._h, _ptr(f, C.c_float), _ptr(t, C.c_float), _ptr(valid, C.c_uint8),
                                     _ptr(fixed, C.c_uint8), cap, C.byref(n), C.byref(total)))
        m = int(n.value)
        return {"features": f[:m], "times_us": t[:m], "valid": valid[:m], "fixed_rule": fixed[:m],
                "total_triangles": int(total.value)}


from .batch import GpuBatch  # noqa: E402  (needs the classes above)


# ---------------------------------------------------------------- schedule network kernels


def schedule_forward(device: GpuDevice, weights, features) -> np.ndarray:
    """Predictions [n, 3] of the schedule network (gcu_schedule_forward)."""
    w = np.ascontiguousarray(np.asarray(weights, dtype=np.uint16))
    x = np.ascontiguousarray(np.asarray(features, dtype=np.float32).reshape(-1, SCHEDULE_FEATURES))
    out = np.zeros((x.shape[0], SCHEDULE_OUTPUTS), dtype=np.float32)
    check(lib.gcu_schedule_forward(device._h, _ptr(w, C.c_uint16), _ptr(x, C.c_float), x.shape[0],
                                   _ptr(out, C.c_float)))
    return out


def schedule_gradient(device: GpuDevice, weights, features, targets, mask) -> tuple[float, np.ndarray]:
    """(masked MSE loss, gradient [1571]) computed on the device."""
    w = np.ascontiguousarray(np.asarray(weights, dtype=np.uint16))
    x = np.ascontiguousarray(np.asarray(features, dtype=np.float32).reshape(-1, SCHEDULE_FEATURES))
    y = np.ascontiguousarray(np.asarray(targets, dtype=np.float32).reshape(-1, SCHEDULE_OUTPUTS))
    m = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8).reshape(-1, SCHEDULE_OUTPUTS))
    loss = C.c_double()
    grad = np.zeros(SCHEDULE_PARAMS, dtype=np.float32)
    check(lib.gcu_schedule_gradient(device._h, _ptr(w, C.c_uint16), _ptr(x, C.c_float), _ptr(y, C.c_float),
                                    _ptr(m, C.c_uint8), x.shape[0], C.byref(loss), _ptr(grad, C.c_float)))
    return float(loss.value), grad


def schedule_train(device: GpuDevice, master, features, targets, mask, steps: int, batch: int = 1024,
                   lr: float = 3e-3, seed: int = 0) -> tuple[np.ndarray, np.ndarray, float]:
    """Adam on the device; returns (FP32 master weights, BF16 weights as uint16, final loss)."""
    mw = np.array(master, dtype=np.float32).copy()
    w16 = np.zeros(SCHEDULE_PARAMS, dtype=np.uint16)
    x = np.ascontiguousarray(np.asarray(features, dtype=np.float32).reshape(-1, SCHEDULE_FEATURES))
    y = np.ascontiguousarray(np.asarray(targets, dtype=np.float32).reshape(-1, SCHEDULE_OUTPUTS))
    m = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8).reshape(-1, SCHEDULE_OUTPUTS))
    loss = C.c_double()
    check(lib.gcu_schedule_train(device._h, _ptr(mw, C.c_float), _ptr(w16, C.c_uint16), _ptr(x, C.c_float),
                                 _ptr(y, C.c_float), _ptr(m, C.c_uint8), x.shape[0], int(steps), int(batch),
                                 float(lr), int(seed), C.byref(loss)))
    return mw, w16, float(loss.value)
