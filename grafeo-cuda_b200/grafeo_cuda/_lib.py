"""ctypes binding of libgrafeo_cuda.so (the C ABI in include/grafeo_cuda.h).

The library is built in place by grafeo-cuda_b200/build.py. There is no
fallback: if the shared library is missing, importing the module raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# GRAFEO_CUDA_LIBRARY may name another build of the same C ABI (for example a
# build with different compile-time tuning); the default is the in-place build.
LIB_PATH = os.environ.get("GRAFEO_CUDA_LIBRARY") or os.path.join(_HERE, "libgrafeo_cuda.so")

u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)
f32p = C.POINTER(C.c_float)
u16p = C.POINTER(C.c_uint16)
u8p = C.POINTER(C.c_uint8)

# name -> (restype, argtypes); mirrors include/grafeo_cuda.h one to one.
SIGNATURES = {
    "gcu_last_error": (C.c_char_p, []),
    "gcu_version": (C.c_char_p, []),
    "gcu_device_count": (C.c_int, []),
    "gcu_device_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "gcu_device_destroy": (None, [C.c_void_p]),
    "gcu_device_name": (C.c_char_p, [C.c_void_p]),
    "gcu_device_ordinal": (C.c_int, [C.c_void_p]),
    "gcu_device_total_memory": (C.c_uint64, [C.c_void_p]),
    "gcu_device_sm_count": (C.c_int, [C.c_void_p]),
    "gcu_device_stream": (C.c_void_p, [C.c_void_p]),
    "gcu_device_synchronize": (C.c_int, [C.c_void_p]),
    "gcu_device_timer_start": (C.c_int, [C.c_void_p]),
    "gcu_device_timer_stop": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "gcu_device_launch_count": (C.c_uint64, [C.c_void_p]),
    "gcu_device_set_kernel_timing": (None, [C.c_void_p, C.c_int]),
    "gcu_device_set_bfs_device_loop": (None, [C.c_void_p, C.c_int]),
    "gcu_device_kernel_stats": (C.c_size_t, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "gcu_device_reset_stats": (None, [C.c_void_p]),
    "gcu_validate_csr": (C.c_int, [u32p, C.c_size_t, u32p, C.c_size_t]),
    "gcu_csr_from_edge_pairs": (C.c_int, [u32p, C.c_size_t, C.c_uint32, C.c_int, C.POINTER(C.c_void_p)]),
    "gcu_csr_from_edge_pairs_oriented": (C.c_int, [u32p, C.c_size_t, C.c_uint32, C.POINTER(C.c_void_p)]),
    "gcu_parse_tsv_to_edges": (
        C.c_int,
        [C.c_char_p, C.POINTER(u32p), C.POINTER(C.c_size_t), C.POINTER(C.c_uint32)],
    ),
    "gcu_free_pairs": (None, [u32p]),
    "gcu_generate_rmat": (
        C.c_int,
        [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint64, C.POINTER(C.c_void_p)],
    ),
    "gcu_generate_erdos_renyi": (C.c_int, [C.c_uint32, C.c_uint64, C.c_uint64, C.POINTER(C.c_void_p)]),
    "gcu_csr_num_nodes": (C.c_uint32, [C.c_void_p]),
    "gcu_csr_num_edges": (C.c_uint64, [C.c_void_p]),
    "gcu_csr_offsets": (u32p, [C.c_void_p]),
    "gcu_csr_targets": (u32p, [C.c_void_p]),
    "gcu_csr_free": (None, [C.c_void_p]),
    "gcu_graph_from_csr": (C.c_int, [C.c_void_p, u32p, C.c_size_t, u32p, C.c_size_t, C.POINTER(C.c_void_p)]),
    "gcu_graph_num_nodes": (C.c_uint32, [C.c_void_p]),
    "gcu_graph_num_edges": (C.c_uint32, [C.c_void_p]),
    "gcu_graph_destroy": (None, [C.c_void_p]),
    "gcu_graph_copy_csr": (C.c_int, [C.c_void_p, u32p, u32p]),
    "gcu_graph_from_edge_pairs": (
        C.c_int,
        [C.c_void_p, u32p, C.c_size_t, C.c_uint32, C.c_int, C.POINTER(C.c_void_p)],
    ),
    "gcu_graph_from_edge_pairs_oriented": (
        C.c_int,
        [C.c_void_p, u32p, C.c_size_t, C.c_uint32, C.POINTER(C.c_void_p)],
    ),
    "gcu_graph_generate_rmat": (
        C.c_int,
        [C.c_void_p, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint64, C.POINTER(C.c_void_p)],
    ),
    "gcu_graph_generate_erdos_renyi": (
        C.c_int,
        [C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64, C.POINTER(C.c_void_p)],
    ),
    "gcu_graph_generate_grid": (
        C.c_int,
        [C.c_void_p, C.c_uint32, C.c_uint32, C.c_double, C.c_uint64, C.POINTER(C.c_void_p)],
    ),
    "gcu_graph_generate_watts_strogatz": (
        C.c_int,
        [C.c_void_p, C.c_uint32, C.c_uint32, C.c_double, C.c_uint64, C.POINTER(C.c_void_p)],
    ),
    "gcu_graph_generate_geometric": (
        C.c_int,
        [C.c_void_p, C.c_uint32, C.c_double, C.c_uint64, C.POINTER(C.c_void_p)],
    ),
    "gcu_triangle_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_double)]),
    "gcu_triangle_count_oriented": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_double)]),
    "gcu_triangle_count_oriented_noalloc": (
        C.c_int,
        [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.POINTER(C.c_uint64)],
    ),
    "gcu_bfs": (
        C.c_int,
        [C.c_void_p, C.c_uint32, i32p, C.POINTER(C.c_uint32), C.POINTER(C.c_int32), C.POINTER(C.c_double)],
    ),
    "gcu_pagerank": (
        C.c_int,
        [
            C.c_void_p,
            C.c_float,
            C.c_uint32,
            C.c_float,
            f32p,
            C.POINTER(C.c_uint32),
            C.POINTER(C.c_int),
            C.POINTER(C.c_double),
        ],
    ),
    "gcu_pagerank_directed": (
        C.c_int,
        [
            C.c_void_p,
            C.c_float,
            C.c_uint32,
            C.c_float,
            f32p,
            C.POINTER(C.c_uint32),
            C.POINTER(C.c_int),
            C.POINTER(C.c_double),
        ],
    ),
    "gcu_personalized_pagerank": (
        C.c_int,
        [
            C.c_void_p,
            u32p,
            C.c_size_t,
            C.c_int,
            C.c_float,
            C.c_uint32,
            C.c_float,
            f32p,
            C.POINTER(C.c_uint32),
            C.POINTER(C.c_int),
            C.POINTER(C.c_double),
        ],
    ),
    "gcu_pagerank_gather_probe": (
        C.c_int,
        [C.c_void_p, C.c_int, C.c_uint32, C.POINTER(C.c_double)],
    ),
    "gcu_k_truss": (
        C.c_int,
        [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p), C.POINTER(C.c_uint32), C.POINTER(C.c_double)],
    ),
    "gcu_truss_decomposition": (
        C.c_int,
        [C.c_void_p, u32p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_double)],
    ),
    "gcu_batch_generate": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint64, C.POINTER(C.c_void_p)]),
    "gcu_batch_from_csr": (
        C.c_int,
        [C.c_void_p, u32p, C.c_size_t, u32p, C.c_size_t, u32p, C.c_size_t, C.POINTER(C.c_void_p)],
    ),
    "gcu_batch_destroy": (None, [C.c_void_p]),
    "gcu_batch_num_graphs": (C.c_uint32, [C.c_void_p]),
    "gcu_batch_num_nodes": (C.c_uint32, [C.c_void_p]),
    "gcu_batch_num_edges": (C.c_uint32, [C.c_void_p]),
    "gcu_batch_vertex_base": (C.c_int, [C.c_void_p, u32p]),
    "gcu_batch_copy_csr": (C.c_int, [C.c_void_p, u32p, u32p]),
    "gcu_batch_member": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)]),
    "gcu_batch_triangle_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_double)]),
    "gcu_batch_set_bfs_sources": (C.c_int, [C.c_void_p, u32p, C.c_uint32, C.c_int]),
    "gcu_batch_bfs": (C.c_int, [C.c_void_p, i32p, u32p, i32p, C.POINTER(C.c_double)]),
    "gcu_batch_set_pagerank_seeds": (
        C.c_int,
        [C.c_void_p, u32p, C.c_uint32, C.c_float, C.c_uint32, C.c_float],
    ),
    "gcu_batch_personalized_pagerank": (C.c_int, [C.c_void_p, f32p, u32p, u8p, C.POINTER(C.c_double)]),
    "gcu_batch_capture": (C.c_int, [C.c_void_p]),
    "gcu_batch_replay": (C.c_int, [C.c_void_p]),
    "gcu_batch_results": (
        C.c_int,
        [C.c_void_p, C.POINTER(C.c_uint64), i32p, u32p, i32p, f32p, u32p, u8p],
    ),
    "gcu_batch_tuning": (C.c_size_t, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "gcu_device_set_schedule": (C.c_int, [C.c_void_p, u16p]),
    "gcu_schedule_forward": (C.c_int, [C.c_void_p, u16p, f32p, C.c_size_t, f32p]),
    "gcu_schedule_gradient": (
        C.c_int,
        [C.c_void_p, u16p, f32p, f32p, u8p, C.c_size_t, C.POINTER(C.c_double), f32p],
    ),
    "gcu_schedule_train": (
        C.c_int,
        [
            C.c_void_p,
            f32p,
            u16p,
            f32p,
            f32p,
            u8p,
            C.c_size_t,
            C.c_uint32,
            C.c_uint32,
            C.c_float,
            C.c_uint64,
            C.POINTER(C.c_double),
        ],
    ),
    "gcu_bfs_trace": (
        C.c_int,
        [C.c_void_p, C.c_uint32, C.c_uint64, f32p, f32p, u8p, u8p, u8p, C.c_size_t, C.POINTER(C.c_size_t)],
    ),
    "gcu_triangle_trace": (
        C.c_int,
        [C.c_void_p, f32p, f32p, u8p, u8p, C.c_size_t, C.POINTER(C.c_size_t), C.POINTER(C.c_uint64)],
    ),
    "gcu_edge_list_len": (C.c_size_t, [C.c_void_p]),
    "gcu_edge_list_data": (u32p, [C.c_void_p]),
    "gcu_edge_list_free": (None, [C.c_void_p]),
}

# gcu_status values (include/grafeo_cuda.h)
OK = 0
ERR_NO_DEVICE = 1
ERR_DRIVER = 2
ERR_OUT_OF_MEMORY = 3
ERR_KERNEL = 4
ERR_EXPORT = 5
ERR_INVALID_CSR = 6


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library with "
            "`python grafeo-cuda_b200/build.py` (there is no CPU fallback)"
        )
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class GrafeoCudaError(RuntimeError):
    """A failed call; `status` is the gcu_status code (CudaError variant)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def check(status: int) -> None:
    if status != OK:
        raise GrafeoCudaError(status, lib.gcu_last_error().decode())
