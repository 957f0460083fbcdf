"""ctypes binding of libb40c_bfs.so (the C ABI in include/b40c_bfs.h).

Loading fails loudly when the library has not been built: there is no CPU
fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libb40c_bfs.so")

# status codes (numerically equal to cudaError_t)
SUCCESS = 0
ERROR_INVALID_VALUE = 1
ERROR_MEMORY_ALLOCATION = 2
ERROR_INVALID_CONFIGURATION = 9
ERROR_INVALID_DEVICE_FUNCTION = 98
ERROR_NO_DEVICE = 100
ERROR_NOT_READY = 600
ERROR_LAUNCH_TIMEOUT = 702
ERROR_NOT_SUPPORTED = 801

VERTEX_FRONTIERS, EDGE_FRONTIERS, MIXED_FRONTIERS, MULTI_GPU_FRONTIERS = 0, 1, 2, 3
EXPAND_CONTRACT, CONTRACT_EXPAND, TWO_PHASE, HYBRID, DIRECTION_OPTIMIZING = 0, 1, 2, 3, 4
ENACT_FUSED, ENACT_ITERATIVE, ENACT_GRAPH = 0, 1, 2


class Policy(C.Structure):
    _fields_ = [
        ("threads", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("chunk_edges", C.c_int32),
        ("warp_gather_threshold", C.c_int32),
        ("cta_gather_threshold", C.c_int32),
        ("saturation_quit", C.c_int32),
        ("warp_cull", C.c_int32),
        ("bitmask_precheck", C.c_int32),
        ("queue_allocation", C.c_int32),
        ("bottom_up_alpha", C.c_int32),
        ("bottom_up_beta", C.c_int32),
        ("small_frontier_edges", C.c_int32),
        ("bottom_up_scan", C.c_int32),
        ("bottom_up_hub_probes", C.c_int32),
        ("bottom_up_list", C.c_int32),
        ("bottom_up_defer_frontier", C.c_int32),
        ("subgrid_frontier_edges", C.c_int32),
        ("bottom_up_long_list", C.c_int32),
        ("history_cull", C.c_int32),
        ("bottom_up_prefetch", C.c_int32),
        ("warp_contract", C.c_int32),
        ("warp_bottom_up", C.c_int32),
    ]


class DeviceView(C.Structure):
    _fields_ = [
        ("d_row_offsets", C.c_void_p),
        ("d_column_indices", C.c_void_p),
        ("d_labels", C.c_void_p),
        ("d_visited_mask", C.c_void_p),
        ("visited_mask_bytes", C.c_int64),
        ("nodes", C.c_int64),
        ("edges", C.c_int64),
        ("device", C.c_int32),
        ("mark_predecessors", C.c_int32),
    ]


class LevelRecord(C.Structure):
    _fields_ = [
        ("vertices", C.c_int32),
        ("edges", C.c_int32),
        ("bottom_up", C.c_int32),
        ("pass_", C.c_int32),
        ("t_ns", C.c_uint64),
    ]


class Csr(C.Structure):
    _fields_ = [
        ("nodes", C.c_int64),
        ("edges", C.c_int64),
        ("row_offsets", C.POINTER(C.c_int32)),
        ("column_indices", C.POINTER(C.c_int32)),
        ("pinned", C.c_int32),
    ]


class ServerOptions(C.Structure):
    _fields_ = [
        ("memory_budget_bytes", C.c_int64),
        ("max_batch", C.c_int32),
        ("single_strategy", C.c_int32),
        ("max_in_flight", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("reserved", C.c_int32 * 4),
    ]


class ServerResult(C.Structure):
    _fields_ = [
        ("ticket", C.c_int64),
        ("graph", C.c_int32),
        ("source", C.c_int32),
        ("depth_limit", C.c_int32),
        ("status", C.c_int32),
        ("search_depth", C.c_int32),
        ("batch_size", C.c_int32),
        ("arrival_ns", C.c_int64),
        ("launch_ns", C.c_int64),
        ("finish_ns", C.c_int64),
        ("gpu_start_ns", C.c_int64),
        ("gpu_end_ns", C.c_int64),
    ]


SERVER_RESULT_DTYPE = np.dtype([("ticket", "<i8"), ("graph", "<i4"), ("source", "<i4"), ("depth_limit", "<i4"),
                                ("status", "<i4"), ("search_depth", "<i4"), ("batch_size", "<i4"),
                                ("arrival_ns", "<i8"), ("launch_ns", "<i8"), ("finish_ns", "<i8"),
                                ("gpu_start_ns", "<i8"), ("gpu_end_ns", "<i8")])


class ServerCounters(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64),
        ("completed", C.c_int64),
        ("failed", C.c_int64),
        ("batches", C.c_int64),
        ("batched_queries", C.c_int64),
        ("single_queries", C.c_int64),
        ("memory_used_bytes", C.c_int64),
        ("memory_budget_bytes", C.c_int64),
        ("graphs", C.c_int32),
        ("reserved", C.c_int32),
        ("joined_queries", C.c_int64),
    ]


class B40cError(RuntimeError):
    """A non-zero status from the library; ``.status`` is the cudaError_t value."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


_P_i32 = C.POINTER(C.c_int32)
_P_i64 = C.POINTER(C.c_int64)

# name -> (restype, argtypes); every symbol declared in include/b40c_bfs.h and include/b40c_server.h
SIGNATURES: dict[str, tuple] = {
    "b40c_last_error_string": (C.c_char_p, []),
    "b40c_version": (C.c_char_p, []),
    "b40c_device_count": (C.c_int, [_P_i32]),
    "b40c_bfs_default_policy": (C.c_int, [C.c_int, C.POINTER(Policy)]),
    "b40c_bfs_problem_create": (C.c_int, [_P_i32, _P_i32, C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_int,
                                          C.POINTER(C.c_void_p)]),
    "b40c_bfs_problem_destroy": (C.c_int, [C.c_void_p]),
    "b40c_bfs_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "b40c_bfs_problem_reset": (C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    "b40c_bfs_enact": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int32, C.c_int, C.POINTER(Policy)]),
    "b40c_bfs_enact_limited": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_int,
                                         C.POINTER(Policy)]),
    "b40c_bfs_extract": (C.c_int, [C.c_void_p, _P_i32]),
    "b40c_bfs_extract_async": (C.c_int, [C.c_void_p, _P_i32, C.c_int]),
    "b40c_bfs_extract_wait": (C.c_int, [C.c_void_p, C.c_int]),
    "b40c_bfs_stats": (C.c_int, [C.c_void_p, _P_i64, _P_i32, C.POINTER(C.c_double)]),
    "b40c_bfs_problem_is_symmetric": (C.c_int, [C.c_void_p, _P_i32]),
    "b40c_bfs_set_instrument": (C.c_int, [C.c_void_p, C.c_int]),
    "b40c_bfs_level_records": (C.c_int, [C.c_void_p, C.POINTER(LevelRecord), C.c_int, _P_i32]),
    "b40c_bfs_cta_arrivals": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.c_int, _P_i32]),
    "b40c_bfs_last_elapsed_ms": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "b40c_bfs_recent_search_ms": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float)]),
    "b40c_bfs_device_view_get": (C.c_int, [C.c_void_p, C.POINTER(DeviceView)]),
    "b40c_msbfs_enact": (C.c_int, [C.c_void_p, _P_i32, _P_i32, C.c_int, C.c_int, C.POINTER(Policy)]),
    "b40c_msbfs_extract": (C.c_int, [C.c_void_p, C.c_int, _P_i32]),
    "b40c_msbfs_join": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
    "b40c_msbfs_joined": (C.c_int, [C.c_void_p, _P_i32, _P_i32]),
    "b40c_msbfs_stats": (C.c_int, [C.c_void_p, _P_i32]),
    "b40c_bfs_problem_device_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "b40c_msbfs_device_labels": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), _P_i32]),
    "b40c_bfs_search_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int32, C.c_void_p,
                                          C.c_void_p]),
    "b40c_host_alloc": (C.c_int, [C.POINTER(C.c_void_p), C.c_size_t, C.c_int]),
    "b40c_host_free": (C.c_int, [C.c_void_p]),
    "b40c_build_grid2d": (C.c_int, [C.c_int32, C.c_int, C.POINTER(Csr)]),
    "b40c_build_grid3d": (C.c_int, [C.c_int32, C.c_int, C.POINTER(Csr)]),
    "b40c_build_rmat": (C.c_int, [C.c_int64, C.c_int64, C.c_int, C.c_double, C.c_double, C.c_double,
                                  C.c_uint64, C.c_int, C.c_int, C.POINTER(Csr)]),
    "b40c_build_random": (C.c_int, [C.c_int64, C.c_int64, C.c_int, C.c_uint64, C.c_int, C.POINTER(Csr)]),
    "b40c_build_rr": (C.c_int, [C.c_int64, C.c_int32, C.c_int, C.c_uint64, C.c_int, C.POINTER(Csr)]),
    "b40c_coo_to_csr_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                         C.c_void_p]),
    "b40c_bfs_problem_create_coo": (C.c_int, [_P_i32, _P_i32, C.c_int64, C.c_int64, C.c_int, C.c_int,
                                              C.POINTER(C.c_void_p)]),
    "b40c_read_market": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.POINTER(Csr)]),
    "b40c_read_dimacs": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(Csr)]),
    "b40c_read_metis": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(Csr)]),
    "b40c_csr_from_coo": (C.c_int, [_P_i32, _P_i32, C.c_int64, C.c_int64, C.c_int, C.POINTER(Csr)]),
    "b40c_sample_sources": (C.c_int, [C.POINTER(Csr), C.c_int32, C.c_uint64, _P_i32]),
    "b40c_graph_free": (None, [C.POINTER(Csr)]),
    # include/b40c_server.h
    "b40c_server_create": (C.c_int, [C.c_int, C.POINTER(ServerOptions), C.POINTER(C.c_void_p)]),
    "b40c_server_destroy": (C.c_int, [C.c_void_p]),
    "b40c_server_add_graph": (C.c_int, [C.c_void_p, _P_i32, _P_i32, C.c_int64, C.c_int64, _P_i32]),
    "b40c_server_remove_graph": (C.c_int, [C.c_void_p, C.c_int32]),
    "b40c_server_graph_info": (C.c_int, [C.c_void_p, C.c_int32, _P_i64, _P_i32]),
    "b40c_server_set_graph_policy": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Policy), C.POINTER(Policy)]),
    "b40c_server_plan_bytes": (C.c_int, [C.c_int64, C.c_int64, C.c_int32, _P_i64]),
    "b40c_server_now_ns": (C.c_int, [C.c_void_p, _P_i64]),
    "b40c_server_submit": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int64, _P_i64]),
    "b40c_server_submit_many": (C.c_int, [C.c_void_p, C.c_int64, _P_i32, _P_i32, _P_i32, _P_i64, _P_i64]),
    "b40c_server_result_get": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(ServerResult)]),
    "b40c_server_wait": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(ServerResult)]),
    "b40c_server_drain": (C.c_int, [C.c_void_p]),
    "b40c_server_results": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p]),
    "b40c_server_counters_get": (C.c_int, [C.c_void_p, C.POINTER(ServerCounters)]),
}

_lib = None


def lib() -> C.CDLL:
    """Loads libb40c_bfs.so (built in-tree by back40computing_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m back40computing_b200.build` "
                "(the BFS path has no CPU fallback)")
        handle = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status: int, what: str = "") -> None:
    if status != SUCCESS:
        msg = lib().b40c_last_error_string().decode(errors="replace")
        raise B40cError(status, f"{what}: {msg}" if what else msg)


def i32p(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_P_i32)


def device_count() -> int:
    c = C.c_int32(0)
    check(lib().b40c_device_count(C.byref(c)), "b40c_device_count")
    return c.value
