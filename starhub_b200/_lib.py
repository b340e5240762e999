"""ctypes binding of libwarpsolve.so (the C ABI in include/warpsolve.h).

The shared library is loaded from the package directory only; there is no
fallback: if it is missing or does not load, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libwarpsolve.so"

WS_OK = 0
WS_ERR_INVALID_ARGUMENT = -1
WS_ERR_CAPACITY = -2
WS_ERR_CUDA = -3
WS_ERR_NAN = -4
WS_ERR_TIMEOUT = -5
WS_ERR_NOT_READY = -6
WS_ERR_NO_DEVICE = -7

WS_PREC_MIXED = 0
WS_PREC_FP32 = 1

WS_NOALLOC_MAX_PIXELS = 1280 * 720

# Every symbol include/warpsolve.h declares.
EXPORTED = [
    "ws_default_penalties", "ws_create", "ws_destroy", "ws_set_inputs", "ws_set_batch", "ws_solve",
    "ws_solve_graph", "ws_sync_status", "ws_get_solution", "ws_get_counts", "ws_get_dense_terms",
    "ws_get_node2term", "ws_get_node_pairs", "ws_get_system", "ws_get_dense_jacobian", "ws_init_nodes", "ws_expand_nodes",
    "ws_build_node_graph", "ws_skinning", "ws_forward_warp", "ws_splat_maps", "ws_measure_maps", "ws_version",
    "ws_error_string", "ws_set_profiling", "ws_get_phase_times", "ws_graph_kernel_count",
    "ws_splat_maps_noalloc", "ws_server_create", "ws_server_destroy", "ws_server_add_scene",
    "ws_server_remove_scene", "ws_submit", "ws_poll", "ws_wait", "ws_server_forget", "ws_server_get_warp",
    "ws_server_copy_warp", "ws_server_set_warp", "ws_server_get_stats", "ws_spmv", "ws_spmv_matrix_free", "ws_autotune",
    "ws_selftest_wait_timeout", "ws_selftest_grid_barrier_timeout", "ws_render_solver_maps",
    "ws_render_observation_maps",
    "ws_build_node_graph_ex", "ws_skinning_ex", "ws_skinning_incremental",
    "ws_set_tuning",
]


class WsRenderParams(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("fx", C.c_float), ("fy", C.c_float), ("cx", C.c_float),
                ("cy", C.c_float), ("world2camera", C.c_float * 16), ("max_depth", C.c_float),
                ("current_time", C.c_float), ("confidence_threshold", C.c_float), ("time_threshold", C.c_float),
                ("footprint", C.c_int)]


class WsConfig(C.Structure):
    _fields_ = [
        ("max_scenes", C.c_int), ("max_total_nodes", C.c_int), ("max_total_pixels", C.c_int),
        ("max_total_edges", C.c_int), ("max_total_features", C.c_int), ("precision", C.c_int),
        ("device", C.c_int),
    ]


class WsInputs(C.Structure):
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int), ("pitch", C.c_int),
        ("fx", C.c_float), ("fy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
        ("cam2world", C.c_float * 16),
        ("measure_vertex_confid", C.c_void_p), ("measure_normal_radius", C.c_void_p),
        ("reference_vertex", C.c_void_p), ("reference_normal", C.c_void_p),
        ("index_map", C.c_void_p), ("opticalflow", C.c_void_p),
        ("num_surfels", C.c_int), ("surfel_knn", C.c_void_p),
        ("surfel_knn_spatial_weight", C.c_void_p), ("surfel_knn_connect_weight", C.c_void_p),
        ("num_nodes", C.c_int), ("reference_node_coords", C.c_void_p),
        ("num_edges", C.c_int), ("node_graph", C.c_void_p), ("graph_k", C.c_int),
        ("node_knn_connect_weight", C.c_void_p), ("node_radius_square", C.c_float),
        ("node_motion_pred", C.c_void_p),
        ("num_features", C.c_int), ("feature_knn", C.c_void_p),
        ("lambda_depth", C.c_float), ("lambda_optical_flow", C.c_float), ("lambda_reg", C.c_float),
        ("lambda_node_translation", C.c_float), ("lambda_feature", C.c_float),
        ("init_node_se3", C.c_void_p),
    ]


class WsServerConfig(C.Structure):
    _fields_ = [
        ("device", C.c_int), ("memory_budget", C.c_ulonglong), ("executors", C.c_int),
        ("max_batch_scenes", C.c_int), ("max_batch_nodes", C.c_int), ("max_batch_pixels", C.c_int),
        ("max_batch_edges", C.c_int), ("gn_iters", C.c_int), ("pcg_iters", C.c_int), ("precision", C.c_int),
    ]


class WsFrame(C.Structure):
    _fields_ = [
        ("measure_vertex_confid", C.c_void_p), ("measure_normal_radius", C.c_void_p),
        ("reference_vertex", C.c_void_p), ("reference_normal", C.c_void_p), ("index_map", C.c_void_p),
        ("opticalflow", C.c_void_p), ("pitch", C.c_int), ("cam2world", C.c_float * 16),
        ("node_motion_pred", C.c_void_p), ("solution_out", C.c_void_p),
    ]


class WsRequestInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int), ("scene", C.c_int), ("num_nodes", C.c_int), ("batch_scenes", C.c_int),
        ("queue_ms", C.c_double), ("solve_ms", C.c_double), ("latency_ms", C.c_double),
    ]


class WsServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_ulonglong), ("completed", C.c_ulonglong), ("failed", C.c_ulonglong),
        ("batches", C.c_ulonglong), ("mean_batch_scenes", C.c_double), ("p50_latency_ms", C.c_double),
        ("p99_latency_ms", C.c_double), ("mean_latency_ms", C.c_double), ("executor_bytes", C.c_ulonglong),
        ("resident_bytes", C.c_ulonglong), ("memory_budget", C.c_ulonglong), ("scenes", C.c_int),
    ]


class WsTuning(C.Structure):
    _fields_ = [
        ("node_threads", C.c_int), ("pair_threads", C.c_int), ("pcg_blocks_per_sm", C.c_int),
        ("node_ms", C.c_float * 3), ("pair_ms", C.c_float * 3), ("pcg_ms", C.c_float * 8),
    ]


class WarpSolveError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = error_string(status) if _lib is not None else str(status)
        super().__init__(f"{what}: {msg} (status {status})" if what else f"{msg} (status {status})")


_lib = None


def load() -> C.CDLL:
    """Loads libwarpsolve.so from the package directory (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: run `python -m starhub_b200.build` (nvcc, sm_100a)")
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | getattr(os, "RTLD_GLOBAL", 0))
    vp, i, f = C.c_void_p, C.c_int, C.c_float
    pi = C.POINTER(C.c_int)
    u = C.c_uint
    sig = {
        "ws_default_penalties": (None, [C.POINTER(WsInputs)]),
        "ws_create": (i, [C.POINTER(WsConfig), C.POINTER(vp)]),
        "ws_destroy": (i, [vp]),
        "ws_set_inputs": (i, [vp, C.POINTER(WsInputs)]),
        "ws_set_batch": (i, [vp, C.POINTER(WsInputs), i]),
        "ws_solve": (i, [vp, i, i, vp]),
        "ws_solve_graph": (i, [vp, i, i, vp]),
        "ws_sync_status": (i, [vp]),
        "ws_get_solution": (i, [vp, i, C.POINTER(vp), pi]),
        "ws_get_counts": (i, [vp, i, pi, pi, pi]),
        "ws_get_dense_terms": (i, [vp, i, vp, vp, vp, vp, i, pi]),
        "ws_get_node2term": (i, [vp, i, vp, vp, i, pi]),
        "ws_get_node_pairs": (i, [vp, i, vp, vp, vp, vp, i, pi, vp, i, pi]),
        "ws_get_system": (i, [vp, i, vp, vp, vp, i, pi, vp, vp, vp]),
        "ws_get_dense_jacobian": (i, [vp, i, vp, vp, i, pi]),
        "ws_init_nodes": (i, [vp, i, f, vp, i, pi, vp]),
        "ws_expand_nodes": (i, [vp, i, f, vp, vp, vp, u, i, pi, vp]),
        "ws_build_node_graph": (i, [vp, i, i, f, vp, vp, vp, vp]),
        "ws_skinning": (i, [vp, i, vp, i, f, vp, vp, vp, vp]),
        "ws_forward_warp": (i, [vp, i, vp, vp, i, vp, vp, vp, vp, vp, vp]),
        "ws_measure_maps": (i, [vp, i, i, i, f, f, f, f, f, f, f, vp, vp, vp]),
        "ws_splat_maps": (i, [vp, vp, vp, i, i, i, f, f, f, f, i, vp, vp, vp, vp]),
        "ws_splat_maps_noalloc": (i, [vp, vp, vp, i, i, i, f, f, f, f, i, vp, vp, vp, vp]),
        "ws_version": (i, []),
        "ws_error_string": (C.c_char_p, [i]),
        "ws_set_profiling": (i, [vp, i]),
        "ws_get_phase_times": (i, [vp, vp, vp, i, pi]),
        "ws_graph_kernel_count": (i, [vp, pi]),
        "ws_server_create": (i, [C.POINTER(WsServerConfig), C.POINTER(vp)]),
        "ws_server_destroy": (i, [vp]),
        "ws_server_add_scene": (i, [vp, C.POINTER(WsInputs), pi]),
        "ws_server_remove_scene": (i, [vp, i]),
        "ws_submit": (i, [vp, i, C.POINTER(WsFrame), C.POINTER(C.c_ulonglong)]),
        "ws_poll": (i, [vp, C.c_ulonglong, C.POINTER(WsRequestInfo)]),
        "ws_wait": (i, [vp, C.c_ulonglong, C.POINTER(WsRequestInfo)]),
        "ws_server_forget": (i, [vp, C.c_ulonglong]),
        "ws_server_get_warp": (i, [vp, i, C.POINTER(vp), pi]),
        "ws_server_copy_warp": (i, [vp, i, vp]),
        "ws_server_set_warp": (i, [vp, i, vp]),
        "ws_server_get_stats": (i, [vp, C.POINTER(WsServerStats)]),
        "ws_spmv": (i, [vp, vp, vp, vp]),
        "ws_spmv_matrix_free": (i, [vp, vp, vp, vp]),
        "ws_selftest_wait_timeout": (i, [vp]),
        "ws_selftest_grid_barrier_timeout": (i, [vp]),
        "ws_render_solver_maps": (i, [vp, vp, vp, i, C.POINTER(WsRenderParams), vp, vp, vp, vp, vp]),
        "ws_render_observation_maps": (i, [vp, vp, vp, i, C.POINTER(WsRenderParams), vp, vp, vp]),
        "ws_build_node_graph_ex": (i, [vp, vp, i, i, f, i, vp, vp, vp, vp]),
        "ws_skinning_ex": (i, [vp, vp, i, vp, i, f, i, vp, vp, vp, vp]),
        "ws_skinning_incremental": (i, [vp, vp, i, i, vp, i, i, f, i, vp, vp, vp, vp]),
        "ws_autotune": (i, [vp, i, vp, C.POINTER(WsTuning)]),
        "ws_set_tuning": (i, [vp, C.POINTER(WsTuning)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def error_string(status: int) -> str:
    return load().ws_error_string(int(status)).decode()


def check(status: int, what: str = "") -> None:
    if status != WS_OK:
        raise WarpSolveError(status, what)
