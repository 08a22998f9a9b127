"""ctypes binding of the C ABI declared in include/gct_fdk.h.

The shared library is built in-tree (``gct_b200/libgct_fdk.so``). Loading never falls back to
another implementation: if the library is missing or stale, ``load()`` builds it with nvcc, and a
failure to build or load raises.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

from . import _build

GCT_OK = 0
GCT_ERR_NOT_READY = 7
STATUS_NAMES = {
    0: "GCT_OK", 1: "GCT_ERR_INVALID_ARG", 2: "GCT_ERR_OUT_OF_MEMORY", 3: "GCT_ERR_BUDGET",
    4: "GCT_ERR_TIMEOUT", 5: "GCT_ERR_CUDA", 6: "GCT_ERR_NOT_SUPPORTED", 7: "GCT_ERR_NOT_READY",
    8: "GCT_ERR_CANCELLED",
}


class GctError(RuntimeError):
    """Raised for a non-OK gct_status; mirrors the reference's std::runtime_error."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class gct_detector(C.Structure):
    _fields_ = [("num_samples", C.c_uint32), ("sampling_width", C.c_double)]


class gct_view_geom(C.Structure):
    _fields_ = [("rot_ang", C.c_double), ("det_row_center", C.c_double), ("det_col_center", C.c_double),
                ("src_det_dist", C.c_double), ("src_iso_dist", C.c_double),
                ("src_pos", C.c_double * 3), ("det_row_dir", C.c_double * 3),
                ("det_col_dir", C.c_double * 3), ("iso_ray_dir", C.c_double * 3)]


class gct_ct_geom(C.Structure):
    _fields_ = [("kind", C.c_int32), ("det_row", gct_detector), ("det_col", gct_detector),
                ("num_views", C.c_uint32), ("views", C.POINTER(gct_view_geom))]


class gct_vol_geom(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("mid", C.c_double * 3)]


class gct_filt_params(C.Structure):
    _fields_ = [("cut_off_freq", C.c_double), ("apod_func", C.c_int32)]


class gct_rotation_geom(C.Structure):
    _fields_ = [("dir", C.c_int32), ("rot_ang_incr", C.c_double), ("rot_ang_range", C.c_double),
                ("num_proj_per_rot", C.c_uint32)]


class gct_geom_params(C.Structure):
    _fields_ = [("det_row_center", C.c_double), ("det_col_center", C.c_double),
                ("src_det_dist", C.c_double), ("src_iso_dist", C.c_double), ("rot_dir", C.c_int32),
                ("init_ang", C.c_double), ("ang_incr", C.c_double), ("num_proj", C.c_uint32),
                ("hel_pitch", C.c_double)]


class gct_fdk_opts(C.Structure):
    _fields_ = [("filter", C.c_int32), ("storage", C.c_int32), ("z_per_thread", C.c_int32),
                ("block_x", C.c_int32), ("block_y", C.c_int32), ("symmetry", C.c_int32),
                ("scan", C.c_int32), ("reserved", C.c_int32 * 1)]


class gct_batch_item(C.Structure):
    _fields_ = [("plan", C.c_void_p), ("proj_dev", C.c_void_p), ("vol_dev", C.c_void_p)]


class gct_batch_opts(C.Structure):
    _fields_ = [("autotune", C.c_int32), ("use_graph", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("reserved", C.c_int32 * 5)]


class gct_batch_item_config(C.Structure):
    _fields_ = [("z_per_thread", C.c_int32), ("block_x", C.c_int32), ("block_y", C.c_int32),
                ("views_per_stage", C.c_int32), ("view_split", C.c_int32), ("tuned_gups", C.c_double)]


class gct_server_opts(C.Structure):
    _fields_ = [("memory_budget_bytes", C.c_uint64), ("max_active", C.c_uint32), ("autotune", C.c_uint32),
                ("round_updates", C.c_double), ("reserved", C.c_int32 * 4)]


class gct_request_info(C.Structure):
    _fields_ = [("state", C.c_int32), ("status", C.c_int32), ("queued_ms", C.c_double), ("latency_ms", C.c_double),
                ("rounds", C.c_uint32), ("views_per_round", C.c_uint32)]


class gct_server_stats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("cancelled", C.c_uint64), ("rejected", C.c_uint64), ("rounds", C.c_uint64),
                ("peak_bytes", C.c_uint64), ("peak_active", C.c_uint32), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("recons_per_s", C.c_double)]


class gct_proj_matrix(C.Structure):
    _fields_ = [("matrix", C.c_double * 12), ("intrinsic", C.c_double * 9), ("rotation", C.c_double * 9),
                ("src_pos", C.c_double * 3)]


class gct_array_metadata(C.Structure):
    _fields_ = [("num_rows", C.c_uint32), ("num_cols", C.c_uint32), ("num_slices", C.c_uint32), ("type", C.c_int32)]


class gct_ellipsoid(C.Structure):
    _fields_ = [("center", C.c_double * 3), ("semi_axes", C.c_double * 3), ("phi", C.c_double),
                ("mu", C.c_double)]


P = C.POINTER
VP = C.c_void_p

# name -> argtypes; every function returns gct_status (int32) unless listed in _RESTYPES
SIGNATURES = {
    "gct_abi_version": [],
    "gct_last_error_string": [],
    "gct_proj_geom_create": [C.c_int32, P(gct_geom_params), C.c_uint32, P(gct_view_geom)],
    "gct_proj_matrix_decompose": [P(C.c_double), P(gct_proj_matrix)],
    "gct_proj_matrix_compose": [P(gct_view_geom), C.c_double, C.c_double, P(gct_proj_matrix)],
    "gct_proj_geom_from_matrix": [P(C.c_double), P(gct_view_geom)],
    "gct_spiral_geom_check": [P(gct_ct_geom), P(C.c_uint32), P(C.c_double)],
    "gct_spiral_proj_indices": [P(gct_ct_geom), C.c_double, P(C.c_int64), P(C.c_int64)],
    "gct_rotation_geom_get": [P(gct_ct_geom), P(gct_rotation_geom), P(C.c_double), P(C.c_double)],
    "gct_is_valid_axial_recon": [P(gct_ct_geom), C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32,
                                 P(C.c_int32)],
    "gct_ramp_filter_taps": [C.c_int32, P(gct_detector), P(gct_filt_params), P(C.c_double)],
    "gct_parker_weights": [P(gct_ct_geom), P(C.c_float)],
    "gct_map_point": [P(gct_ct_geom), P(gct_vol_geom), C.c_uint32, P(C.c_double), P(C.c_double),
                      P(C.c_double), P(C.c_double), P(C.c_double)],
    "gct_fdk_plan_create": [P(gct_ct_geom), P(gct_vol_geom), P(gct_filt_params), P(gct_fdk_opts), P(VP)],
    "gct_fdk_plan_destroy": [VP],
    "gct_fdk_plan_check": [VP],
    "gct_fdk_plan_workspace_bytes": [VP, P(C.c_uint64)],
    "gct_fdk_plan_symmetry": [VP, P(C.c_int32)],
    "gct_fdk_plan_z_mirror": [VP, P(C.c_int32)],
    "gct_fdk_execute": [VP, VP, VP, VP, VP],
    "gct_fdk_filter": [VP, VP, VP, VP],
    "gct_fdk_prepare": [VP, VP, VP, C.c_uint32, C.c_uint32, VP],
    "gct_fdk_backproject": [VP, VP, VP, C.c_uint32, C.c_uint32, C.c_int32, VP],
    "gct_fdk_execute_host": [VP, P(C.c_float), P(C.c_float), VP],
    "gct_fdk_execute_noalloc": [VP, VP, VP, VP],
    "gct_fdk_execute_host_async": [VP, P(C.c_float), P(C.c_float), VP],
    "gct_fdk_host_sync": [VP],
    "gct_fdk_execute_host_budget": [VP, P(C.c_float), P(C.c_float), C.c_uint64, VP],
    "gct_reconstruct": [P(gct_ct_geom), P(gct_vol_geom), P(C.c_float), P(C.c_float)],
    "gct_reconstruct_ex": [P(gct_ct_geom), P(gct_vol_geom), P(gct_filt_params), P(gct_fdk_opts),
                           P(C.c_float), P(C.c_float)],
    "gct_fdk_batch_create": [P(gct_batch_item), C.c_uint32, P(gct_batch_opts), P(VP)],
    "gct_fdk_batch_launch": [VP, VP],
    "gct_fdk_batch_item_config": [VP, C.c_uint32, P(gct_batch_item_config)],
    "gct_fdk_batch_work": [VP, P(C.c_uint64), P(C.c_uint64)],
    "gct_fdk_batch_destroy": [VP],
    "gct_fdk_server_create": [P(gct_server_opts), P(VP)],
    "gct_fdk_server_submit": [VP, VP, P(C.c_float), P(C.c_float), P(C.c_uint64)],
    "gct_fdk_server_info": [VP, C.c_uint64, P(gct_request_info)],
    "gct_fdk_server_wait": [VP, C.c_uint64, C.c_double],
    "gct_fdk_server_cancel": [VP, C.c_uint64],
    "gct_fdk_server_stats": [VP, P(gct_server_stats)],
    "gct_fdk_server_destroy": [VP],
    "gct_phantom_project": [P(gct_ct_geom), P(gct_ellipsoid), C.c_uint32, VP, VP],
    "gct_forward_project": [P(gct_ct_geom), P(gct_vol_geom), VP, C.c_float, VP, VP],
    "gct_array_read_metadata": [C.c_char_p, C.c_int32, P(gct_array_metadata)],
    "gct_array_read": [C.c_char_p, C.c_int32, C.c_int32, P(gct_array_metadata), C.c_int32, VP, C.c_uint64,
                       P(C.c_uint64)],
    "gct_meta_image_write": [C.c_char_p, C.c_uint32, P(C.c_uint32), P(C.c_float), P(C.c_float), C.c_int32, VP,
                             C.c_uint64],
    "gct_den_write": [C.c_char_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32, VP, C.c_uint64],
    "gct_raw_write": [C.c_char_p, C.c_int32, VP, C.c_uint64],
}
_RESTYPES = {"gct_abi_version": C.c_int32, "gct_last_error_string": C.c_char_p}

_lib = None
_lock = threading.Lock()


def library_path() -> Path:
    return _build.LIB_PATH


def load() -> C.CDLL:
    """Load (building first if needed) the native library and bind every exported symbol."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = _build.build_library()
        lib = C.CDLL(str(path))
        for name, argtypes in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = _RESTYPES.get(name, C.c_int32)
        _lib = lib
        return lib


def check(status: int) -> None:
    if status != GCT_OK:
        msg = load().gct_last_error_string()
        raise GctError(status, msg.decode() if msg else "")
