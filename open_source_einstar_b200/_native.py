"""ctypes binding of include/depth_cuda.h (libdepth_cuda.so). No torch types cross the boundary.

The library is the product path. There is no fallback: if it is missing or cannot be loaded, import
of the stereo classes raises.
"""
from __future__ import annotations

import ctypes as C
import os

from .build import LIB


class SgmParamsC(C.Structure):
    _fields_ = [
        ("min_disparity", C.c_int), ("num_disparities", C.c_int),
        ("census_radius_x", C.c_int), ("census_radius_y", C.c_int),
        ("p1", C.c_int), ("p2", C.c_int), ("adaptive_p2", C.c_int),
        ("eight_paths", C.c_int), ("slant_steps", C.c_int),
        ("uniqueness", C.c_float), ("lr_max_diff", C.c_int),
    ]


class StereoParamsC(C.Structure):
    _fields_ = [
        ("pyramid_levels", C.c_int), ("sgm", SgmParamsC), ("subpixel", C.c_int), ("median", C.c_int),
        ("detail_enabled", C.c_int), ("filter_occlusion", C.c_int), ("filter_spikes", C.c_int),
        ("speckle_max_region_size", C.c_int), ("wide_costs", C.c_int),
        ("refine_search_radius", C.c_int), ("refine_zncc_radius", C.c_int), ("refine_min_zncc", C.c_float),
        ("refine_reject_edge_winners", C.c_int), ("detail_radius", C.c_int), ("detail_search", C.c_float),
        ("detail_step", C.c_float), ("detail_min_zncc", C.c_float), ("occlusion_tolerance", C.c_float),
        ("spike_threshold", C.c_float), ("speckle_max_diff", C.c_float),
    ]


class GeometryC(C.Structure):
    _fields_ = [("f", C.c_double), ("cx", C.c_double), ("cy", C.c_double), ("baseline", C.c_double),
                ("cx_offset", C.c_double)]


class TimingsC(C.Structure):
    _fields_ = [("gpu_ms", C.c_double), ("speckle_ms", C.c_double), ("total_ms", C.c_double)]


class OutputsC(C.Structure):
    _fields_ = [("disparity", C.c_void_p), ("confidence", C.c_void_p), ("disparity_u16", C.c_void_p),
                ("depth", C.c_void_p), ("rect_left", C.c_void_p), ("rect_right", C.c_void_p)]


class KernelConfigC(C.Structure):
    _fields_ = [("regs_per_lane", C.c_int), ("lanes_per_line", C.c_int), ("materialize_costs", C.c_int),
                ("path_warps_per_block", C.c_int), ("wta_threads", C.c_int), ("prefetch_steps", C.c_int),
                ("fused_pairs", C.c_int), ("horz_warps_per_block", C.c_int)]


class PairDescC(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("params", StereoParamsC), ("raw", C.c_int), ("calib", C.c_int),
                ("have_geometry", C.c_int), ("geometry", GeometryC), ("min_depth_mm", C.c_float),
                ("max_depth_mm", C.c_float), ("kernel", KernelConfigC)]


class BatchOptionsC(C.Structure):
    _fields_ = [("micro_batch", C.c_int), ("branches", C.c_int)]


class PointParamsC(C.Structure):
    _fields_ = [("min_depth_mm", C.c_float), ("max_depth_mm", C.c_float), ("max_depth_jump_mm", C.c_float),
                ("edge_weight", C.c_float), ("weight_reference_depth_mm", C.c_float)]


class BlobParamsC(C.Structure):
    _fields_ = [("threshold", C.c_uint32), ("min_diameter", C.c_uint32), ("max_diameter", C.c_uint32),
                ("max_aspect", C.c_float), ("min_fill", C.c_float), ("border", C.c_uint32), ("max_axis_ratio", C.c_float),
                ("ring_scale", C.c_float), ("ring_contrast", C.c_float), ("ring_max_bright", C.c_float),
                ("max_blobs", C.c_uint32)]


class BlobBoxesC(C.Structure):
    _fields_ = [("left", C.c_void_p), ("right", C.c_void_p), ("capacity", C.c_uint32), ("found", C.c_uint32 * 2),
                ("kept", C.c_uint32 * 2)]


BLOB_CALLBACK = C.CFUNCTYPE(None, C.POINTER(BlobBoxesC), C.c_void_p)


class FrameRequestC(C.Structure):
    _fields_ = [("marker_blobs", C.c_int), ("on_blobs", BLOB_CALLBACK), ("user", C.c_void_p)]


class FrameOutputsC(C.Structure):
    _fields_ = [("points_xyzw", C.c_void_p), ("normals_xyzw", C.c_void_p), ("weights", C.c_void_p), ("host", OutputsC),
                ("blobs", C.POINTER(BlobBoxesC))]


class ServerOptionsC(C.Structure):
    _fields_ = [("volume_budget_bytes", C.c_size_t), ("max_slots", C.c_int), ("max_pending", C.c_int)]


class RequestC(C.Structure):
    _fields_ = [("calib", C.c_int), ("width", C.c_int), ("height", C.c_int), ("params", StereoParamsC),
                ("left", C.c_void_p), ("right", C.c_void_p), ("stride", C.c_ssize_t), ("out", OutputsC),
                ("tag", C.c_uint64)]


class CompletionC(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("tag", C.c_uint64), ("status", C.c_int), ("queue_ms", C.c_double),
                ("gpu_ms", C.c_double), ("latency_ms", C.c_double)]


class ServerStatsC(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("pending", C.c_int), ("running", C.c_int), ("peak_running", C.c_int), ("slots", C.c_int),
                ("running_volume_bytes", C.c_size_t), ("peak_running_volume_bytes", C.c_size_t),
                ("volume_bytes", C.c_size_t), ("device_bytes", C.c_size_t)]


# Every symbol include/depth_cuda.h declares: name -> (restype, argtypes).
_vp, _i, _f, _sz = C.c_void_p, C.c_int, C.c_float, C.c_size_t
SIGNATURES = {
    "ds_default_params": (None, [C.POINTER(StereoParamsC)]),
    "ds_create": (_i, [C.POINTER(StereoParamsC), _i, _i, C.POINTER(_vp)]),
    "ds_destroy": (None, [_vp]),
    "ds_set_rectification": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _i]),
    "ds_set_point_params": (_i, [_vp, C.POINTER(GeometryC), _f, _f, _f]),
    "ds_compute": (_i, [_vp, _vp, _vp, C.c_ssize_t, C.POINTER(OutputsC)]),
    "ds_compute_raw": (_i, [_vp, _vp, _vp, C.c_ssize_t, C.POINTER(OutputsC)]),
    "ds_compute_device": (_i, [_vp, _vp, _vp, C.POINTER(OutputsC), _vp]),
    "ds_compute_raw_device": (_i, [_vp, _vp, _vp, C.POINTER(OutputsC), _vp]),
    "ds_last_timings": (_i, [_vp, C.POINTER(TimingsC)]),
    "ds_last_error": (C.c_char_p, [_vp]),
    "ds_last_global_error": (C.c_char_p, []),
    "ds_debug_read": (_i, [_vp, _vp, _vp, _vp]),
    "ds_device_bytes": (_sz, [_vp]),
    "ds_profile_enable": (_i, [_vp, _i]),
    "ds_profile_collect": (_i, [_vp, _vp, _i, C.POINTER(_i)]),
    "ds_kernel_launches": (C.c_uint64, []),
    "ds_set_kernel_config": (_i, [_vp, C.POINTER(KernelConfigC)]),
    "ds_get_kernel_config": (_i, [_vp, C.POINTER(KernelConfigC)]),
    "ds_batch_create": (_i, [C.POINTER(PairDescC), _i, _i, C.POINTER(BatchOptionsC), C.POINTER(_vp)]),
    "ds_batch_destroy": (None, [_vp]),
    "ds_batch_last_error": (C.c_char_p, [_vp]),
    "ds_batch_set_rectification": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _i, _i, _i, _i]),
    "ds_batch_bind": (_i, [_vp, _i, _vp, _vp, C.POINTER(OutputsC)]),
    "ds_batch_run": (_i, [_vp, _vp]),
    "ds_batch_run_eager": (_i, [_vp, _vp]),
    "ds_batch_device_bytes": (_sz, [_vp]),
    "ds_batch_launches_per_run": (_i, [_vp]),
    "ds_batch_get_options": (_i, [_vp, C.POINTER(BatchOptionsC)]),
    "ds_batch_profile": (_i, [_vp, _i]),
    "ds_batch_stage_ms": (_i, [_vp, _vp]),
    "ds_default_point_params": (None, [C.POINTER(PointParamsC)]),
    "ds_disparity_to_points": (_i, [_vp, _vp, _i, _i, C.POINTER(GeometryC), C.POINTER(PointParamsC), _vp, _vp, _vp, _vp]),
    "ds_pack_depth": (_i, [_vp, _vp, _i, _i, _vp, _vp]),
    "ds_undelta_rows": (_i, [_vp, C.c_ssize_t, _vp, C.c_ssize_t, _i, _i, _vp]),
    "ds_default_blob_params": (None, [C.POINTER(BlobParamsC)]),
    "ds_set_blob_params": (_i, [_vp, C.POINTER(BlobParamsC)]),
    "ds_compute_raw_blobs": (_i, [_vp, _vp, _vp, C.c_ssize_t, C.POINTER(OutputsC), C.POINTER(BlobBoxesC)]),
    "ds_compute_frame": (_i, [_vp, _vp, _vp, C.c_ssize_t, C.POINTER(FrameRequestC), C.POINTER(FrameOutputsC)]),
    "ds_compute_frame_raw": (_i, [_vp, _vp, _vp, C.c_ssize_t, _vp, _vp, _vp, _vp, _vp]),
    "ds_find_blobs": (_i, [_vp, _vp, _i, _i, C.c_ssize_t, _vp, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "ds_server_create": (_i, [C.POINTER(ServerOptionsC), C.POINTER(_vp)]),
    "ds_server_destroy": (None, [_vp]),
    "ds_server_last_error": (C.c_char_p, [_vp]),
    "ds_server_add_calibration": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _i, _i, _i, _i, C.POINTER(GeometryC), _f, _f]),
    "ds_server_reserve": (_i, [_vp, _i, _i, C.POINTER(StereoParamsC), _i, _i]),
    "ds_server_submit": (_i, [_vp, C.POINTER(RequestC), C.POINTER(C.c_uint64)]),
    "ds_server_poll": (_i, [_vp, C.POINTER(CompletionC), _i, C.POINTER(_i), _i]),
    "ds_server_get_stats": (_i, [_vp, C.POINTER(ServerStatsC)]),
    "ds_sgm_disparity_noalloc": (_i, [_vp, _vp, _i, _i, C.POINTER(SgmParamsC), _i, _vp, _vp]),
}

_lib = None


def lib() -> C.CDLL:
    """Loads libdepth_cuda.so (in-tree); raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise ImportError(f"{LIB} is not built: run open_source_einstar_b200.build.build_native() "
                              "(or __graft_entry__.build()); there is no CPU fallback")
        L = C.CDLL(LIB)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib
