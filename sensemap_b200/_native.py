"""ctypes binding of the engine's C ABI (include/smvs.h).

Loads ``sensemap_b200/libsmvs.so`` (built in-tree by ``sensemap_b200.build``).
There is no fallback: if the library is missing or does not load, every entry
point raises ``NativeLibraryError``.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

SMVS_MAX_SRC = 32
SMVS_POSE_FLOATS = 43
SMVS_CROSS_MAX_SRC = 31

SMVS_OK, SMVS_EINVAL, SMVS_ENOMEM, SMVS_ECUDA, SMVS_ESTATE, SMVS_EIO, SMVS_ETIMEDOUT, SMVS_ECANCELED = range(8)
PIX_U8, PIX_F32 = 0, 1
STORE_U8, STORE_F16, STORE_F32 = 0, 1, 2
MEM_HOST, MEM_DEVICE = 0, 1
(KERNEL_CONVERT, KERNEL_PREP, KERNEL_INIT, KERNEL_INIT_CONF, KERNEL_SWEEP, KERNEL_LOCAL_OPT, KERNEL_MASK,
 KERNEL_FILTER, KERNEL_POST) = range(9)
KERNEL_NAMES = ["convert", "prep_ref", "init", "init_conf", "sweep", "local_opt", "mask", "filter", "post"]
JOB_QUEUED, JOB_ACTIVE, JOB_DONE, JOB_FAILED = range(4)
MAP_DEPTH, MAP_NORMAL, MAP_CONF, MAP_COST, MAP_VIEW_SEL = range(5)
CF_KERNEL_RUN, CF_KERNEL_DEDUP, CF_KERNEL_OTHER = range(3)
CF_KERNEL_NAMES = ["cross_filter", "dedup", "other"]
FUSION_KERNEL_CLOSURE, FUSION_KERNEL_ORDER, FUSION_KERNEL_REPLAY, FUSION_KERNEL_OTHER = range(4)
FUSION_KERNEL_NAMES = ["closure", "order", "replay", "other"]

STATUS_NAMES = {0: "SMVS_OK", 1: "SMVS_EINVAL", 2: "SMVS_ENOMEM", 3: "SMVS_ECUDA", 4: "SMVS_ESTATE",
                5: "SMVS_EIO", 6: "SMVS_ETIMEDOUT", 7: "SMVS_ECANCELED"}


class NativeLibraryError(RuntimeError):
    pass


class SmvsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class smvs_options(C.Structure):
    _fields_ = [
        ("depth_min", C.c_double), ("depth_max", C.c_double),
        ("window_radius", C.c_int), ("window_step", C.c_int),
        ("sigma_spatial", C.c_double), ("sigma_color", C.c_double),
        ("num_samples", C.c_int), ("num_iterations", C.c_int),
        ("geom_consistency", C.c_int),
        ("geom_consistency_regularizer", C.c_double), ("geom_consistency_max_cost", C.c_double),
        ("filter", C.c_int), ("filter_min_num_consistent", C.c_int),
        ("filter_geom_consistency_max_cost", C.c_double),
        ("max_normal_error", C.c_double),
        ("init_depth_random", C.c_int),
        ("random_depth_ratio", C.c_float), ("random_angle1_range", C.c_float), ("random_angle2_range", C.c_float),
        ("init_ncc_matching_cost", C.c_double), ("max_ncc_matching_cost", C.c_double),
        ("alpha", C.c_double), ("beta", C.c_double),
        ("thk", C.c_int), ("num_good_hypothesis", C.c_int), ("num_bad_hypothesis", C.c_int),
        ("random_optimization", C.c_int), ("local_optimization", C.c_int),
        ("est_curvature", C.c_int), ("median_filter", C.c_int), ("conf_filter", C.c_int),
        ("depth_diff_threshold", C.c_float), ("conf_threshold", C.c_float),
        ("has_prior_depth", C.c_int), ("propagate_depth", C.c_int),
        ("random_seed", C.c_uint64), ("image_storage", C.c_int), ("gpu_index", C.c_int),
    ]


class smvs_view(C.Structure):
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int), ("pixel_format", C.c_int),
        ("row_stride", C.c_size_t), ("pixels", C.c_void_p),
        ("K", C.c_float * 9), ("R", C.c_float * 9), ("T", C.c_float * 3),
        ("scale", C.c_float),
        ("depth", C.c_void_p), ("normal", C.c_void_p),
    ]


class smvs_problem(C.Structure):
    _fields_ = [
        ("ref", smvs_view), ("src", C.POINTER(smvs_view)), ("num_src", C.c_int),
        ("ref_mask", C.c_void_p), ("memory", C.c_int), ("ref_prior_wgt", C.c_void_p),
    ]


class smvs_tuning(C.Structure):
    _fields_ = [("sweep_block_x", C.c_int), ("ref_tile_tma", C.c_int), ("threads_per_pixel", C.c_int),
                ("persistent", C.c_int)]


class smvs_pool_options(C.Structure):
    _fields_ = [("memory_budget_bytes", C.c_size_t), ("max_active_jobs", C.c_int), ("image_storage", C.c_int),
                ("sweep_block_x", C.c_int), ("use_graphs", C.c_int), ("gpu_index", C.c_int),
                ("ref_tile_tma", C.c_int), ("sweep_threads_per_pixel", C.c_int), ("sweep_persistent", C.c_int)]


class smvs_pool_stats(C.Structure):
    _fields_ = [("queued", C.c_int), ("active", C.c_int), ("done", C.c_int), ("bytes_used", C.c_size_t),
                ("bytes_budget", C.c_size_t), ("views_resident", C.c_int), ("launches", C.c_int64),
                ("graphs_built", C.c_int64), ("evictions", C.c_int64), ("steps", C.c_int64)]


class smvs_device_maps(C.Structure):
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int), ("num_src", C.c_int),
        ("depth", C.c_void_p), ("normal", C.c_void_p), ("conf", C.c_void_p),
        ("cost", C.c_void_p), ("view_sel", C.c_void_p),
    ]


class smvs_filter_view(C.Structure):
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int),
        ("K", C.c_float * 9), ("R", C.c_float * 9), ("T", C.c_float * 3),
        ("depth", C.c_void_p), ("normal", C.c_void_p), ("ref_flag", C.c_int),
    ]


class smvs_filter_problem(C.Structure):
    _fields_ = [("ref", C.c_int), ("src", C.POINTER(C.c_int)), ("num_src", C.c_int)]


class smvs_model_image(C.Structure):
    _fields_ = [("R", C.c_float * 9), ("T", C.c_float * 3), ("is_rig", C.c_int)]


class smvs_fusion_options(C.Structure):
    _fields_ = [
        ("step_size", C.c_int), ("min_num_pixels", C.c_int), ("max_num_pixels", C.c_int),
        ("min_num_visible_images", C.c_int), ("max_traversal_depth", C.c_int),
        ("max_reproj_error", C.c_double), ("max_depth_error", C.c_double), ("max_normal_error", C.c_double),
        ("with_normal", C.c_int), ("num_slices", C.c_int), ("gpu_index", C.c_int),
    ]


class smvs_fusion_view(C.Structure):
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int),
        ("K", C.c_float * 9), ("R", C.c_float * 9), ("T", C.c_float * 3),
        ("depth", C.c_void_p), ("normal", C.c_void_p), ("color", C.c_void_p), ("is_rig", C.c_int),
    ]


class smvs_fused_point(C.Structure):
    _fields_ = [
        ("x", C.c_float), ("y", C.c_float), ("z", C.c_float),
        ("nx", C.c_float), ("ny", C.c_float), ("nz", C.c_float),
        ("r", C.c_uint8), ("g", C.c_uint8), ("b", C.c_uint8), ("pad", C.c_uint8),
        ("score", C.c_float),
    ]


# numpy view of smvs_fused_point
FUSED_POINT_DTYPE = [("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("nx", "<f4"), ("ny", "<f4"), ("nz", "<f4"),
                     ("r", "u1"), ("g", "u1"), ("b", "u1"), ("pad", "u1"), ("score", "<f4")]


# name -> (restype, argtypes)
_SIGNATURES = {
    "smvs_options_default": (C.c_int, [C.POINTER(smvs_options)]),
    "smvs_options_check": (C.c_int, [C.POINTER(smvs_options)]),
    "smvs_create": (C.c_int, [C.POINTER(smvs_options), C.POINTER(smvs_problem), C.c_void_p, C.POINTER(C.c_void_p)]),
    "smvs_run": (C.c_int, [C.c_void_p]),
    "smvs_run_filter": (C.c_int, [C.c_void_p, C.c_int]),
    "smvs_get_depth_map": (C.c_int, [C.c_void_p, C.c_void_p]),
    "smvs_get_normal_map": (C.c_int, [C.c_void_p, C.c_void_p]),
    "smvs_get_conf_map": (C.c_int, [C.c_void_p, C.c_void_p]),
    "smvs_get_cost_map": (C.c_int, [C.c_void_p, C.c_void_p]),
    "smvs_get_view_sel_map": (C.c_int, [C.c_void_p, C.c_void_p]),
    "smvs_get_curvature_map": (C.c_int, [C.c_void_p, C.c_void_p]),
    "smvs_get_size": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "smvs_get_device_maps": (C.c_int, [C.c_void_p, C.POINTER(smvs_device_maps)]),
    "smvs_synchronize": (C.c_int, [C.c_void_p]),
    "smvs_launch_count": (C.c_int64, [C.c_void_p]),
    "smvs_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "smvs_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(smvs_tuning)]),
    "smvs_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(smvs_tuning)]),
    "smvs_autotune": (C.c_int, [C.POINTER(smvs_options), C.POINTER(smvs_problem), C.c_void_p, C.c_int,
                                C.POINTER(smvs_tuning), C.POINTER(smvs_tuning), C.POINTER(C.c_double), C.c_int,
                                C.POINTER(C.c_int)]),
    "smvs_get_profile": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "smvs_destroy": (None, [C.c_void_p]),
    "smvs_last_error": (C.c_char_p, []),
    "smvs_write_mat_f32": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "smvs_write_mat_u32": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "smvs_write_mat_u16": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "smvs_read_mat": (C.c_int, [C.c_char_p, C.c_void_p, C.c_size_t, C.c_int, C.POINTER(C.c_int),
                                C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "smvs_encode_normal_map": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "smvs_decode_normal_map": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "smvs_write_maps": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p]),
    "smvs_cross_filter_create": (C.c_int, [C.POINTER(smvs_options), C.POINTER(smvs_filter_view), C.c_int,
                                           C.POINTER(smvs_filter_problem), C.c_int, C.c_int, C.c_void_p,
                                           C.POINTER(C.c_void_p)]),
    "smvs_cross_filter_run": (C.c_int, [C.c_void_p]),
    "smvs_cross_filter_dedup_run": (C.c_int, [C.c_void_p]),
    "smvs_cross_filter_get_refined_depth_map": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "smvs_cross_filter_get_dedup_depth_map": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "smvs_cross_filter_get_delta_depth_map": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "smvs_cross_filter_get_visibility_map": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "smvs_cross_filter_get_device_maps": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p),
                                                    C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "smvs_cross_filter_launch_count": (C.c_int64, [C.c_void_p]),
    "smvs_cross_filter_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "smvs_cross_filter_get_profile": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "smvs_cross_filter_dedup_levels": (C.c_int, [C.c_void_p]),
    "smvs_cross_filter_synchronize": (C.c_int, [C.c_void_p]),
    "smvs_cross_filter_destroy": (None, [C.c_void_p]),
    "smvs_cross_filter_release_cache": (C.c_int, [C.c_int]),
    "smvs_init_depth_from_sparse_points": (C.c_int, [C.POINTER(smvs_view), C.c_void_p, C.c_size_t, C.c_int,
                                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "smvs_init_depth_from_delaunay": (C.c_int, [C.POINTER(smvs_view), C.c_void_p, C.c_size_t, C.c_int,
                                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "smvs_init_depth_from_mesh": (C.c_int, [C.POINTER(smvs_view), C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                            C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "smvs_init_depth_from_dense_points": (C.c_int, [C.POINTER(smvs_view), C.c_void_p, C.c_void_p, C.c_size_t, C.c_int,
                                                    C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "smvs_select_views": (C.c_int, [C.POINTER(smvs_model_image), C.c_int, C.c_void_p, C.c_size_t, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p]),
    "smvs_compute_depth_ranges": (C.c_int, [C.POINTER(smvs_model_image), C.c_int, C.c_void_p, C.c_void_p,
                                            C.c_void_p]),
    "smvs_fusion_options_default": (C.c_int, [C.POINTER(smvs_fusion_options)]),
    "smvs_fusion_create": (C.c_int, [C.POINTER(smvs_fusion_options), C.POINTER(smvs_fusion_view), C.c_int,
                                     C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "smvs_fusion_run": (C.c_int, [C.c_void_p]),
    "smvs_fusion_get_sizes": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "smvs_fusion_get_points": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "smvs_fusion_get_device_points": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                                C.POINTER(C.c_void_p)]),
    "smvs_fusion_get_image_order": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]),
    "smvs_fusion_remove_duplicate_points": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "smvs_fusion_remove_outliers": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_size_t)]),
    "smvs_fusion_get_mask": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "smvs_fusion_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "smvs_fusion_get_profile": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "smvs_fusion_launch_count": (C.c_int64, [C.c_void_p]),
    "smvs_fusion_destroy": (None, [C.c_void_p]),
    "smvs_pool_options_default": (C.c_int, [C.POINTER(smvs_pool_options)]),
    "smvs_pool_create": (C.c_int, [C.POINTER(smvs_pool_options), C.c_void_p, C.POINTER(C.c_void_p)]),
    "smvs_pool_add_view": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(smvs_view), C.c_int]),
    "smvs_pool_has_view": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_int)]),
    "smvs_pool_set_view_maps": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int]),
    "smvs_pool_submit": (C.c_int, [C.c_void_p, C.POINTER(smvs_options), C.c_int64, C.POINTER(C.c_int64), C.c_int,
                                   C.POINTER(C.c_int64)]),
    "smvs_pool_step": (C.c_int, [C.c_void_p, C.POINTER(smvs_pool_stats)]),
    "smvs_pool_job_state": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "smvs_pool_wait": (C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.POINTER(C.c_int)]),
    "smvs_pool_get_map": (C.c_int, [C.c_void_p, C.c_int64, C.c_int, C.c_void_p]),
    "smvs_pool_keep_maps": (C.c_int, [C.c_void_p, C.c_int64]),
    "smvs_pool_release": (C.c_int, [C.c_void_p, C.c_int64]),
    "smvs_pool_stats_get": (C.c_int, [C.c_void_p, C.POINTER(smvs_pool_stats)]),
    "smvs_pool_destroy": (None, [C.c_void_p]),
    "smvs_filter_depth_map_noalloc": (C.c_int, [C.POINTER(smvs_options), C.POINTER(smvs_problem), C.c_void_p,
                                                C.c_int, C.c_void_p]),
    # include/smvs_testing.h
    "smvs_test_sample_texture": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                           C.c_void_p]),
    "smvs_test_calibrate": (C.c_int, [C.c_int, C.c_double, C.POINTER(C.c_double)]),
    "smvs_test_take_cuda_error": (C.c_int, []),
    "smvs_test_fusion_waits": (C.c_int, [C.c_double, C.c_longlong]),
    "smvs_test_tile_waits": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "smvs_test_persistent_grid": (C.c_int, [C.c_int]),
    "smvs_test_propagate_init": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "smvs_test_delaunay": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "smvs_pyramid_level_size": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                          C.POINTER(C.c_float)]),
    "smvs_rescale_image": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                     C.c_void_p]),
    "smvs_resample_maps": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                     C.c_int, C.c_void_p]),
    "smvs_synth_render_aerial": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_uint32, C.c_float,
                                           C.c_float, C.c_float, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                           C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "smvs_test_fusion_caps": (C.c_int, [C.c_int, C.c_int, C.c_int]),
    "smvs_test_fusion_chains": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "smvs_test_fusion_image_ms": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "smvs_test_fusion_replay_times": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
}

_LIB = None


def library_path() -> Path:
    return Path(os.environ.get("SMVS_LIBRARY", Path(__file__).resolve().parent / "libsmvs.so"))


def lib():
    """The loaded engine library (raises NativeLibraryError if absent)."""
    global _LIB
    if _LIB is None:
        path = library_path()
        if not path.exists():
            raise NativeLibraryError(f"{path} is missing: build it with sensemap_b200.build.build()")
        try:
            handle = C.CDLL(str(path))
        except OSError as exc:
            raise NativeLibraryError(f"cannot load {path}: {exc}") from exc
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = handle
    return _LIB


def last_error() -> str:
    msg = lib().smvs_last_error()
    return msg.decode() if msg else ""


def check(status: int) -> None:
    if status != SMVS_OK:
        raise SmvsError(status, last_error())


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)
