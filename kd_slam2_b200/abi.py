"""ctypes declarations of libkds.so (include/kds.h).

The library is loaded from this package directory.  There is no fallback: if the
shared object is missing or fails to load, importing fails with an error that says
how to build it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkds.so")

KDS_OK = 0
KDS_ERR_INVALID_ARG = -1
KDS_ERR_CUDA = -2
KDS_ERR_OOM = -3
KDS_ERR_TREE_REJECTED = -4
KDS_ERR_RANGE = -5
KDS_ERR_BAD_TREE = -6
KDS_ERR_STATE = -7
KDS_ERR_TIMEOUT = -8
KDS_ERR_ADMISSION = -9
KDS_ERR_NO_DEVICE = -10
KDS_ERR_CAPACITY = -11
KDS_ERR_DIVERGED = -12

KDS_ICP = 0
KDS_CTICP = 1
KDS_MEM_HOST = 0
KDS_MEM_DEVICE = 1
KDS_JOB_COMPUTE = 0
KDS_JOB_LINEARIZE = 1
KDS_JOB_LINEARIZE_DUAL = 2
KDS_MOTION_ZERO_VEL = 0
KDS_MOTION_CONST_VEL = 1
KDS_STATUS_INIT = 0
KDS_STATUS_TRACKING = 1


class TreeParams(C.Structure):
    _fields_ = [
        ("propagate_normal", C.c_int32),
        ("tree_min_good_leaves", C.c_int32),
        ("leaf_min_points", C.c_int32),
        ("leaf_max_points", C.c_int32),
        ("leaf_density", C.c_float),
        ("leaf_min_normal_incidence", C.c_float),
        ("leaf_eigenvalue_threshold", C.c_float),
        ("leaf_normal_eigenratio", C.c_float),
        ("prune_min_normal_incidence", C.c_float),
        ("max_level", C.c_int32),
    ]


class TreeInfo(C.Structure):
    _fields_ = [
        ("num_nodes", C.c_int64),
        ("num_leaves", C.c_int64),
        ("num_points", C.c_int64),
        ("num_unpruned", C.c_int64),
        ("ts_start", C.c_double),
        ("accepted", C.c_int32),
        ("depth", C.c_int32),
        ("global_levels", C.c_int32),
        ("pad_", C.c_int32),
    ]


class KDNode3f(C.Structure):
    """kd_slam2_msgs/msg/KDNode3f (kds_kdnode3f, 56 bytes)."""
    _fields_ = [
        ("mean", C.c_float * 3),
        ("direction", C.c_float * 3),
        ("idx_start", C.c_uint32),
        ("idx_end", C.c_uint32),
        ("idx_left", C.c_int32),
        ("idx_right", C.c_int32),
        ("dts_mean", C.c_double),
        ("dts_covariance", C.c_double),
    ]


# the same record as a numpy dtype (arrays of KDNode3f without per-record ctypes objects)
KDNODE3F_DTYPE = np.dtype({
    "names": ["mean", "direction", "idx_start", "idx_end", "idx_left", "idx_right", "dts_mean", "dts_covariance"],
    "formats": [("<f4", (3,)), ("<f4", (3,)), "<u4", "<u4", "<i4", "<i4", "<f8", "<f8"],
    "offsets": [0, 12, 24, 28, 32, 36, 40, 48],
    "itemsize": 56,
})


class KDTree3f(C.Structure):
    """The tree fields of kd_slam2_msgs/msg/KDTree3f (kds_kdtree3f)."""
    _fields_ = [
        ("ts_start", C.c_double),
        ("root_mean", C.c_float * 3),
        ("root_eigenvalues", C.c_float * 3),
        ("root_eigenvectors", C.c_float * 9),
        ("num_nodes", C.c_int64),
        ("nodes", C.c_void_p),
    ]


class Factor(C.Structure):
    """kds_factor: a multi-view BA factor over a batch job."""
    _fields_ = [("job", C.c_int32), ("var", C.c_int32 * 4)]


class VoxelParams(C.Structure):
    """kds_voxel_params: Voxelizer_ PARAMs."""
    _fields_ = [
        ("range_min", C.c_float),
        ("range_max", C.c_float),
        ("space_res", C.c_float),
        ("time_res", C.c_float),
        ("use_boundary", C.c_int32),
    ]


class AlignerParams(C.Structure):
    _fields_ = [
        ("kernel_threshold", C.c_float),
        ("damping", C.c_float),
        ("max_error", C.c_float),
        ("min_normal_cos", C.c_float),
        ("min_good_measurements", C.c_int32),
        ("max_iterations", C.c_int32),
        ("velocity_damping", C.c_float),
        ("term_crit", C.c_int32),
        ("d_pert", C.c_float),
        ("d_score", C.c_float),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("num_inliers", C.c_int32),
        ("num_outliers", C.c_int32),
        ("num_bad", C.c_int32),
        ("num_err_normal", C.c_int32),
        ("num_err_fn", C.c_int32),
        ("chi2", C.c_float),
        ("chi2_kernelized", C.c_float),
        ("pert_pose_norm", C.c_float),
        ("pert_vel_norm", C.c_float),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class Job(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("mode", C.c_int32),
        ("stats_mode", C.c_int32),
        ("pad_", C.c_int32),
        ("fixed", C.c_void_p),
        ("moving", C.c_void_p),
        ("params", AlignerParams),
        ("X", C.c_double * 12),
        ("fixed_X", C.c_double * 12),
        ("v", C.c_double * 6),
        ("fixed_v", C.c_double * 6),
        ("result", C.c_int32),
        ("iterations", C.c_int32),
        ("stats", Stats),
        ("H", C.c_double * 144),
        ("b", C.c_double * 12),
        ("H_vel_B", C.c_double * 36),
        ("b_vel_B", C.c_double * 6),
        ("H_cross_pose_vel_B", C.c_double * 36),
        ("H_cross_vel_AB", C.c_double * 36),
    ]


class ServerParams(C.Structure):
    _fields_ = [
        ("max_slots", C.c_int32),
        ("map_every", C.c_int32),
        ("max_build_trees", C.c_int32),
        ("serial", C.c_int32),
        ("profile", C.c_int32),
        ("max_tiles", C.c_int32),
        ("iters_per_tick", C.c_int32),
        ("hbm_cap", C.c_int64),
        ("max_build_points", C.c_int64),
        ("tree", TreeParams),
        ("icp", AlignerParams),
        ("ct", AlignerParams),
        ("build_threads", C.c_int32),
        ("pad_", C.c_int32),
    ]


class Request(C.Structure):
    _fields_ = [
        ("stream", C.c_int32),
        ("type", C.c_int32),
        ("n", C.c_int64),
        ("xyz", C.c_void_p),
        ("stamps", C.c_void_p),
        ("X0", C.c_double * 12),
        ("v0", C.c_double * 6),
        ("arrival", C.c_double),
    ]


class Result(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("result", C.c_int32),
        ("iterations", C.c_int32),
        ("map_version", C.c_int32),
        ("stats", Stats),
        ("X", C.c_double * 12),
        ("v", C.c_double * 6),
        ("t_arrival", C.c_double),
        ("t_admit", C.c_double),
        ("t_built", C.c_double),
        ("t_done", C.c_double),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64),
        ("completed", C.c_int64),
        ("ticks", C.c_int64),
        ("build_passes", C.c_int64),
        ("map_builds", C.c_int64),
        ("built_trees", C.c_int64),
        ("hbm_cap", C.c_int64),
        ("peak_reserved", C.c_int64),
        ("mean_active", C.c_double),
        ("lin_ms", C.c_double),
        ("lin_ticks", C.c_int64),
        ("leaf_iterations", C.c_int64),
        ("alg_bytes", C.c_double),
        ("h2d_bytes", C.c_int64),
        ("d2h_bytes", C.c_int64),
        ("build_ms", C.c_double),
        ("build_points", C.c_int64),
        ("build_point_levels", C.c_double),
        ("build_global_point_levels", C.c_double),
        ("build_busy_ms", C.c_double),
        ("build_released_ahead", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


# Every entry point declared in include/kds.h: name -> (restype, argtypes)
_P = C.c_void_p
_I32 = C.c_int32
_I64 = C.c_int64

class TrackerParams(C.Structure):
    """kds_tracker_params: TrackerProc_ PARAMs, its odometry aligner and motion model."""
    _fields_ = [
        ("aligner_type", C.c_int32),
        ("aligner", AlignerParams),
        ("motion_model", C.c_int32),
        ("motion_model_alpha", C.c_float),
        ("min_inlier_frac", C.c_float),
        ("max_kf_trans", C.c_float),
        ("max_kf_rot_deg", C.c_float),
    ]


class TrackerResult(C.Structure):
    """kds_tracker_result: what one addFrame produced."""
    _fields_ = [
        ("status", C.c_int32),
        ("result", C.c_int32),
        ("new_keyframe", C.c_int32),
        ("frame_idx", C.c_int32),
        ("keyframe_count", C.c_int32),
        ("pad_", C.c_int32),
        ("frame_duration", C.c_double),
        ("pose_in_kf", C.c_double * 12),
        ("pose_in_world", C.c_double * 12),
        ("velocity", C.c_double * 6),
        ("ct_velocity", C.c_double * 6),
        ("stats", Stats),
    ]


class TrackerState(C.Structure):
    """kds_tracker_state: a tracker checkpoint without its keyframe tree."""
    _fields_ = [
        ("params", TrackerParams),
        ("last_ts", C.c_double),
        ("frame_duration", C.c_double),
        ("T_delta_log", C.c_double * 6),
        ("kf_pose_in_world", C.c_double * 12),
        ("pose_in_kf", C.c_double * 12),
        ("pose_global", C.c_double * 12),
        ("frame_idx", C.c_int32),
        ("keyframe_count", C.c_int32),
        ("has_keyframe", C.c_int32),
        ("pad_", C.c_int32),
    ]

SIGNATURES = {
    "kds_last_error": (C.c_char_p, []),
    "kds_init": (C.c_int, [_I32, _I32]),
    "kds_launch_count": (_I64, []),
    "kds_tree_params_default": (None, [C.POINTER(TreeParams)]),
    "kds_tree_build": (C.c_int, [_P, _P, _I64, _I32, C.POINTER(TreeParams), _P, C.POINTER(_P)]),
    "kds_tree_build_batch": (C.c_int, [_P, _P, _P, _I32, _I32, C.POINTER(TreeParams), _P, C.POINTER(_P),
                                       C.POINTER(_I32)]),
    "kds_tree_import": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _I64, C.c_double, C.POINTER(_P)]),
    "kds_tree_get_info": (C.c_int, [_P, C.POINTER(TreeInfo)]),
    "kds_tree_get_root": (C.c_int, [_P, _P, _P, _P]),
    "kds_voxel_params_default": (None, [C.POINTER(VoxelParams)]),
    "kds_points_voxelize": (C.c_int, [_P, _P, _I64, _I32, C.c_double, C.c_double, C.POINTER(VoxelParams), _P, _P,
                                      _P, C.POINTER(_I64)]),
    "kds_tree_from_msg": (C.c_int, [C.POINTER(KDTree3f), C.POINTER(_P)]),
    "kds_tree_to_msg": (C.c_int, [_P, C.POINTER(KDTree3f)]),
    "kds_tree_export": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "kds_tree_apply_velocities": (C.c_int, [_P, _P, _I32, _P]),
    "kds_tree_apply_isometry": (C.c_int, [_P, _P, _P]),
    "kds_tree_extract_compressed_leaves": (C.c_int, [_P, _P, _P, _P]),
    "kds_tree_extract_compressed_leaves_device": (C.c_int, [_P, _P, _P, _P]),
    "kds_tree_free": (None, [_P]),
    "kds_aligner_params_default": (None, [C.POINTER(AlignerParams)]),
    "kds_aligner_create": (C.c_int, [_I32, C.POINTER(AlignerParams), C.POINTER(_P)]),
    "kds_aligner_set_params": (C.c_int, [_P, C.POINTER(AlignerParams)]),
    "kds_aligner_set_stream": (C.c_int, [_P, _P]),
    "kds_aligner_set_fixed": (C.c_int, [_P, _P]),
    "kds_aligner_set_moving": (C.c_int, [_P, _P]),
    "kds_aligner_set_x": (C.c_int, [_P, _P]),
    "kds_aligner_get_x": (C.c_int, [_P, _P]),
    "kds_aligner_set_fixed_x": (C.c_int, [_P, _P]),
    "kds_aligner_set_velocities": (C.c_int, [_P, _P]),
    "kds_aligner_get_velocities": (C.c_int, [_P, _P]),
    "kds_aligner_set_fixed_velocities": (C.c_int, [_P, _P]),
    "kds_aligner_reset_moving_state": (C.c_int, [_P]),
    "kds_aligner_set_pose_prior": (C.c_int, [_P, _P, _P, _P]),
    "kds_aligner_add_fixed_entry": (C.c_int, [_P, _P, _P]),
    "kds_aligner_clear_fixed_forest": (C.c_int, [_P]),
    "kds_aligner_compute": (C.c_int, [_P, _I32, C.POINTER(_I32)]),
    "kds_aligner_one_round": (C.c_int, [_P, _I32, C.POINTER(_I32)]),
    "kds_aligner_build_quadratic_form": (C.c_int, [_P, _I32]),
    "kds_aligner_build_quadratic_form_dual": (C.c_int, [_P, _I32]),
    "kds_aligner_get_hb": (C.c_int, [_P, _P, _P, _P]),
    "kds_aligner_get_dual": (C.c_int, [_P, _P, _P, _P, _P]),
    "kds_aligner_get_pose_hessian": (C.c_int, [_P, _P]),
    "kds_aligner_get_stats": (C.c_int, [_P, C.POINTER(Stats)]),
    "kds_aligner_get_stats_log": (C.c_int, [_P, C.POINTER(Stats), _I32, C.POINTER(_I32)]),
    "kds_aligner_linearize_debug": (C.c_int, [_P, _P, _P, _P, _I32, _I32, _P, _P, _P, _P, C.POINTER(Stats)]),
    "kds_aligner_set_profiling": (C.c_int, [_P, _I32]),
    "kds_aligner_get_profile": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(_I32)]),
    "kds_aligner_count_touched_nodes": (C.c_int, [_P, C.POINTER(_I64)]),
    "kds_phase_stamps": (C.c_int, [_P]),
    "kds_set_tma_wait_limit": (C.c_int, [C.c_int32]),
    "kds_aligner_free": (None, [_P]),
    "kds_batch_create": (C.c_int, [C.POINTER(_P)]),
    "kds_batch_run": (C.c_int, [_P, C.POINTER(Job), _I32, _I32, _P]),
    "kds_batch_autotune": (C.c_int, [_P, C.POINTER(Job), _I32, _P, C.POINTER(_I32), _P]),
    "kds_batch_configure": (C.c_int, [_P, C.c_int32]),
    "kds_batch_assemble": (C.c_int, [_P, C.POINTER(Factor), _I32, _I32, C.c_float, _P, C.POINTER(_I32), _P, _P,
                                     _P, _P]),
    "kds_batch_free": (None, [_P]),
    "kds_server_params_default": (None, [C.POINTER(ServerParams)]),
    "kds_server_create": (C.c_int, [C.POINTER(ServerParams), C.POINTER(_P)]),
    "kds_server_add_stream": (C.c_int, [_P, _P, _I64, _I64, C.POINTER(_I32)]),
    "kds_server_submit": (C.c_int, [_P, C.POINTER(Request), C.POINTER(_I64)]),
    "kds_server_start": (C.c_int, [_P]),
    "kds_server_drain": (C.c_int, [_P, C.c_double]),
    "kds_server_wait": (C.c_int, [_P, _I64, C.c_double, C.POINTER(Result)]),
    "kds_server_get_stats": (C.c_int, [_P, C.POINTER(ServerStats)]),
    "kds_server_get_trace": (C.c_int, [_P, _P, _I32, C.POINTER(_I32)]),
    "kds_server_free": (None, [_P]),
    "kds_tree_build_batch_gather": (C.c_int, [_P, _P, _P, _I32, C.POINTER(TreeParams), _P, _P, _P]),
    "kds_tracker_params_default": (None, [C.POINTER(TrackerParams)]),
    "kds_tracker_create": (C.c_int, [C.POINTER(TrackerParams), _P, C.POINTER(_P)]),
    "kds_tracker_add_frame": (C.c_int, [_P, _P, C.c_double, _P, C.POINTER(TrackerResult)]),
    "kds_tracker_add_frames": (C.c_int, [_P, _P, _P, _P, _I32, _P, _P, C.POINTER(TrackerResult), _P]),
    "kds_tracker_get_pose": (C.c_int, [_P, _P, _P]),
    "kds_tracker_get_keyframe": (C.c_int, [_P, C.POINTER(_P), _P]),
    "kds_tracker_get_state": (C.c_int, [_P, C.POINTER(TrackerState)]),
    "kds_tracker_set_state": (C.c_int, [_P, C.POINTER(TrackerState), _P]),
    "kds_tracker_reset": (C.c_int, [_P]),
    "kds_tracker_free": (None, [_P]),
    "kds_linearize_static": (C.c_int, [_P, _P, _I32, C.POINTER(AlignerParams), _P, _P, _P, _P, _I32, _P, _P, _P,
                                       C.POINTER(Stats)]),
}


def load(path: str = LIB_PATH) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(
            f"libkds.so not found at {path}; build it with `python -m kd_slam2_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class KdsError(RuntimeError):
    def __init__(self, code: int, where: str, text: str):
        super().__init__(f"{where}: status {code}: {text}")
        self.code = code
