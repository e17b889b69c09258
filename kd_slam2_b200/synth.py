"""Seeded synthetic spinning-LiDAR scans (ctypes over libkds_synth.so).

Scene: ground plane z = 0 and axis-aligned boxes.  A scan is cast from a sensor
pose with an optional constant body velocity during the sweep; every point is
returned in the sensor frame at its own firing time, with that time as its stamp
(column i fires at t_start + i * scan_time / cols).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libkds_synth.so")
        if not os.path.exists(path):
            raise ImportError(f"{path} missing; run `python -m kd_slam2_b200.build`")
        lib = C.CDLL(path)
        lib.kds_synth_scene.restype = C.c_int32
        lib.kds_synth_scene.argtypes = [C.c_uint64, C.c_int32, C.c_double, C.c_void_p]
        lib.kds_synth_scan.restype = C.c_int64
        lib.kds_synth_scan.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32,
                                       C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_uint64, C.c_int32, C.c_void_p, C.c_void_p]
        lib.kds_synth_transform.restype = None
        lib.kds_synth_transform.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
        _LIB = lib
    return _LIB


def scene(seed: int, num_boxes: int = 40, radius: float = 60.0) -> np.ndarray:
    out = np.zeros((num_boxes, 6), dtype=np.float64)
    n = _lib().kds_synth_scene(seed, num_boxes, radius, out.ctypes.data)
    return out[:n].copy()


def pose(t=(0.0, 0.0, 0.0), rotvec=(0.0, 0.0, 0.0)) -> np.ndarray:
    """3x4 row-major [R|t] from a translation and a rotation vector (float64)."""
    w = np.asarray(rotvec, dtype=np.float64)
    a = np.linalg.norm(w)
    R = np.eye(3)
    if a > 1e-15:
        k = w / a
        K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
        R = np.eye(3) + np.sin(a) * K + (1 - np.cos(a)) * (K @ K)
    X = np.zeros((3, 4))
    X[:, :3] = R
    X[:, 3] = t
    return X


def scan(boxes: np.ndarray, start_pose: np.ndarray, vel=None, beams: int = 16, cols: int = 1024,
         elev=(-15.0, 15.0), scan_time: float = 0.1, t_start: float = 0.0, r_min: float = 1.0,
         r_max: float = 60.0, noise: float = 0.02, seed: int = 0, threads: int = 8):
    """Returns (xyz float32 [n,3], stamps float64 [n])."""
    boxes = np.ascontiguousarray(boxes, dtype=np.float64)
    P = np.ascontiguousarray(start_pose, dtype=np.float64).reshape(12)
    v = np.zeros(6) if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
    cap = beams * cols
    xyz = np.zeros((cap, 3), dtype=np.float32)
    st = np.zeros(cap, dtype=np.float64)
    n = _lib().kds_synth_scan(boxes.ctypes.data, len(boxes), P.ctypes.data, v.ctypes.data, beams, cols,
                              elev[0], elev[1], scan_time, t_start, r_min, r_max, noise, seed, threads,
                              xyz.ctypes.data, st.ctypes.data)
    return xyz[:n].copy(), st[:n].copy()


def transform(xyz: np.ndarray, X: np.ndarray) -> np.ndarray:
    out = np.ascontiguousarray(xyz, dtype=np.float32).copy()
    P = np.ascontiguousarray(X, dtype=np.float64).reshape(12)
    _lib().kds_synth_transform(out.ctypes.data, len(out), P.ctypes.data)
    return out
