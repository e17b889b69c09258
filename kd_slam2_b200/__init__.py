"""B200-native KD-SLAM registration path: Python mirror of the reference's aligner API.

The classes here wrap the C ABI of libkds.so (include/kds.h) and follow the method and
parameter names of the reference types they stand in for:

  TreeGeneratorB2003D  ~ TreeGenerator3D   (kd/tree/tree_generator_.h:10-47)
  ICPB2003D            ~ ICPCUDA3D / ICPCPU3D   (kd/icp/tree_aligner_base_.h:25-161)
  CTICPB2003D          ~ CTICPCUDA3D / CTICPCPU3D (kd/cticp/cticp_.h:20-261)
  Tracker3D            ~ the odometry of TrackerProc_ / SLAMProc_ (kd/tracker/tracker_proc_.h)

Poses are 3x4 numpy arrays [R | t] (world <- body); velocities are [v; w].
All compute runs on the GPU; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import abi as L
from .abi import KdsError

class _Lazy:
    """Loads libkds.so on first use, so that `python -m kd_slam2_b200.build` can run
    before the library exists.  A missing library raises ImportError at that point."""

    def __getattr__(self, name):
        real = L.load()
        globals()["_lib"] = real
        return getattr(real, name)


_lib = _Lazy()


def lib():
    """The loaded libkds.so (ctypes.CDLL)."""
    global _lib
    if isinstance(_lib, _Lazy):
        _lib = L.load()
    return _lib


def _check(rc: int, where: str) -> None:
    if rc != L.KDS_OK:
        raise KdsError(rc, where, (_lib.kds_last_error() or b"").decode())


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def _pose12(X) -> np.ndarray:
    X = np.asarray(X, dtype=np.float64)
    if X.shape == (4, 4):
        X = X[:3]
    return np.ascontiguousarray(X.reshape(12))


def identity() -> np.ndarray:
    X = np.zeros((3, 4))
    X[:, :3] = np.eye(3)
    return X


def init(device: int = 0, blocking_sync: bool = False) -> None:
    _check(_lib.kds_init(device, 1 if blocking_sync else 0), "kds_init")


# ---------------------------------------------------------------------------- trees
class Tree:
    """A surfel KD-tree resident on the GPU (Tree_ / TreeCUDA_, kd/tree/tree_.h:15-56)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def __del__(self):
        if _lib is not None:  # None once the interpreter tears the module down
            self.free()

    def free(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.kds_tree_free(self._h)
            self._h = C.c_void_p(None)

    @property
    def info(self) -> L.TreeInfo:
        inf = L.TreeInfo()
        _check(_lib.kds_tree_get_info(self._h, C.byref(inf)), "kds_tree_get_info")
        return inf

    @property
    def num_nodes(self) -> int:
        return self.info.num_nodes

    @property
    def num_leaves(self) -> int:
        return self.info.num_leaves

    def export(self) -> dict:
        inf = self.info
        n, nl, npnt = inf.num_nodes, inf.num_leaves, inf.num_points
        out = {
            "mean": np.zeros((n, 3), np.float32), "dir": np.zeros((n, 3), np.float32),
            "dts_mean": np.zeros(n), "dts_cov": np.zeros(n),
            "start": np.zeros(n, np.int64), "end": np.zeros(n, np.int64),
            "left": np.zeros(n, np.int32), "right": np.zeros(n, np.int32), "level": np.zeros(n, np.int32),
            "leaves": np.zeros(nl, np.int64), "perm": np.zeros(npnt, np.int64),
        }
        _check(_lib.kds_tree_export(self._h, *(out[k].ctypes.data for k in (
            "mean", "dir", "dts_mean", "dts_cov", "start", "end", "left", "right", "level", "leaves")),
            out["perm"].ctypes.data if npnt else None), "kds_tree_export")
        out["ts_start"] = inf.ts_start
        return out

    def root(self) -> dict:
        """Tree_::root_mean / root_eigenvalues / root_eigenvectors (3x3, columns = vectors)."""
        m, ev, V = np.zeros(3, np.float32), np.zeros(3, np.float32), np.zeros(9, np.float32)
        _check(_lib.kds_tree_get_root(self._h, m.ctypes.data, ev.ctypes.data, V.ctypes.data), "kds_tree_get_root")
        return {"root_mean": m, "root_eigenvalues": ev, "root_eigenvectors": V.reshape(3, 3).T.copy()}

    def to_msg(self) -> dict:
        """toMessage (lib/kd_io/slam_messages.h:47-80): the tree fields of a KDTree3f message;
        nodes as a KDNODE3F_DTYPE array, root_eigenvectors column-major (9 floats)."""
        m = L.KDTree3f()
        _check(_lib.kds_tree_to_msg(self._h, C.byref(m)), "kds_tree_to_msg")  # count query
        nodes = np.zeros(m.num_nodes, L.KDNODE3F_DTYPE)
        m.nodes = nodes.ctypes.data
        _check(_lib.kds_tree_to_msg(self._h, C.byref(m)), "kds_tree_to_msg")
        return {"ts_start": m.ts_start, "root_mean": np.array(m.root_mean, np.float32),
                "root_eigenvalues": np.array(m.root_eigenvalues, np.float32),
                "root_eigenvectors": np.array(m.root_eigenvectors, np.float32), "nodes": nodes}

    @staticmethod
    def from_msg(msg: dict) -> "Tree":
        """TreeLoader_::fromTreeMsg (lib/kd_io/tree_loader_impl_.h:59-70): a device tree (no
        points) from the tree fields of a KDTree3f message (the dict of Tree.to_msg)."""
        nodes = np.ascontiguousarray(msg["nodes"], L.KDNODE3F_DTYPE)
        m = L.KDTree3f()
        m.ts_start = float(msg.get("ts_start", 0.0))
        for k in ("root_mean", "root_eigenvalues", "root_eigenvectors"):
            if k in msg:
                getattr(m, k)[:] = [float(x) for x in np.asarray(msg[k], np.float32).reshape(-1)]
        m.num_nodes = len(nodes)
        m.nodes = nodes.ctypes.data
        h = C.c_void_p()
        _check(_lib.kds_tree_from_msg(C.byref(m), C.byref(h)), "kds_tree_from_msg")
        return Tree(h.value)

    @staticmethod
    def import_nodes(mean, dir, left, right, dts_mean=None, dts_cov=None, start=None, end=None,
                     ts_start: float = 0.0) -> "Tree":
        """Tree_CUDAfromCPU_: uploads a BFS-ordered node array (Node_ fields)."""
        mean = np.ascontiguousarray(mean, np.float32)
        dir = np.ascontiguousarray(dir, np.float32)
        left = np.ascontiguousarray(left, np.int32)
        right = np.ascontiguousarray(right, np.int32)
        dm = None if dts_mean is None else np.ascontiguousarray(dts_mean, np.float64)
        dc = None if dts_cov is None else np.ascontiguousarray(dts_cov, np.float64)
        s0 = None if start is None else np.ascontiguousarray(start, np.int64)
        e0 = None if end is None else np.ascontiguousarray(end, np.int64)
        h = C.c_void_p()
        _check(_lib.kds_tree_import(mean.ctypes.data, dir.ctypes.data, _ptr(dm), _ptr(dc), _ptr(s0), _ptr(e0),
                                    left.ctypes.data, right.ctypes.data, len(mean), ts_start, C.byref(h)),
               "kds_tree_import")
        return Tree(h.value)

    def apply_velocities_in_place(self, v, skip_leaves: bool = False) -> None:
        vv = np.ascontiguousarray(v, np.float32)
        _check(_lib.kds_tree_apply_velocities(self._h, vv.ctypes.data, 1 if skip_leaves else 0, None),
               "kds_tree_apply_velocities")

    def apply_isometry_in_place(self, X) -> None:
        XX = np.ascontiguousarray(_pose12(X), np.float32)
        _check(_lib.kds_tree_apply_isometry(self._h, XX.ctypes.data, None), "kds_tree_apply_isometry")

    def extract_compressed_leaves(self, v=None) -> np.ndarray:
        out = np.zeros((self.num_leaves, 6), np.float32)
        vv = None if v is None else np.ascontiguousarray(v, np.float32)
        _check(_lib.kds_tree_extract_compressed_leaves(self._h, _ptr(vv), out.ctypes.data, None),
               "kds_tree_extract_compressed_leaves")
        return out

    def extract_compressed_leaves_device(self, out, v=None, stream=None) -> None:
        """The same gather into a CUDA tensor `out` of shape (num_leaves, 6), float32
        (kds_tree_extract_compressed_leaves_device: no allocation, asynchronous)."""
        if tuple(out.shape) != (self.num_leaves, 6) or str(out.dtype) != "torch.float32" or not out.is_cuda \
                or not out.is_contiguous():
            raise ValueError("out must be a contiguous float32 CUDA tensor of shape (num_leaves, 6)")
        vv = None if v is None else np.ascontiguousarray(v, np.float32)
        _check(_lib.kds_tree_extract_compressed_leaves_device(self._h, _ptr(vv), out.data_ptr(), stream),
               "kds_tree_extract_compressed_leaves_device")


class TreeGeneratorB2003D:
    """TreeGenerator3D with the same PARAM names and defaults; builds on the GPU."""

    def __init__(self, **params):
        self.params = L.TreeParams()
        _lib.kds_tree_params_default(C.byref(self.params))
        for k, v in params.items():
            if not hasattr(self.params, k):
                raise AttributeError(f"TreeGeneratorB2003D has no parameter {k}")
            setattr(self.params, k, v)

    def make_tree(self, xyz, stamps=None, device: bool = False, stream=None) -> Tree | None:
        """makeTree: returns None where the reference returns nullptr."""
        if device:
            n = int(xyz.shape[0])
            px, ps, mem = int(xyz.data_ptr()), (int(stamps.data_ptr()) if stamps is not None else None), L.KDS_MEM_DEVICE
        else:
            xyz = np.ascontiguousarray(xyz, np.float32)
            st = None if stamps is None else np.ascontiguousarray(stamps, np.float64)
            n, px, ps, mem = len(xyz), xyz.ctypes.data, _ptr(st), L.KDS_MEM_HOST
        h = C.c_void_p()
        rc = _lib.kds_tree_build(px, ps, n, mem, C.byref(self.params), stream, C.byref(h))
        if rc == L.KDS_ERR_TREE_REJECTED:
            return None
        _check(rc, "kds_tree_build")
        return Tree(h.value)

    def make_trees(self, clouds, stream=None) -> list:
        """Builds one tree per (xyz, stamps) cloud in a single batched pass; None entries
        where makeTree would return nullptr.  The clouds are copied to the device one by
        one (kds_tree_build_batch_gather), without packing them on the host first."""
        xs = [np.ascontiguousarray(np.asarray(c[0], np.float32).reshape(-1, 3)) for c in clouds]
        ss = [None if c[1] is None else np.ascontiguousarray(c[1], np.float64) for c in clouds]
        R = len(clouds)
        xp = (C.c_void_p * R)(*[x.ctypes.data for x in xs])
        sp = (C.c_void_p * R)(*[None if t is None else t.ctypes.data for t in ss])
        counts = np.array([len(x) for x in xs], np.int64)
        hs = (C.c_void_p * R)()
        status = (C.c_int32 * R)()
        _check(_lib.kds_tree_build_batch_gather(xp, sp, counts.ctypes.data, R, C.byref(self.params), stream, hs,
                                                status), "kds_tree_build_batch_gather")
        return [Tree(hs[i]) if status[i] == L.KDS_OK else None for i in range(R)]


# ---------------------------------------------------------------------------- aligners
class _AlignerBase:
    TYPE = L.KDS_ICP
    D = 6

    def __init__(self, **params):
        self.params = L.AlignerParams()
        _lib.kds_aligner_params_default(C.byref(self.params))
        for k, v in params.items():
            self.set_param(k, v)
        h = C.c_void_p()
        _check(_lib.kds_aligner_create(self.TYPE, C.byref(self.params), C.byref(h)), "kds_aligner_create")
        self._h = h
        self._keep = []
        self.stats_log: list[dict] = []

    def set_param(self, k, v):
        if k == "term_crit" and isinstance(v, dict):
            self.params.term_crit = 1
            self.params.d_pert = v.get("d_pert", 1e-3)
            self.params.d_score = v.get("d_score", 1e-3)
            return
        if not hasattr(self.params, k):
            raise AttributeError(f"{type(self).__name__} has no parameter {k}")
        setattr(self.params, k, v)
        if getattr(self, "_h", None) is not None:
            _check(_lib.kds_aligner_set_params(self._h, C.byref(self.params)), "kds_aligner_set_params")

    def __del__(self):
        if _lib is not None and getattr(self, "_h", None) is not None and self._h.value:
            _lib.kds_aligner_free(self._h)
            self._h = C.c_void_p(None)

    def set_fixed(self, t: Tree) -> None:
        self._fixed = t
        _check(_lib.kds_aligner_set_fixed(self._h, t.handle), "kds_aligner_set_fixed")

    def set_moving(self, t: Tree) -> None:
        self._moving = t
        _check(_lib.kds_aligner_set_moving(self._h, t.handle), "kds_aligner_set_moving")

    def set_x(self, X) -> None:
        _check(_lib.kds_aligner_set_x(self._h, _pose12(X).ctypes.data), "kds_aligner_set_x")

    def get_x(self) -> np.ndarray:
        X = np.zeros(12)
        _check(_lib.kds_aligner_get_x(self._h, X.ctypes.data), "kds_aligner_get_x")
        return X.reshape(3, 4)

    def set_fixed_x(self, X) -> None:
        _check(_lib.kds_aligner_set_fixed_x(self._h, _pose12(X).ctypes.data), "kds_aligner_set_fixed_x")

    def set_velocities(self, v) -> None:
        vv = np.ascontiguousarray(v, np.float64)
        _check(_lib.kds_aligner_set_velocities(self._h, vv.ctypes.data), "kds_aligner_set_velocities")

    def velocities(self) -> np.ndarray:
        v = np.zeros(6)
        _check(_lib.kds_aligner_get_velocities(self._h, v.ctypes.data), "kds_aligner_get_velocities")
        return v

    def set_fixed_velocities(self, v) -> None:
        vv = np.ascontiguousarray(v, np.float64)
        _check(_lib.kds_aligner_set_fixed_velocities(self._h, vv.ctypes.data), "kds_aligner_set_fixed_velocities")

    def reset_moving_state(self) -> None:
        _check(_lib.kds_aligner_reset_moving_state(self._h), "kds_aligner_reset_moving_state")

    def set_pose_prior(self, X_ref=None, Z=None, info=None) -> None:
        X_ref = identity() if X_ref is None else X_ref
        Z = identity() if Z is None else Z
        info = np.zeros((6, 6)) if info is None else np.asarray(info, np.float64)
        inf = np.ascontiguousarray(info.reshape(36))
        _check(_lib.kds_aligner_set_pose_prior(self._h, _pose12(X_ref).ctypes.data, _pose12(Z).ctypes.data,
                                               inf.ctypes.data), "kds_aligner_set_pose_prior")

    def add_fixed_entry(self, t: Tree, X) -> None:
        """makeFixedEntry + _fixed_forest insertion."""
        self._keep.append(t)
        _check(_lib.kds_aligner_add_fixed_entry(self._h, t.handle, _pose12(X).ctypes.data),
               "kds_aligner_add_fixed_entry")

    def clear_fixed_forest(self) -> None:
        self._keep.clear()
        _check(_lib.kds_aligner_clear_fixed_forest(self._h), "kds_aligner_clear_fixed_forest")

    def compute(self, stats_mode: bool = False) -> int:
        r = C.c_int32()
        _check(_lib.kds_aligner_compute(self._h, 1 if stats_mode else 0, C.byref(r)), "kds_aligner_compute")
        log = (L.Stats * 64)()
        n = C.c_int32()
        _check(_lib.kds_aligner_get_stats_log(self._h, log, 64, C.byref(n)), "kds_aligner_get_stats_log")
        self.stats_log = [log[i].as_dict() for i in range(min(n.value, 64))]
        return r.value

    def one_round(self, stats_mode: bool = False) -> bool:
        ok = C.c_int32()
        _check(_lib.kds_aligner_one_round(self._h, 1 if stats_mode else 0, C.byref(ok)), "kds_aligner_one_round")
        return bool(ok.value)

    def build_quadratic_form(self, stats_mode: bool = False) -> None:
        _check(_lib.kds_aligner_build_quadratic_form(self._h, 1 if stats_mode else 0),
               "kds_aligner_build_quadratic_form")

    def _hb(self):
        D = self.D
        H, b, dx = np.zeros(D * D), np.zeros(D), np.zeros(D)
        _check(_lib.kds_aligner_get_hb(self._h, H.ctypes.data, b.ctypes.data, dx.ctypes.data), "kds_aligner_get_hb")
        return H.reshape(D, D), b, dx

    @property
    def H(self) -> np.ndarray:
        return self._hb()[0]

    @property
    def b(self) -> np.ndarray:
        return self._hb()[1]

    @property
    def dx(self) -> np.ndarray:
        return self._hb()[2]

    @property
    def stats(self) -> dict:
        s = L.Stats()
        _check(_lib.kds_aligner_get_stats(self._h, C.byref(s)), "kds_aligner_get_stats")
        return s.as_dict()

    def get_pose_hessian(self) -> np.ndarray:
        H = np.zeros(36)
        _check(_lib.kds_aligner_get_pose_hessian(self._h, H.ctypes.data), "kds_aligner_get_pose_hessian")
        return H.reshape(6, 6)

    def set_profiling(self, on: bool = True) -> None:
        _check(_lib.kds_aligner_set_profiling(self._h, 1 if on else 0), "kds_aligner_set_profiling")

    def profile(self) -> tuple[float, int]:
        """(mean linearization launch duration in ms, launches) of the last compute."""
        m = C.c_double()
        n = C.c_int32()
        _check(_lib.kds_aligner_get_profile(self._h, C.byref(m), C.byref(n)), "kds_aligner_get_profile")
        return m.value, n.value

    def count_touched_nodes(self) -> int:
        c = C.c_int64()
        _check(_lib.kds_aligner_count_touched_nodes(self._h, C.byref(c)), "kds_aligner_count_touched_nodes")
        return c.value

    def set_stream(self, stream) -> None:
        _check(_lib.kds_aligner_set_stream(self._h, stream), "kds_aligner_set_stream")

    def linearize_debug(self, caches36, v=None, fixed_v=None, kind=None, stats_mode=False):
        """One linearization at explicit float caches (Xm, Xf, Xmf): per-leaf matches and status."""
        n = self._moving.num_leaves
        kind = (0 if self.TYPE == L.KDS_ICP else 1) if kind is None else kind
        D = 6 if kind == 0 else 12
        c = np.ascontiguousarray(caches36, np.float32)
        vv = None if v is None else np.ascontiguousarray(v, np.float32)
        fv = None if fixed_v is None else np.ascontiguousarray(fixed_v, np.float32)
        match = np.zeros(n, np.int32)
        status = np.zeros(n, np.int32)
        H, b = np.zeros(D * D), np.zeros(D)
        st = L.Stats()
        _check(_lib.kds_aligner_linearize_debug(self._h, c.ctypes.data, _ptr(vv), _ptr(fv), kind,
                                                1 if stats_mode else 0, match.ctypes.data, status.ctypes.data,
                                                H.ctypes.data, b.ctypes.data, C.byref(st)),
               "kds_aligner_linearize_debug")
        return match, status, H.reshape(D, D), b, st.as_dict()


class ICPB2003D(_AlignerBase):
    TYPE = L.KDS_ICP
    D = 6


class CTICPB2003D(_AlignerBase):
    TYPE = L.KDS_CTICP
    D = 12

    def __init__(self, **params):
        params.setdefault("velocity_damping", 100.0)
        super().__init__(**params)

    def build_quadratic_form_dual(self, stats_mode: bool = False) -> None:
        _check(_lib.kds_aligner_build_quadratic_form_dual(self._h, 1 if stats_mode else 0),
               "kds_aligner_build_quadratic_form_dual")

    def dual(self) -> dict:
        a, b, c, d = np.zeros(36), np.zeros(6), np.zeros(36), np.zeros(36)
        _check(_lib.kds_aligner_get_dual(self._h, a.ctypes.data, b.ctypes.data, c.ctypes.data, d.ctypes.data),
               "kds_aligner_get_dual")
        return {"H_dual_vel_B": a.reshape(6, 6), "b_dual_vel_B": b,
                "H_dual_cross_pose_vel_B": c.reshape(6, 6), "H_dual_cross_vel_AB": d.reshape(6, 6)}


# ---------------------------------------------------------------------------- batches
class _TreeView(Tree):
    """A tree handle owned elsewhere (the tracker's keyframe): never freed here."""

    def free(self) -> None:
        self._h = C.c_void_p(None)


class ZeroVelMotionModel3D:
    """ZeroVelMotionModel_ (kd/motion_model/zero_vel_motion_model_.h): identity prediction."""
    KIND = L.KDS_MOTION_ZERO_VEL

    def __init__(self):
        self.motion_model_alpha = 0.9


class ConstVelMotionModel3D(ZeroVelMotionModel3D):
    """ConstVelMotionModel_ (kd/motion_model/const_vel_motion_model_.h): prediction
    expmap(T_delta_log), updated by T_delta_log <- alpha T_delta_log + (1 - alpha) log(delta)."""
    KIND = L.KDS_MOTION_CONST_VEL

    def __init__(self, motion_model_alpha: float = 0.9):
        self.motion_model_alpha = motion_model_alpha


class Tracker3D:
    """Odometry of TrackerProc_::addFrame (kd/tracker/tracker_proc_frame_impl_.h:33-115)
    with SLAMProc_'s keyframe switch (kd/slam/slam_proc_frame_impl_.h:8-49) and no
    relocalisation, loop search or pose graph.

    odom_aligner: an ICPB2003D or CTICPB2003D whose parameters the tracker copies (the
    tracker runs its own aligner); motion_model: ZeroVelMotionModel3D (the reference's
    default) or ConstVelMotionModel3D.  add_frame transforms the frame tree in place
    (T_base_lidar, then the velocity morphs) as the reference does; the keyframe is a
    device copy owned by the tracker.
    """

    def __init__(self, odom_aligner=None, motion_model=None, min_inlier_frac: float = 0.6,
                 max_kf_trans: float = 3.0, max_kf_rot_deg: float = 360.0, stream=None):
        p = L.TrackerParams()
        _lib.kds_tracker_params_default(C.byref(p))
        if odom_aligner is not None:
            p.aligner_type = odom_aligner.TYPE
            p.aligner = odom_aligner.params
        mm = motion_model if motion_model is not None else ZeroVelMotionModel3D()
        p.motion_model = mm.KIND
        p.motion_model_alpha = mm.motion_model_alpha
        p.min_inlier_frac = min_inlier_frac
        p.max_kf_trans = max_kf_trans
        p.max_kf_rot_deg = max_kf_rot_deg
        self.params = p
        h = C.c_void_p()
        _check(_lib.kds_tracker_create(C.byref(p), stream, C.byref(h)), "kds_tracker_create")
        self._h = h

    def __del__(self):
        if _lib is not None:  # None once the interpreter tears the module down
            self.free()

    def free(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.kds_tracker_free(self._h)
            self._h = C.c_void_p(None)

    def add_frame(self, tree: Tree, ts: float, T_base_lidar=None) -> dict:
        r = L.TrackerResult()
        X = None if T_base_lidar is None else _pose12(T_base_lidar)
        _check(_lib.kds_tracker_add_frame(self._h, tree.handle, float(ts), _ptr(X), C.byref(r)),
               "kds_tracker_add_frame")
        return self._result(r)

    @staticmethod
    def _result(r) -> dict:
        return {"status": r.status, "result": r.result, "new_keyframe": bool(r.new_keyframe),
                "frame_idx": r.frame_idx, "keyframe_count": r.keyframe_count, "frame_duration": r.frame_duration,
                "pose_in_kf": np.array(r.pose_in_kf[:]).reshape(3, 4),
                "pose_in_world": np.array(r.pose_in_world[:]).reshape(3, 4),
                "velocity": np.array(r.velocity[:]), "ct_velocity": np.array(r.ct_velocity[:]),
                "stats": r.stats.as_dict()}

    @staticmethod
    def add_frames(trackers, trees, ts, batch: "Batch", T_base_lidar=None, stream=None):
        """One step of many trackers with their alignments in one batch
        (kds_tracker_add_frames).  Returns (results, codes); raises on a call error other
        than a tracker's divergence, which shows as that tracker's code."""
        n = len(trackers)
        hs = (C.c_void_p * n)(*[t._h.value for t in trackers])
        fs = (C.c_void_p * n)(*[t.handle.value for t in trees])
        tt = np.ascontiguousarray(ts, np.float64)
        X = None if T_base_lidar is None else np.ascontiguousarray(
            np.stack([_pose12(x) for x in T_base_lidar]))
        out = (L.TrackerResult * n)()
        codes = np.zeros(n, np.int32)
        rc = _lib.kds_tracker_add_frames(hs, fs, tt.ctypes.data, _ptr(X), n, batch._h, stream, out,
                                         codes.ctypes.data)
        if rc not in (L.KDS_OK, L.KDS_ERR_DIVERGED):
            _check(rc, "kds_tracker_add_frames")
        return [Tracker3D._result(out[i]) for i in range(n)], codes

    def pose_global(self) -> np.ndarray:
        X = np.zeros(12)
        _check(_lib.kds_tracker_get_pose(self._h, X.ctypes.data, None), "kds_tracker_get_pose")
        return X.reshape(3, 4)

    def pose_in_kf(self) -> np.ndarray:
        X = np.zeros(12)
        _check(_lib.kds_tracker_get_pose(self._h, None, X.ctypes.data), "kds_tracker_get_pose")
        return X.reshape(3, 4)

    def keyframe(self) -> tuple[dict | None, np.ndarray]:
        """The keyframe tree's export (None before the first frame) and its pose_in_world."""
        h = C.c_void_p()
        X = np.zeros(12)
        _check(_lib.kds_tracker_get_keyframe(self._h, C.byref(h), X.ctypes.data), "kds_tracker_get_keyframe")
        if not h.value:
            return None, X.reshape(3, 4)
        return _TreeView(h.value).export(), X.reshape(3, 4)

    def reset(self) -> None:
        _check(_lib.kds_tracker_reset(self._h), "kds_tracker_reset")

    def checkpoint(self) -> dict:
        """The tracker's state (kds_tracker_get_state, as bytes) and its keyframe as a
        KDTree3f message (Tree.to_msg), both plain host data."""
        st = L.TrackerState()
        _check(_lib.kds_tracker_get_state(self._h, C.byref(st)), "kds_tracker_get_state")
        kf = None
        if st.has_keyframe:
            h = C.c_void_p()
            _check(_lib.kds_tracker_get_keyframe(self._h, C.byref(h), None), "kds_tracker_get_keyframe")
            kf = _TreeView(h.value).to_msg()
        return {"state": bytes(st), "keyframe": kf}

    def restore(self, ckpt: dict) -> None:
        """Resumes from checkpoint() output (kds_tracker_set_state)."""
        st = L.TrackerState.from_buffer_copy(ckpt["state"])
        kf = Tree.from_msg(ckpt["keyframe"]) if ckpt["keyframe"] is not None else None
        _check(_lib.kds_tracker_set_state(self._h, C.byref(st), kf.handle if kf is not None else None),
               "kds_tracker_set_state")


class Batch:
    """Many independent alignments / linearizations per launch (kds_batch_run)."""

    def __init__(self):
        h = C.c_void_p()
        _check(_lib.kds_batch_create(C.byref(h)), "kds_batch_create")
        self._h = h

    def __del__(self):
        if _lib is not None and getattr(self, "_h", None) is not None and self._h.value:
            _lib.kds_batch_free(self._h)
            self._h = C.c_void_p(None)

    def autotune(self, jobs, stream=None):
        """Chooses the launch configuration for this job set; returns (index, ms per config)."""
        arr = (L.Job * len(jobs))(*jobs)
        chosen = C.c_int32()
        ms = np.zeros(18)
        _check(_lib.kds_batch_autotune(self._h, arr, len(jobs), stream, C.byref(chosen), ms.ctypes.data),
               "kds_batch_autotune")
        return chosen.value, ms

    def configure(self, config: int) -> None:
        """Launch configuration by index (stage + 3 * order + 6 * form), as autotune reports it."""
        _check(_lib.kds_batch_configure(self._h, int(config)), "kds_batch_configure")

    def run(self, jobs, use_graph: bool = True, stream=None):
        arr = (L.Job * len(jobs))(*jobs)
        _check(_lib.kds_batch_run(self._h, arr, len(jobs), 1 if use_graph else 0, stream), "kds_batch_run")
        return arr

    def assemble(self, factors, num_vars: int, disable_inlier_ratio: float = 1.0, stream=None):
        """MultiViewICPFactor_ / MultiViewCTICPFactor_ block updates of the last run, on the
        device (kds_batch_assemble).  factors: (job, [vars]) pairs.  Returns (block_rc (K,2),
        H_blocks (K,6,6), b (num_vars,6), enabled (num_factors,))."""
        fa = (L.Factor * len(factors))()
        for f, (job, vs) in enumerate(factors):
            fa[f].job = job
            fa[f].var[:] = list(vs) + [-1] * (4 - len(vs))
        nb = C.c_int32(0)
        _check(_lib.kds_batch_assemble(self._h, fa, len(factors), num_vars, disable_inlier_ratio, stream,
                                       C.byref(nb), None, None, None, None), "kds_batch_assemble")
        rc = np.zeros((nb.value, 2), np.int32)
        H = np.zeros((nb.value, 6, 6))
        b = np.zeros((num_vars, 6))
        en = np.zeros(len(factors), np.int32)
        _check(_lib.kds_batch_assemble(self._h, fa, len(factors), num_vars, disable_inlier_ratio, stream,
                                       C.byref(nb), rc.ctypes.data, H.ctypes.data, b.ctypes.data, en.ctypes.data),
               "kds_batch_assemble")
        return rc, H, b, en.astype(bool)


# ---------------------------------------------------------------------------- serving
class Server:
    """Served registration for many sensor streams (kds_server_*).

    Streams are added with their initial map before start(); requests are submitted
    with an arrival time (seconds after start).  The host arrays of a request are kept
    alive by this object until the server is freed.  serial=True runs the plain
    drop-in: one request at a time through the per-call API.
    """

    def __init__(self, tree=None, icp=None, ct=None, **params):
        p = L.ServerParams()
        _lib.kds_server_params_default(C.byref(p))
        for k, v in params.items():
            if not hasattr(p, k):
                raise AttributeError(f"Server has no parameter {k}")
            setattr(p, k, v)
        for name, kw in (("tree", tree), ("icp", icp), ("ct", ct)):
            for k, v in (kw or {}).items():
                setattr(getattr(p, name), k, v)
        self.params = p
        h = C.c_void_p()
        _check(_lib.kds_server_create(C.byref(p), C.byref(h)), "kds_server_create")
        self._h = h
        self._keep = []

    def __del__(self):
        if _lib is not None:  # None once the interpreter tears the module down
            self.free()

    def free(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.kds_server_free(self._h)
            self._h = C.c_void_p(None)
        self._keep = []

    def add_stream(self, map_xyz, max_scan_points: int) -> int:
        m = np.ascontiguousarray(map_xyz, np.float32).reshape(-1, 3)
        sid = C.c_int32()
        _check(_lib.kds_server_add_stream(self._h, m.ctypes.data, len(m), int(max_scan_points), C.byref(sid)),
               "kds_server_add_stream")
        return sid.value

    def submit(self, stream: int, kind: int, xyz, stamps=None, X0=None, v0=None, arrival: float = 0.0) -> int:
        """xyz/stamps: numpy arrays, or torch tensors (device or pinned host memory)."""
        r = L.Request()
        if hasattr(xyz, "data_ptr"):  # torch tensor: float32 [n, 3] and float64 [n], contiguous
            assert xyz.is_contiguous() and (stamps is None or stamps.is_contiguous())
            self._keep.append((xyz, stamps))
            r.n = int(xyz.shape[0])
            r.xyz = xyz.data_ptr()
            r.stamps = None if stamps is None else stamps.data_ptr()
        else:
            x = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
            st = None if stamps is None else np.ascontiguousarray(stamps, np.float64)
            self._keep.append((x, st))
            r.n = len(x)
            r.xyz = x.ctypes.data
            r.stamps = None if st is None else st.ctypes.data
        r.stream = stream
        r.type = kind
        r.X0[:] = list(_pose12(identity() if X0 is None else X0))
        r.v0[:] = list(np.zeros(6) if v0 is None else np.asarray(v0, np.float64))
        r.arrival = float(arrival)
        t = C.c_int64()
        _check(_lib.kds_server_submit(self._h, C.byref(r), C.byref(t)), "kds_server_submit")
        return t.value

    def start(self) -> None:
        _check(_lib.kds_server_start(self._h), "kds_server_start")

    def drain(self, timeout: float = 0.0) -> None:
        _check(_lib.kds_server_drain(self._h, float(timeout)), "kds_server_drain")

    def result(self, ticket: int, timeout: float = 0.0) -> dict:
        r = L.Result()
        _check(_lib.kds_server_wait(self._h, int(ticket), float(timeout), C.byref(r)), "kds_server_wait")
        return {"status": r.status, "result": r.result, "iterations": r.iterations, "map_version": r.map_version,
                "stats": r.stats.as_dict(), "X": np.array(r.X[:]).reshape(3, 4), "v": np.array(r.v[:]),
                "t_arrival": r.t_arrival, "t_admit": r.t_admit, "t_built": r.t_built, "t_done": r.t_done}

    def trace(self) -> np.ndarray:
        """Timeline rows (kind, count, begin_s, end_s): kind 0 build pass, 1 tick."""
        n = C.c_int32()
        _check(_lib.kds_server_get_trace(self._h, None, 0, C.byref(n)), "kds_server_get_trace")
        out = np.zeros((max(n.value, 1), 4))
        _check(_lib.kds_server_get_trace(self._h, out.ctypes.data, n.value, C.byref(n)), "kds_server_get_trace")
        return out[:n.value]

    def stats(self) -> dict:
        s = L.ServerStats()
        _check(_lib.kds_server_get_stats(self._h, C.byref(s)), "kds_server_get_stats")
        return s.as_dict()


def make_job(kind: int, fixed: Tree, moving: Tree, params: L.AlignerParams, X=None, fixed_X=None, v=None,
             fixed_v=None, mode: int = L.KDS_JOB_COMPUTE, stats_mode: bool = False) -> L.Job:
    j = L.Job()
    j.type = kind
    j.mode = mode
    j.stats_mode = 1 if stats_mode else 0
    j.fixed = fixed.handle.value
    j.moving = moving.handle.value
    j.params = params
    j.X[:] = list(_pose12(identity() if X is None else X))
    j.fixed_X[:] = list(_pose12(identity() if fixed_X is None else fixed_X))
    j.v[:] = list(np.zeros(6) if v is None else np.asarray(v, np.float64))
    j.fixed_v[:] = list(np.zeros(6) if fixed_v is None else np.asarray(fixed_v, np.float64))
    return j


def aligner_params(**kw) -> L.AlignerParams:
    p = L.AlignerParams()
    _lib.kds_aligner_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def voxel_params(**kw) -> L.VoxelParams:
    p = L.VoxelParams()
    _lib.kds_voxel_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def voxelize(xyz, stamps=None, msg_t: float = 0.0, scan_duration: float = 0.0, stream=None, **params):
    """toPointsVector + Voxelizer_::voxelize (kds_points_voxelize).  xyz (n, 3) float32 and
    stamps (n,) float64 (or None) as numpy arrays (host) or CUDA tensors (device); params
    are Voxelizer_'s (range_min, range_max, space_res, time_res, use_boundary).  Returns
    (xyz, stamps) of the kept points or voxel means, of the same kind as the inputs."""
    prm = voxel_params(**params)
    n = C.c_int64(0)
    if hasattr(xyz, "is_cuda") and xyz.is_cuda:
        import torch
        x = xyz.contiguous().to(torch.float32)
        st = None if stamps is None else stamps.contiguous().to(torch.float64)
        ox = torch.empty_like(x)
        ost = torch.empty(len(x), dtype=torch.float64, device=x.device)
        _check(_lib.kds_points_voxelize(x.data_ptr(), None if st is None else st.data_ptr(), len(x),
                                        L.KDS_MEM_DEVICE, msg_t, scan_duration, C.byref(prm), stream, ox.data_ptr(),
                                        ost.data_ptr(), C.byref(n)), "kds_points_voxelize")
        return ox[:n.value], ost[:n.value]
    x = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    st = None if stamps is None else np.ascontiguousarray(stamps, np.float64)
    ox = np.zeros_like(x)
    ost = np.zeros(len(x))
    _check(_lib.kds_points_voxelize(x.ctypes.data, _ptr(st), len(x), L.KDS_MEM_HOST, msg_t, scan_duration,
                                    C.byref(prm), stream, ox.ctypes.data, ost.ctypes.data, C.byref(n)),
           "kds_points_voxelize")
    return ox[:n.value].copy(), ost[:n.value].copy()


def tree_params(**kw) -> L.TreeParams:
    p = L.TreeParams()
    _lib.kds_tree_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


__all__ = ["Tree", "TreeGeneratorB2003D", "ICPB2003D", "CTICPB2003D", "Batch", "Server", "make_job", "aligner_params",
           "tree_params", "identity", "init", "KdsError"]
