"""CPU restatement of the tracker step -- TEST INFRASTRUCTURE ONLY.

Imported by tests/ as the checker of kds_tracker_add_frame; never part of the product
path.  It follows, step for step:

  TrackerProc_::addFrame       kd/tracker/tracker_proc_frame_impl_.h:33-115
  shouldSwitchKeyframe         kd/tracker/tracker_proc_frame_impl_.h:118-123
  SLAMProc_::addFrame          kd/slam/slam_proc_frame_impl_.h:8-49 (no relocalisation,
                               loop search or pose graph: a switch makes a keyframe)
  SLAMProc_::addKeyframe       kd/slam/slam_proc_frame_impl_.h:73-138 (tracker part)
  ZeroVelMotionModel_          kd/motion_model/zero_vel_motion_model_.h:13-35
  ConstVelMotionModel_         kd/motion_model/const_vel_motion_model_.h:21-45
  Frame::applyVelocity         kd/map/map_.h:103-110
  alignFrames                  kd/map/map_align_utils_.h:10-31

with the alignment and the tree morphs done by the oracle's aligner and tree
(liborc.so) and the pose arithmetic in FP64 (Python floats), in the same evaluation
order as the library's host code.
"""
from __future__ import annotations

import math

import numpy as np

from . import orc


def _iso_identity():
    return [1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0]


def iso_mul(A, B):
    C = [0.0] * 12
    for r in range(3):
        a = A[4 * r:4 * r + 4]
        for c in range(4):
            s = a[0] * B[c] + a[1] * B[4 + c] + a[2] * B[8 + c]
            C[4 * r + c] = s + a[3] if c == 3 else s
    return C


def iso_inv(A):
    C = [0.0] * 12
    for r in range(3):
        for c in range(3):
            C[4 * r + c] = A[4 * c + r]
    for r in range(3):
        C[4 * r + 3] = -(C[4 * r] * A[3] + C[4 * r + 1] * A[7] + C[4 * r + 2] * A[11])
    return C


def rodrigues(w):
    """rodrigues(w), kd/utils/geometry_3d_impl_.h:37-46 (row-major 3x3)."""
    angle = math.sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2])
    R = [1.0 if i % 4 == 0 else 0.0 for i in range(9)]
    if angle < 1e-9:
        return R
    inv = 1.0 / angle
    n = [w[0] * inv, w[1] * inv, w[2] * inv]
    S = [0.0, -n[2], n[1], n[2], 0.0, -n[0], -n[1], n[0], 0.0]
    S2 = [S[3 * i] * S[j] + S[3 * i + 1] * S[3 + j] + S[3 * i + 2] * S[6 + j] for i in range(3) for j in range(3)]
    s, omc = math.sin(angle), 1.0 - math.cos(angle)
    return [(R[i] + s * S[i]) + omc * S2[i] for i in range(9)]


def expmap(v):
    """expmap, kd/utils/geometry_3d_impl_.h:176-184: t = v[0:3], R = rodrigues(v[3:6])."""
    R = rodrigues(v[3:6])
    X = [0.0] * 12
    for r in range(3):
        X[4 * r:4 * r + 3] = R[3 * r:3 * r + 3]
        X[4 * r + 3] = v[r]
    return X


def logmap(X):
    """logmap = [t, logSO3(R)], kd/utils/geometry_3d_impl_.h:48-59."""
    cos_a = 0.5 * (((X[0] + X[5]) + X[10]) - 1.0)
    cos_a = max(-1.0, min(1.0, cos_a))
    angle = math.acos(cos_a)
    ax = [X[9] - X[6], X[2] - X[8], X[4] - X[1]]
    f = 0.5 if angle < 1e-7 else angle / (2.0 * math.sin(angle))
    return [X[3], X[7], X[11], ax[0] * f, ax[1] * f, ax[2] * f]


def rotation_angle(X):
    """Eigen::AngleAxis(R).angle() (kd/utils/geometry_3d_.h:83-85): quaternion by Shepperd's
    method, then 2 atan2(|q.xyz|, |q.w|)."""
    def M(i, j):
        return X[4 * i + j]
    q = [0.0, 0.0, 0.0, 0.0]
    tr = (M(0, 0) + M(1, 1)) + M(2, 2)
    if tr > 0.0:
        t = math.sqrt(tr + 1.0)
        q[3] = 0.5 * t
        t = 0.5 / t
        q[0] = (M(2, 1) - M(1, 2)) * t
        q[1] = (M(0, 2) - M(2, 0)) * t
        q[2] = (M(1, 0) - M(0, 1)) * t
    else:
        i = 0
        if M(1, 1) > M(0, 0):
            i = 1
        if M(2, 2) > M(i, i):
            i = 2
        j, k = (i + 1) % 3, (i + 2) % 3
        t = math.sqrt(((M(i, i) - M(j, j)) - M(k, k)) + 1.0)
        q[i] = 0.5 * t
        t = 0.5 / t
        q[3] = (M(k, j) - M(j, k)) * t
        q[j] = (M(j, i) + M(i, j)) * t
        q[k] = (M(k, i) + M(i, k)) * t
    n = math.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2])
    return 0.0 if n == 0.0 else 2.0 * math.atan2(n, abs(q[3]))


class OTracker:
    """The tracker step over oracle trees.  kind: orc.KIND_ICP / orc.KIND_CT;
    const_vel: ConstVelMotionModel_ (else ZeroVelMotionModel_)."""

    def __init__(self, kind: int, params: orc.AlignParams, const_vel: bool = False, alpha: float = 0.9,
                 min_inlier_frac: float = 0.6, max_kf_trans: float = 3.0, max_kf_rot_deg: float = 360.0,
                 mode: int = orc.MODE_MIXED):
        self.kind, self.params, self.mode = kind, params, mode
        self.const_vel = const_vel
        self.alpha = float(np.float32(alpha))
        self.min_inlier_frac = np.float32(min_inlier_frac)
        self.max_kf_trans = float(np.float32(max_kf_trans))
        self.max_kf_rot_rad = float(np.float32(np.float32(max_kf_rot_deg) * np.float32(math.pi / 180.0)))
        self.keyframe = None
        self.kf_pose_in_world = _iso_identity()
        self.pose_in_kf = _iso_identity()
        self.last_ts = -1.0
        self.frame_duration = 0.0
        self.T_delta_log = [0.0] * 6
        self.frame_idx = 0
        self.keyframe_count = 0

    def _apply_velocity(self, tree: orc.OTree, v) -> None:
        if any(x != 0.0 for x in v):
            tree.apply_velocities_in_place(np.array(v, np.float64).astype(np.float32))

    def _should_switch(self, X, st) -> bool:
        leaves = st["num_inliers"] + st["num_outliers"] + st["num_bad"] + st["num_err_normal"] + st["num_err_fn"]
        ratio = np.float32(st["num_inliers"]) / np.float32(leaves) if leaves else np.float32(0)
        tn = math.sqrt(X[3] * X[3] + X[7] * X[7] + X[11] * X[11])
        return bool(ratio < self.min_inlier_frac) or tn > self.max_kf_trans or \
            abs(rotation_angle(X)) > self.max_kf_rot_rad

    def _make_keyframe(self, tree: orc.OTree, pose_in_world) -> None:
        self.keyframe = tree.clone()
        self.kf_pose_in_world = list(pose_in_world)
        self.pose_in_kf = _iso_identity()
        self.keyframe_count += 1

    def add_frame(self, tree: orc.OTree, ts: float, T_base_lidar=None) -> dict:
        """One step; tree is transformed in place.  Returns the fields of kds_tracker_result."""
        if T_base_lidar is not None:
            tree.apply_isometry_in_place(np.asarray(T_base_lidar, np.float64).reshape(3, 4).astype(np.float32))
        out = {"frame_idx": self.frame_idx, "result": -1, "new_keyframe": False, "ct_velocity": [0.0] * 6}
        prev = list(self.pose_in_kf)
        self.frame_duration = 0.0 if self.last_ts < 0 else ts - self.last_ts
        self.last_ts = ts
        out["frame_duration"] = self.frame_duration
        vel = [0.0] * 6
        if self.frame_duration > 0:
            vl = self.T_delta_log if self.const_vel else [0.0] * 6
            vel = [vl[i] / self.frame_duration for i in range(6)]
            self._apply_velocity(tree, vel)
        out["velocity"] = vel
        if self.keyframe is None:
            self._make_keyframe(tree, _iso_identity())
            out.update(status=0, new_keyframe=True, keyframe_count=self.keyframe_count,
                       pose_in_kf=_iso_identity(), pose_in_world=_iso_identity(), stats=None)
            self.frame_idx += 1
            return out
        pred = expmap(self.T_delta_log) if self.const_vel else _iso_identity()
        X0 = iso_mul(self.pose_in_kf, pred)
        r = orc.align(self.kind, self.mode, self.keyframe, tree, self.params, np.array(X0).reshape(3, 4),
                      v0=np.zeros(6) if self.kind == orc.KIND_CT else None)
        X = [float(x) for x in np.asarray(r["X"]).reshape(12)]
        out["result"] = r["ret"]
        out["stats"] = r["stats"]
        if not all(math.isfinite(x) for x in X):
            raise FloatingPointError("divergence")
        self.pose_in_kf = X
        pose_in_world = iso_mul(self.kf_pose_in_world, X)
        if self.const_vel:
            dv = logmap(iso_mul(iso_inv(prev), X))
            self.T_delta_log = [self.alpha * self.T_delta_log[i] + (1.0 - self.alpha) * dv[i] for i in range(6)]
        if self.kind == orc.KIND_CT:
            cv = [float(x) for x in r["v"]]
            self._apply_velocity(tree, cv)
            out["ct_velocity"] = cv
        out.update(status=1, pose_in_kf=X, pose_in_world=pose_in_world)
        if self._should_switch(X, r["stats"]):
            self._make_keyframe(tree, pose_in_world)
            out["new_keyframe"] = True
        out["keyframe_count"] = self.keyframe_count
        self.frame_idx += 1
        return out
