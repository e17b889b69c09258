"""Seeded bundle-adjustment pair workload: keyframes along a closed loop, each with its
own surfel KD-tree, and the overlapping keyframe pairs that a multi-view BA factor
graph would linearize (MultiViewICPFactor_ / MultiViewCTICPFactor_ call
buildQuadraticForm once per pair, kd/map/multiview_icp_factor_impl_.h:10-62).

The loop is a stadium-shaped 2 km track: two parallel straights 20 m apart joined by
half circles.  A keyframe every 10 m (200 keyframes); each is a 128 x 2048 sweep (a
deskewed keyframe: the sensor pose is fixed over the sweep, the points keep their
firing stamps), cut to a log-uniform size in [20k, 260k] points.  Boxes stand along both sides of the track.  A pair is two keyframes closer
than 30 m; each pair is aligned rigidly (ICP) and with CT-ICP from a perturbed relative
pose, moving = the later keyframe, fixed = the earlier one.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import synth
from .streams import compose

SPACING = 10.0
LANE_GAP = 20.0
LOOP_LEN = 2000.0


@dataclass
class Keyframe:
    X: np.ndarray      # pose at the sweep start (world <- sensor)
    vel: np.ndarray    # body velocity [v; w]
    xyz: np.ndarray
    stamps: np.ndarray


@dataclass
class Pair:
    i: int             # fixed keyframe
    j: int             # moving keyframe
    kind: int          # 0 ICP, 1 CT-ICP
    X0: np.ndarray     # initial guess of the moving keyframe in the fixed keyframe's frame
    X_true: np.ndarray


@dataclass
class Workload:
    keyframes: list = field(default_factory=list)
    pairs: list = field(default_factory=list)


def track_pose(s: float):
    """Position and heading at arc length s on the stadium track (straights along x)."""
    r = LANE_GAP / 2.0
    straight = (LOOP_LEN - 2 * np.pi * r) / 2.0
    s = s % LOOP_LEN
    if s < straight:
        return np.array([s, 0.0]), 0.0
    s -= straight
    if s < np.pi * r:
        a = s / r
        return np.array([straight + r * np.sin(a), r - r * np.cos(a)]), a
    s -= np.pi * r
    if s < straight:
        return np.array([straight - s, LANE_GAP]), np.pi
    s -= straight
    a = s / r
    return np.array([-r * np.sin(a), LANE_GAP - (r - r * np.cos(a))]), np.pi + a


def make_boxes(rng, n_boxes: int = 1600):
    """Boxes on both sides of the track, outside a 6 m road band around each lane."""
    out = []
    r = LANE_GAP / 2.0
    straight = (LOOP_LEN - 2 * np.pi * r) / 2.0
    while len(out) < n_boxes:
        x = rng.uniform(-60.0, straight + 60.0)
        y = rng.uniform(-60.0, LANE_GAP + 60.0)
        # distance to the track centre lines
        if -6.0 < y < 6.0 or LANE_GAP - 6.0 < y < LANE_GAP + 6.0:
            continue
        if 0.0 < y < LANE_GAP and -r - 6 < x < straight + r + 6:
            continue  # median between the lanes stays empty
        sx, sy, h = rng.uniform(1.0, 8.0), rng.uniform(1.0, 8.0), rng.uniform(2.0, 15.0)
        out.append([x - sx / 2, y - sy / 2, 0.0, x + sx / 2, y + sy / 2, h])
    return np.array(out)


def make_workload(seed: int = 4, num_keyframes: int = 200, radius: float = 30.0, min_pts: int = 20000,
                  max_pts: int = 260000, beams: int = 128, cols: int = 2048, guess_t: float = 0.1,
                  guess_deg: float = 1.0, threads: int = 16) -> Workload:
    rng = np.random.default_rng(seed)
    boxes = make_boxes(rng)
    wl = Workload()
    for k in range(num_keyframes):
        pos, yaw = track_pose(k * SPACING)
        X = synth.pose((pos[0], pos[1], 1.8), (0.0, 0.0, yaw))
        vel = np.zeros(6)
        near = boxes[np.hypot((boxes[:, 0] + boxes[:, 3]) / 2 - pos[0], (boxes[:, 1] + boxes[:, 4]) / 2 - pos[1]) < 75]
        xyz, st = synth.scan(near, X, vel, beams=beams, cols=cols, elev=(-22.5, 22.5), seed=seed * 7919 + k,
                             threads=threads)
        target = int(np.exp(rng.uniform(np.log(min_pts), np.log(max_pts))))
        if len(xyz) > target:
            keep = np.sort(rng.choice(len(xyz), target, replace=False))
            xyz, st = xyz[keep], st[keep]
        wl.keyframes.append(Keyframe(X=X, vel=vel, xyz=np.ascontiguousarray(xyz), stamps=np.ascontiguousarray(st)))
    P = np.array([kf.X[:2, 3] for kf in wl.keyframes])
    for i in range(num_keyframes):
        for j in range(i + 1, num_keyframes):
            if np.linalg.norm(P[i] - P[j]) >= radius:
                continue
            Xi, Xj = wl.keyframes[i].X, wl.keyframes[j].X
            Ri = Xi[:, :3]
            T = np.zeros((3, 4))
            T[:, :3] = Ri.T @ Xj[:, :3]
            T[:, 3] = Ri.T @ (Xj[:, 3] - Xi[:, 3])
            for kind in (0, 1):
                d = rng.normal(size=3)
                d /= np.linalg.norm(d)
                a = rng.normal(size=3)
                a /= np.linalg.norm(a)
                E = synth.pose(guess_t * d, np.deg2rad(guess_deg) * a)
                wl.pairs.append(Pair(i=i, j=j, kind=kind, X0=compose(T, E), X_true=T))
    return wl


def build_trees(wl: Workload, tree_params: dict, stream=None, inputs=None):
    """All keyframe trees in one batched build pass (stamps kept: CT pairs deskew).
    inputs: the keyframes already on the device, as returned by device_inputs (the pass
    then reads device memory); otherwise the host arrays are gathered and copied."""
    import ctypes as C

    from . import Tree, TreeGeneratorB2003D, _check, lib, tree_params as tp
    from .abi import KDS_MEM_DEVICE, KDS_OK
    if inputs is None:
        gen = TreeGeneratorB2003D(**tree_params)
        return gen.make_trees([(kf.xyz, kf.stamps) for kf in wl.keyframes], stream=stream)
    xyz, st, off = inputs
    R = len(off) - 1
    hs = (C.c_void_p * R)()
    status = (C.c_int32 * R)()
    prm = tp(**tree_params)
    _check(lib().kds_tree_build_batch(xyz.data_ptr(), st.data_ptr(), off.ctypes.data, R, KDS_MEM_DEVICE,
                                      C.byref(prm), stream, hs, status), "kds_tree_build_batch")
    return [Tree(hs[i]) if status[i] == KDS_OK else None for i in range(R)]


def device_inputs(wl: Workload):
    """The keyframes' points and stamps back to back in device memory, with their offsets."""
    import torch
    xyz = torch.from_numpy(np.ascontiguousarray(np.concatenate([kf.xyz for kf in wl.keyframes]))).cuda()
    st = torch.from_numpy(np.ascontiguousarray(np.concatenate([kf.stamps for kf in wl.keyframes]))).cuda()
    off = np.zeros(len(wl.keyframes) + 1, np.int64)
    off[1:] = np.cumsum([len(kf.xyz) for kf in wl.keyframes])
    return xyz, st, off


def jobs(wl: Workload, trees, icp_params: dict, ct_params: dict):
    """One kds_job per pair and kind."""
    from . import aligner_params, make_job
    from .abi import KDS_CTICP, KDS_ICP
    pi, pc = aligner_params(**icp_params), aligner_params(**ct_params)
    out = []
    for p in wl.pairs:
        kf_i, kf_j = wl.keyframes[p.i], wl.keyframes[p.j]
        if p.kind == 0:
            out.append(make_job(KDS_ICP, trees[p.i], trees[p.j], pi, X=p.X0))
        else:
            out.append(make_job(KDS_CTICP, trees[p.i], trees[p.j], pc, X=p.X0, v=kf_j.vel, fixed_v=kf_i.vel))
    return out


def factor_jobs(wl: Workload, trees, icp_params: dict, ct_params: dict, X=None, v=None):
    """The linearizations of one bundle-adjustment step: per pair, the rigid factor
    (MultiViewICPFactor_: buildQuadraticForm at the two keyframes' world poses) and the
    continuous-time factor (MultiViewCTICPFactor_: buildQuadraticFormDual at the poses
    and velocities).  X, v: per-keyframe estimates (default: the keyframes' own).
    Variables: pose of keyframe k = 2k, its velocity = 2k + 1.
    Returns (jobs, factors as (job, vars), number of variables)."""
    from . import aligner_params, make_job
    from .abi import KDS_CTICP, KDS_ICP, KDS_JOB_LINEARIZE, KDS_JOB_LINEARIZE_DUAL
    X = [kf.X for kf in wl.keyframes] if X is None else X
    v = [kf.vel for kf in wl.keyframes] if v is None else v
    pi, pc = aligner_params(**icp_params), aligner_params(**ct_params)
    jobs, factors = [], []
    for p in wl.pairs:
        i, j = p.i, p.j
        if p.kind == 0:
            jobs.append(make_job(KDS_ICP, trees[i], trees[j], pi, X=X[j], fixed_X=X[i], mode=KDS_JOB_LINEARIZE))
            factors.append((len(jobs) - 1, [2 * i, 2 * j]))
        else:
            jobs.append(make_job(KDS_CTICP, trees[i], trees[j], pc, X=X[j], fixed_X=X[i], v=v[j], fixed_v=v[i],
                                 mode=KDS_JOB_LINEARIZE_DUAL))
            factors.append((len(jobs) - 1, [2 * i, 2 * i + 1, 2 * j, 2 * j + 1]))
    return jobs, factors, 2 * len(wl.keyframes)
