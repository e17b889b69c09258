"""The tracker step (kds_tracker_add_frame) against the oracle's restatement of
TrackerProc_::addFrame + SLAMProc_'s keyframe switch (oracle/tracker.py).

A seeded trajectory through the box scene (2 m/s forward, 0.1 rad/s yaw, 0.1 s scans
that start where the previous one ended, in-scan motion included) is tracked by the
library and by the oracle frame by frame.  Both build the same trees (bit-identical
builds), so the chains differ only by the aligner's floating-point differences
(within 1e-5 per alignment); they compound through the morphs and keyframes, so the
per-frame poses are compared at 1e-4 m / rad.  Keyframe decisions, result codes and
frame durations must be identical: the trajectory keeps every decision well away from
its threshold (translation switches at about 0.57 m against max_kf_trans 0.5; inlier
ratios 0.67-0.77 against min_inlier_frac 0.3).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import pose_err
from oracle import orc
from oracle.tracker import OTracker

pytestmark = pytest.mark.gpu

POSE_TOL_CHAIN = 1e-4  # m and rad, per frame along the chain
VEL_TOL = 1e-3         # m/s and rad/s
TREE_P = dict(leaf_max_points=16)


def trajectory(scene, n, vel=(2.0, 0.1, 0.0, 0.0, 0.0, 0.1), seed=50):
    from kd_slam2_b200 import streams, synth
    v = np.asarray(vel, np.float64)
    P = synth.pose((0.0, 0.0, 1.8))
    M = streams.motion(v, 0.1)
    for k in range(n):
        xyz, st = synth.scan(scene, P, vel=v, beams=16, cols=1024, seed=seed + k, t_start=0.1 * k)
        yield 0.1 * k, xyz, st
        P = streams.compose(P, M)


def run_both(scene, n, kind, const_vel, T_base_lidar=None, vel=(2.0, 0.1, 0.0, 0.0, 0.0, 0.1), **tp):
    import kd_slam2_b200 as kds
    P = dict(max_error=0.5, max_iterations=10)
    if kind == orc.KIND_CT:
        P["velocity_damping"] = 100.0
        aligner = kds.CTICPB2003D(**P)
    else:
        aligner = kds.ICPB2003D(**P)
    mm = kds.ConstVelMotionModel3D(0.9) if const_vel else kds.ZeroVelMotionModel3D()
    trk = kds.Tracker3D(odom_aligner=aligner, motion_model=mm, **tp)
    otrk = OTracker(kind, orc.align_params(**P), const_vel=const_vel, alpha=0.9, **tp)
    gen = kds.TreeGeneratorB2003D(**TREE_P)
    rows = []
    for ts, xyz, st in trajectory(scene, n, vel=vel):
        G = gen.make_tree(xyz, st)
        O = orc.OTree.build(xyz, st, orc.tree_params(**TREE_P))
        rg = trk.add_frame(G, ts, T_base_lidar)
        ro = otrk.add_frame(O, ts, T_base_lidar)
        rows.append((rg, ro, G.export(), O.export()))
    return trk, otrk, rows


def compare(rows):
    for rg, ro, eg, eo in rows:
        k = rg["frame_idx"]
        assert k == ro["frame_idx"]
        assert rg["status"] == ro["status"], k
        assert rg["result"] == ro["result"], k
        assert rg["new_keyframe"] == ro["new_keyframe"], k
        assert rg["keyframe_count"] == ro["keyframe_count"], k
        assert rg["frame_duration"] == ro["frame_duration"], k
        for key in ("pose_in_kf", "pose_in_world"):
            dt, dr = pose_err(rg[key], np.array(ro[key]).reshape(3, 4))
            assert dt <= POSE_TOL_CHAIN and dr <= POSE_TOL_CHAIN, (k, key, dt, dr)
        assert np.abs(rg["velocity"] - np.array(ro["velocity"])).max() <= VEL_TOL, k
        assert np.abs(rg["ct_velocity"] - np.array(ro["ct_velocity"])).max() <= VEL_TOL, k
        if ro["stats"] is not None:
            for f in ("num_inliers", "num_outliers", "num_bad", "num_err_normal", "num_err_fn"):
                assert abs(rg["stats"][f] - ro["stats"][f]) <= 3, (k, f)
        # the frame tree after the step (pre-deskew and CT morphs applied in place)
        assert np.abs(eg["mean"] - eo["mean"]).max() <= 2e-3, k
        assert np.abs(eg["dir"] - eo["dir"]).max() <= 2e-3, k


def test_ct_const_vel_chain_matches_oracle(scene):
    trk, otrk, rows = run_both(scene, 12, orc.KIND_CT, True, max_kf_trans=0.5, min_inlier_frac=0.3)
    compare(rows)
    flags = [r[0]["new_keyframe"] for r in rows]
    assert flags[0] and sum(flags) >= 3, flags           # the chain did switch keyframes
    assert any(np.abs(r[0]["velocity"]).max() > 0.1 for r in rows[2:])   # pre-deskew ran
    assert any(np.abs(r[0]["ct_velocity"]).max() > 1e-3 for r in rows[1:])
    # the tracker's keyframe is a copy of the last switching frame's deskewed tree
    last_kf = max(i for i, r in enumerate(rows) if r[0]["new_keyframe"])
    kf, kf_pose = trk.keyframe()
    assert np.array_equal(kf["mean"], rows[last_kf][2]["mean"])
    assert np.array_equal(kf["dir"], rows[last_kf][2]["dir"])
    assert np.array_equal(kf["left"], rows[last_kf][2]["left"])
    assert np.allclose(kf_pose, rows[last_kf][0]["pose_in_world"], atol=0, rtol=0)
    # poseGlobal: the last frame's pose_in_world; pose_in_kf reset by a switch
    assert np.array_equal(trk.pose_global(), rows[-1][0]["pose_in_world"])
    if rows[-1][0]["new_keyframe"]:
        assert np.array_equal(trk.pose_in_kf(), np.eye(3, 4))
    else:
        assert np.array_equal(trk.pose_in_kf(), rows[-1][0]["pose_in_kf"])


def test_icp_zero_vel_with_base_transform_matches_oracle(scene):
    from kd_slam2_b200 import synth
    T = synth.pose((0.3, -0.1, 0.2), (0.0, 0.02, 0.05))
    trk, otrk, rows = run_both(scene, 6, orc.KIND_ICP, False, T_base_lidar=T, max_kf_trans=0.5,
                               min_inlier_frac=0.3)
    compare(rows)
    for rg, _, _, _ in rows:
        assert not np.any(rg["velocity"]) and not np.any(rg["ct_velocity"])


def test_rotation_switches_keyframes_as_the_oracle_does(scene):
    """A turning trajectory (0.5 rad/s yaw: 2.9 deg per frame) with max_kf_rot_deg 4: the
    rotation test of shouldSwitchKeyframe switches every second frame (5.7 deg), away
    from the threshold; translation and inlier tests stay off."""
    trk, otrk, rows = run_both(scene, 8, orc.KIND_CT, True, vel=(1.0, 0.0, 0.0, 0.0, 0.0, 0.5), max_kf_rot_deg=4.0,
                               max_kf_trans=100.0, min_inlier_frac=0.0)
    compare(rows)
    flags = [r[0]["new_keyframe"] for r in rows]
    assert sum(flags[1:]) >= 3, flags


def test_first_frame_reset_and_argument_errors(scene):
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import abi as L
    gen = kds.TreeGeneratorB2003D(**TREE_P)
    trk = kds.Tracker3D(odom_aligner=kds.ICPB2003D(max_iterations=5), motion_model=kds.ConstVelMotionModel3D())
    assert trk.keyframe()[0] is None
    frames = list(trajectory(scene, 2))
    r0 = trk.add_frame(gen.make_tree(frames[0][1], frames[0][2]), frames[0][0])
    assert (r0["status"], r0["result"], r0["new_keyframe"], r0["frame_duration"]) == (L.KDS_STATUS_INIT, -1, True, 0.0)
    r1 = trk.add_frame(gen.make_tree(frames[1][1], frames[1][2]), frames[1][0])
    assert r1["status"] == L.KDS_STATUS_TRACKING and r1["frame_idx"] == 1
    assert r1["frame_duration"] == pytest.approx(0.1)
    trk.reset()
    assert trk.keyframe()[0] is None
    r2 = trk.add_frame(gen.make_tree(frames[1][1], frames[1][2]), frames[1][0])
    assert r2["status"] == L.KDS_STATUS_INIT and r2["frame_idx"] == 0
    with pytest.raises(kds.KdsError) as ei:
        trk.add_frame(gen.make_tree(frames[0][1], frames[0][2]), float("nan"))
    assert ei.value.code == L.KDS_ERR_INVALID_ARG
    p = L.TrackerParams()
    kds.lib().kds_tracker_params_default(C.byref(p))
    p.motion_model = 7
    h = C.c_void_p()
    assert kds.lib().kds_tracker_create(C.byref(p), None, C.byref(h)) == L.KDS_ERR_INVALID_ARG and not h.value


def test_batched_trackers_equal_sequential_trackers(scene):
    """kds_tracker_add_frames over four streams (two CT-ICP + ConstVel, two ICP + ZeroVel,
    different starts and speeds) gives every tracker exactly what kds_tracker_add_frame
    gives it one frame at a time."""
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import streams, synth
    gen = kds.TreeGeneratorB2003D(**TREE_P)
    P = dict(max_error=0.5, max_iterations=10)

    def make(i):
        if i % 2 == 0:
            al, mm = kds.CTICPB2003D(velocity_damping=100.0, **P), kds.ConstVelMotionModel3D()
        else:
            al, mm = kds.ICPB2003D(**P), kds.ZeroVelMotionModel3D()
        return kds.Tracker3D(odom_aligner=al, motion_model=mm, max_kf_trans=0.5, min_inlier_frac=0.3)

    seqs = []
    for i in range(4):
        v = np.array([1.5 + 0.25 * i, 0.1, 0.0, 0.0, 0.0, 0.05 * (i - 1)])
        Pi = synth.pose((2.0 * i - 3.0, 1.0 - i, 1.8), (0.0, 0.0, 0.3 * i))
        M = streams.motion(v, 0.1)
        frames = []
        for k in range(6):
            xyz, st = synth.scan(scene, Pi, vel=v, beams=16, cols=1024, seed=300 + 10 * i + k, t_start=0.1 * k)
            frames.append((0.1 * k, xyz, st))
            Pi = streams.compose(Pi, M)
        seqs.append(frames)
    seq_trk = [make(i) for i in range(4)]
    bat_trk = [make(i) for i in range(4)]
    batch = kds.Batch()
    for k in range(6):
        single = [seq_trk[i].add_frame(gen.make_tree(seqs[i][k][1], seqs[i][k][2]), seqs[i][k][0]) for i in range(4)]
        trees = [gen.make_tree(seqs[i][k][1], seqs[i][k][2]) for i in range(4)]
        multi, codes = kds.Tracker3D.add_frames(bat_trk, trees, [seqs[i][k][0] for i in range(4)], batch)
        assert list(codes) == [0, 0, 0, 0]
        for i, (a, b) in enumerate(zip(single, multi)):
            for key in ("status", "result", "new_keyframe", "frame_idx", "keyframe_count", "frame_duration",
                        "stats"):
                assert a[key] == b[key], (k, i, key)
            for key in ("pose_in_kf", "pose_in_world", "velocity", "ct_velocity"):
                assert np.array_equal(a[key], b[key]), (k, i, key)
    for a, b in zip(seq_trk, bat_trk):
        assert np.array_equal(a.pose_global(), b.pose_global())
        ka, _ = a.keyframe()
        kb, _ = b.keyframe()
        assert np.array_equal(ka["mean"], kb["mean"])


def test_checkpoint_resume_continues_identically(scene):
    """A tracker checkpointed after five frames (state + keyframe as a KDTree3f message,
    through plain bytes and a pickle) and restored into a new tracker gives the same
    results on the following frames as the original."""
    import pickle

    import kd_slam2_b200 as kds
    gen = kds.TreeGeneratorB2003D(**TREE_P)

    def make():
        return kds.Tracker3D(odom_aligner=kds.CTICPB2003D(max_error=0.5, max_iterations=10, velocity_damping=100.0),
                             motion_model=kds.ConstVelMotionModel3D(), max_kf_trans=0.5, min_inlier_frac=0.3)

    frames = list(trajectory(scene, 9))
    a = make()
    for ts, xyz, st in frames[:5]:
        a.add_frame(gen.make_tree(xyz, st), ts)
    ck = pickle.loads(pickle.dumps(a.checkpoint()))
    b = make()
    b.restore(ck)
    assert np.array_equal(a.pose_global(), b.pose_global())
    for ts, xyz, st in frames[5:]:
        ra = a.add_frame(gen.make_tree(xyz, st), ts)
        rb = b.add_frame(gen.make_tree(xyz, st), ts)
        for key in ("status", "result", "new_keyframe", "frame_idx", "keyframe_count", "stats"):
            assert ra[key] == rb[key], key
        for key in ("pose_in_kf", "pose_in_world", "velocity", "ct_velocity"):
            assert np.array_equal(ra[key], rb[key]), key
    # a state for another motion model is refused
    z = kds.Tracker3D(odom_aligner=kds.CTICPB2003D(), motion_model=kds.ZeroVelMotionModel3D())
    with pytest.raises(kds.KdsError):
        z.restore(ck)
    # so is a state saved under other aligner settings, naming the setting, and the
    # tracker is left as it was
    w = kds.Tracker3D(odom_aligner=kds.CTICPB2003D(max_error=0.5, max_iterations=12, velocity_damping=100.0),
                      motion_model=kds.ConstVelMotionModel3D(), max_kf_trans=0.5, min_inlier_frac=0.3)
    before = w.pose_global()
    with pytest.raises(kds.KdsError, match="max_iterations"):
        w.restore(ck)
    assert np.array_equal(w.pose_global(), before)
