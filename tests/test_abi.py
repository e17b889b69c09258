"""The drop-in boundary: libkds.so loads without a GPU and exports every entry point
declared in include/kds.h; the ctypes struct mirrors have the header's layout."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(kds_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_loads_and_exports_every_declared_symbol():
    from kd_slam2_b200 import abi as _lib
    lib = C.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and every declared function has a ctypes signature in the binding
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_struct_layouts():
    from kd_slam2_b200 import abi as L
    assert C.sizeof(L.TreeParams) == 40
    assert C.sizeof(L.AlignerParams) == 40
    assert C.sizeof(L.Stats) == 36
    # kds_job: 4 ints, 2 pointers, params, 36 doubles, 2 ints, stats, 144+12+36+6+36+36 doubles
    assert L.Job.X.offset == 4 * 4 + 2 * 8 + 40
    assert L.Job.result.offset == L.Job.X.offset + 36 * 8
    assert L.Job.H.offset % 8 == 0
    # kds_kdnode3f / kds_kdtree3f: kd_slam2_msgs/msg/KDNode3f.msg and KDTree3f.msg, field for
    # field in message order (the generated C++ struct layout: 56-byte nodes)
    node_fields = [("mean", C.c_float * 3), ("direction", C.c_float * 3), ("idx_start", C.c_uint32),
                   ("idx_end", C.c_uint32), ("idx_left", C.c_int32), ("idx_right", C.c_int32),
                   ("dts_mean", C.c_double), ("dts_covariance", C.c_double)]
    assert [(n, C.sizeof(t)) for n, t in L.KDNode3f._fields_] == [(n, C.sizeof(t)) for n, t in node_fields]
    assert C.sizeof(L.KDNode3f) == 56 and L.KDNode3f.dts_mean.offset == 40
    assert L.KDNODE3F_DTYPE.itemsize == 56
    assert all(L.KDNODE3F_DTYPE.fields[n][1] == getattr(L.KDNode3f, n).offset for n, _ in node_fields)
    assert C.sizeof(L.KDTree3f) == 88 and L.KDTree3f.num_nodes.offset == 72


def test_defaults_match_reference_params():
    from kd_slam2_b200 import tree_params, aligner_params
    import math
    tp = tree_params()
    # TreeGenerator_ PARAM defaults, kd/tree/tree_generator_.h:18-25
    assert (tp.propagate_normal, tp.tree_min_good_leaves, tp.leaf_min_points, tp.leaf_max_points) == (0, 10, 5, 30)
    assert tp.leaf_density == pytest.approx(100.0)
    assert tp.leaf_min_normal_incidence == pytest.approx(0.1)
    assert tp.leaf_normal_eigenratio == pytest.approx(0.1)
    ap = aligner_params()
    # TreeAlignerBase_ PARAM defaults, kd/icp/tree_aligner_base_.h:39-47; CT velocity_damping kd/cticp/cticp_.h:61
    assert ap.kernel_threshold == pytest.approx(0.1)
    assert ap.damping == pytest.approx(1.0)
    assert ap.max_error == pytest.approx(1.0)
    assert ap.min_normal_cos == pytest.approx(math.cos(25 / 180 * math.pi), rel=1e-7)
    assert (ap.min_good_measurements, ap.max_iterations, ap.term_crit) == (10, 20, 0)
    assert ap.velocity_damping == pytest.approx(100.0)
    # TrackerProc_ PARAMs (kd/tracker/tracker_proc_.h:55-60): motion_model defaults to
    # ZeroVelMotionModel_; ConstVelMotionModel_ motion_model_alpha 0.9
    import ctypes
    from kd_slam2_b200 import abi as L, lib
    tr = L.TrackerParams()
    lib().kds_tracker_params_default(ctypes.byref(tr))
    assert (tr.aligner_type, tr.motion_model) == (L.KDS_CTICP, L.KDS_MOTION_ZERO_VEL)
    assert (tr.min_inlier_frac, tr.max_kf_trans, tr.max_kf_rot_deg) == pytest.approx((0.6, 3.0, 360.0))
    assert tr.motion_model_alpha == pytest.approx(0.9)
    assert tr.aligner.max_iterations == ap.max_iterations


def test_calls_without_a_device_fail_with_a_status_not_a_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    from kd_slam2_b200 import abi as L, lib
    h = C.c_void_p()
    rc = lib().kds_aligner_create(0, None, C.byref(h))
    assert rc == L.KDS_ERR_NO_DEVICE
    tp = L.TrackerParams()
    lib().kds_tracker_params_default(C.byref(tp))
    assert lib().kds_tracker_create(C.byref(tp), None, C.byref(h)) == L.KDS_ERR_NO_DEVICE and not h.value
    assert b"device" in lib().kds_last_error()
    # argument checks come before any device use
    xp = (C.c_void_p * 1)(None)
    counts = (C.c_int64 * 1)(-1)
    hs = (C.c_void_p * 1)()
    st = (C.c_int32 * 1)()
    assert lib().kds_tree_build_batch_gather(xp, None, counts, 1, None, None, hs, st) == L.KDS_ERR_INVALID_ARG
    assert lib().kds_tracker_add_frames(None, None, None, None, 1, None, None, None, None) == L.KDS_ERR_INVALID_ARG
    assert lib().kds_tracker_add_frames(None, None, None, None, 0, None, None, None, None) == L.KDS_OK


def test_struct_layouts_match_the_c_header(tmp_path):
    """The ctypes mirrors against the C compiler's own sizeof/offsetof of include/kds.h."""
    import shutil
    import subprocess
    from kd_slam2_b200 import abi as L
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    checks = [("kds_tracker_params", L.TrackerParams, ["aligner", "motion_model", "max_kf_rot_deg"]),
              ("kds_tracker_result", L.TrackerResult, ["frame_duration", "pose_in_kf", "velocity", "stats"]),
              ("kds_tracker_state", L.TrackerState, ["last_ts", "T_delta_log", "pose_global", "has_keyframe"]),
              ("kds_aligner_params", L.AlignerParams, ["velocity_damping", "d_score"]),
              ("kds_stats", L.Stats, ["chi2", "pert_vel_norm"])]
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "kds.h"', "int main(void) {"]
    for cname, _, fields in checks:
        lines.append(f'  printf("%zu\\n", sizeof({cname}));')
        lines += [f'  printf("%zu\\n", offsetof({cname}, {f}));' for f in fields]
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True, capture_output=True, text=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = []
    for _, ct, fields in checks:
        want.append(C.sizeof(ct))
        want += [getattr(ct, f).offset for f in fields]
    assert got == want
