"""The C++ adapter (include/kds.hpp), its .conf reader, and the conf rewrite script.

CPU: the reader takes the PARAM values of a BOSS .conf (term_crit resolved through its
#pointer), and make_b200_confs.sh rewrites CUDA/CPU aligner types to the B200 ones
without touching the values.
GPU: a C++ program using the adapter gives the same CT-ICP result as the Python API on
the same inputs (same library, same kernels: identical).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, make_scan, perturbation

FIXTURE = os.path.join(ROOT, "tests", "golden", "b200_sample.conf")
SCRIPT = os.path.join(ROOT, "kd_slam2_b200", "configs", "make_b200_confs.sh")


@pytest.fixture(scope="module")
def adapter_bin(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    lib_dir = os.path.join(ROOT, "kd_slam2_b200")
    if not os.path.exists(os.path.join(lib_dir, "libkds.so")):
        pytest.fail("libkds.so is not built (python -m kd_slam2_b200.build)")
    out = str(tmp_path_factory.mktemp("adapter") / "adapter_main")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "adapter_main.cpp"), "-L", lib_dir, "-lkds",
           f"-Wl,-rpath,{lib_dir}", "-o", out]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


def parse_conf_output(text):
    rows = {}
    for line in text.strip().splitlines():
        k, *vals = line.split()
        rows[k] = [float(v) for v in vals]
    return rows


def test_conf_reader_takes_the_param_values(adapter_bin):
    r = subprocess.run([adapter_bin, "conf", FIXTURE], check=True, capture_output=True, text=True)
    rows = parse_conf_output(r.stdout)
    # propagate_normal, tree_min_good_leaves, leaf_min_points, leaf_max_points, density, incidence, eig, ratio
    assert rows["tree"] == pytest.approx([0, 10, 5, 16, 100, 0.1, 1e-3, 0.1], rel=1e-6)
    # kernel_threshold, damping, max_error, min_normal_cos, min_good, max_it, vel_damping, term_crit, d_pert, d_score
    assert rows["CTICPB2003D"] == pytest.approx([0.2, 1, 0.5, 0.7, 10, 15, 10, 1, 2e-3, 5e-4], rel=1e-6)
    # a negative #pointer is no criterion; velocity_damping keeps its default (ICP has none)
    assert rows["ICPB2003D"] == pytest.approx([0.1, 2, 3, 0.6, 10, 20, 100, 0, 1e-3, 1e-3], rel=1e-6)


def test_make_b200_confs_renames_types_only(tmp_path, adapter_bin):
    text = open(FIXTURE).read()
    cuda = (text.replace('"CTICPB2003D"', '"CTICPCUDA3D"').replace('"ICPB2003D"', '"ICPCPU3D"')
            .replace('"TreeGeneratorB2003D"', '"TreeGenerator3D"'))
    (tmp_path / "slam.conf").write_text(cuda)
    (tmp_path / "dl.conf").write_text('"ICPCUDA3D" : { }\n')
    (tmp_path / "viewer.conf").write_text('"Viewer" : { "#id" : 1 }\n')
    r = subprocess.run(["bash", SCRIPT, str(tmp_path)], check=True, capture_output=True, text=True)
    assert r.stdout.split() == ["slam_b200.conf"]
    out = (tmp_path / "slam_b200.conf").read_text()
    assert out == text
    r1 = subprocess.run([adapter_bin, "conf", str(tmp_path / "slam_b200.conf")], check=True, capture_output=True,
                        text=True)
    r0 = subprocess.run([adapter_bin, "conf", FIXTURE], check=True, capture_output=True, text=True)
    assert r1.stdout == r0.stdout


def _write_cloud(path, xyz, st):
    with open(path, "wb") as f:
        f.write(np.int64(len(st)).tobytes())
        f.write(np.ascontiguousarray(xyz, np.float32).tobytes())
        f.write(np.ascontiguousarray(st, np.float64).tobytes())


@pytest.mark.gpu
def test_cpp_adapter_matches_python_api(adapter_bin, scene, tmp_path):
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import synth
    vel = np.array([10.0, 0, 0, 0, 0, np.deg2rad(30.0)])
    xf, sf = make_scan(scene, 4100, beams=32)
    xm, sm = make_scan(scene, 4101, beams=32, pose=synth.pose((0.0, 0.0, 1.8)), vel=vel)
    X0 = perturbation(np.random.default_rng(3), 0.2, 2.0)
    v0 = vel * 0.9
    _write_cloud(tmp_path / "f.bin", xf, sf)
    _write_cloud(tmp_path / "m.bin", xm, sm)
    np.asarray(X0, np.float64).reshape(12).tofile(tmp_path / "x0.bin")
    np.asarray(v0, np.float64).tofile(tmp_path / "v0.bin")
    subprocess.run([adapter_bin, "align", FIXTURE, str(tmp_path / "f.bin"), str(tmp_path / "m.bin"),
                    str(tmp_path / "x0.bin"), str(tmp_path / "v0.bin"), str(tmp_path / "out.bin")], check=True,
                   capture_output=True, text=True)
    out = np.fromfile(tmp_path / "out.bin", np.float64)

    gen = kds.TreeGeneratorB2003D(leaf_max_points=16, tree_min_good_leaves=10, propagate_normal=0)
    Gf, Gm = gen.make_tree(xf, sf), gen.make_tree(xm, sm)
    a = kds.CTICPB2003D(kernel_threshold=np.float32(0.200000003), damping=1.0, max_error=0.5,
                        min_normal_cos=np.float32(0.699999988), max_iterations=15, velocity_damping=10.0,
                        term_crit=dict(d_pert=np.float32(0.00200000009), d_score=np.float32(0.000500000024)))
    a.set_fixed(Gf)
    a.set_moving(Gm)
    a.set_x(X0)
    a.set_velocities(v0)
    r = a.compute()
    assert out[0] == r
    assert np.array_equal(out[1:13], np.asarray(a.get_x(), np.float64).reshape(12))
    assert np.array_equal(out[13:19], a.velocities())


@pytest.mark.gpu
def test_cpp_tracker_adapter_matches_python_api(adapter_bin, scene, tmp_path):
    """TrackerB200 (include/kds.hpp) over four frames gives what Tracker3D gives: the same
    library, so keyframe flags, result codes and poses are identical."""
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import streams, synth
    v = np.array([2.0, 0.1, 0.0, 0.0, 0.0, 0.1])
    P = synth.pose((0.0, 0.0, 1.8))
    M = streams.motion(v, 0.1)
    frames = []
    for k in range(4):
        xyz, st = synth.scan(scene, P, vel=v, beams=16, cols=1024, seed=60 + k, t_start=0.1 * k)
        frames.append((xyz, st))
        _write_cloud(tmp_path / f"fr{k}.bin", xyz, st)
        P = streams.compose(P, M)
    subprocess.run([adapter_bin, "track", FIXTURE, str(tmp_path / "trk.bin")] +
                   [str(tmp_path / f"fr{k}.bin") for k in range(4)], check=True, capture_output=True, text=True)
    out = np.fromfile(tmp_path / "trk.bin", np.float64).reshape(4, 14)

    gen = kds.TreeGeneratorB2003D(leaf_max_points=16, tree_min_good_leaves=10, propagate_normal=0)
    odom = kds.CTICPB2003D(kernel_threshold=np.float32(0.200000003), damping=1.0, max_error=0.5,
                           min_normal_cos=np.float32(0.699999988), max_iterations=15, velocity_damping=10.0,
                           term_crit=dict(d_pert=np.float32(0.00200000009), d_score=np.float32(0.000500000024)))
    trk = kds.Tracker3D(odom_aligner=odom, motion_model=kds.ConstVelMotionModel3D(), max_kf_trans=0.5,
                        min_inlier_frac=0.3)
    for k, (xyz, st) in enumerate(frames):
        r = trk.add_frame(gen.make_tree(xyz, st), 0.1 * k)
        assert out[k, 0] == float(r["new_keyframe"]) and out[k, 1] == r["result"], k
        assert np.array_equal(out[k, 2:], r["pose_in_world"].reshape(12)), k
