import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the product kernels")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


# ---------------------------------------------------------------- shared inputs
@pytest.fixture(scope="session")
def scene():
    from kd_slam2_b200 import synth
    return synth.scene(1001)


def make_scan(boxes, seed, beams=16, cols=1024, elev=(-15.0, 15.0), pose=None, vel=None, noise=0.02):
    from kd_slam2_b200 import synth
    P = synth.pose((0.0, 0.0, 1.8)) if pose is None else pose
    return synth.scan(boxes, P, vel=vel, beams=beams, cols=cols, elev=elev, seed=seed, noise=noise)


def perturbation(rng, t_max=0.2, r_deg=2.0):
    from kd_slam2_b200 import synth
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    a = rng.normal(size=3)
    a /= np.linalg.norm(a)
    return synth.pose(t_max * d, np.deg2rad(r_deg) * a)


def pose_err(A, B):
    """translation (m) and rotation (rad) difference of two 3x4 poses"""
    A = np.asarray(A, np.float64).reshape(3, 4)
    B = np.asarray(B, np.float64).reshape(3, 4)
    dR = A[:, :3].T @ B[:, :3]
    # atan2 of the skew part and the trace: arccos of the trace alone bottoms out near 3e-8 rad
    w = 0.5 * np.array([dR[2, 1] - dR[1, 2], dR[0, 2] - dR[2, 0], dR[1, 0] - dR[0, 1]])
    return float(np.linalg.norm(A[:, 3] - B[:, 3])), float(np.arctan2(np.linalg.norm(w), (np.trace(dR) - 1) / 2))


def assert_same_tree(O, G):
    """Oracle tree O and GPU tree G: node arrays, leaf list, point order and root frame
    bit-identical."""
    eo, eg = O.export(), G.export()
    assert len(eo["mean"]) == len(eg["mean"])
    for k in ("left", "right", "level", "start", "end", "leaves", "perm"):
        assert np.array_equal(eo[k], eg[k]), k
    for k in ("mean", "dir"):
        assert np.array_equal(eo[k].view(np.uint32), eg[k].view(np.uint32)), k
    for k in ("dts_mean", "dts_cov"):
        assert np.array_equal(eo[k].view(np.uint64), eg[k].view(np.uint64)), k
    assert eo["ts_start"] == eg["ts_start"]
    assert G.info.num_unpruned == eo["num_unpruned"]
    ro, rg = O.root(), G.root()  # Tree_::root_* as TreeCPU_'s constructor sets them
    for k in ("root_mean", "root_eigenvalues", "root_eigenvectors"):
        assert np.array_equal(ro[k].view(np.uint32), rg[k].view(np.uint32)), k
