"""Scan input on the device (kds_points_voxelize: toPointsVector + Voxelizer_::voxelize)
against the restatement in oracle/voxel.py: bit-identical points and stamps with and
without a voxel grid, host and device inputs alike, and a tree built from the output
equal to the oracle's tree built from the oracle's output."""
import numpy as np
import pytest

from conftest import make_scan
from oracle import orc
from oracle import voxel as OV

pytestmark = pytest.mark.gpu


def same(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint32 if a.dtype == np.float32 else np.uint64),
                                                 b.view(np.uint32 if b.dtype == np.float32 else np.uint64))


@pytest.mark.parametrize("params", [
    dict(range_min=2.0, range_max=40.0),
    dict(range_min=1.0, range_max=50.0, space_res=0.25),
    dict(range_min=1.0, range_max=35.0, space_res=0.5, time_res=0.02, use_boundary=1),
])
def test_voxelize_matches_restatement(scene, params):
    import kd_slam2_b200 as kds
    xyz, st = make_scan(scene, 4300, beams=32, elev=(-15.0, 15.0), vel=[4.0, 0, 0, 0, 0, 0.3])
    gx, gs = kds.voxelize(xyz, st, **params)
    ox, os_ = OV.voxelize(xyz, st, **params)
    assert len(gx) > 100 and same(gx, ox) and same(gs, os_)
    if params.get("space_res", 0) > 0:
        assert len(gx) < len(xyz)


def test_azimuth_stamps_and_device_inputs(scene):
    import torch

    import kd_slam2_b200 as kds
    xyz, _ = make_scan(scene, 4301, beams=16, elev=(-15.0, 15.0))
    prm = dict(range_min=1.0, range_max=60.0, space_res=0.3, time_res=0.01)
    gx, gs = kds.voxelize(xyz, None, msg_t=1.7e9, scan_duration=0.1, **prm)
    ox, os_ = OV.voxelize(xyz, None, msg_t=1.7e9, scan_duration=0.1, **prm)
    assert same(gx, ox)
    # CUDA's atan2 and the C library's may differ in the last bit; the stamps' rounding
    # at 1.7e9 s absorbs that
    assert np.allclose(gs, os_, rtol=1e-15, atol=0)
    dx, ds = kds.voxelize(torch.from_numpy(xyz).cuda(), None, msg_t=1.7e9, scan_duration=0.1, **prm)
    assert same(dx.cpu().numpy(), gx) and same(ds.cpu().numpy(), gs)


def test_voxelized_scan_builds_the_oracles_tree(scene):
    import kd_slam2_b200 as kds
    xyz, st = make_scan(scene, 4302, beams=32, elev=(-15.0, 15.0), vel=[3.0, 0, 0, 0, 0, 0.2])
    prm = dict(range_min=1.0, range_max=50.0, space_res=0.2)
    gx, gs = kds.voxelize(xyz, st, **prm)
    ox, os_ = OV.voxelize(xyz, st, **prm)
    G = kds.TreeGeneratorB2003D(leaf_max_points=16).make_tree(gx, gs)
    O = orc.OTree.build(ox, os_, orc.tree_params(leaf_max_points=16))
    eg, eo = G.export(), O.export()
    for k in ("left", "right", "start", "end", "leaves", "perm"):
        assert np.array_equal(eg[k], eo[k]), k
    assert np.array_equal(eg["mean"], eo["mean"]) and np.array_equal(eg["dir"], eo["dir"])


def test_voxelize_full_sweep():
    """A full 128 x 2048 sweep (about 200k returns) at the grid used by the benchmark."""
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import synth
    boxes = synth.scene(1003)
    xyz, st = synth.scan(boxes, synth.pose((0.0, 0.0, 1.8)), beams=128, cols=2048, elev=(-22.5, 22.5), seed=7000,
                         threads=16)
    prm = dict(range_min=1.0, range_max=100.0, space_res=0.1)
    gx, gs = kds.voxelize(xyz, st, **prm)
    ox, os_ = OV.voxelize(xyz, st, **prm)
    assert len(xyz) > 150000 and same(gx, ox) and same(gs, os_)
