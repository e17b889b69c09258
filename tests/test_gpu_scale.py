"""Parity at the named configurations' own sizes.

  rigid_16x1024       rigid ICP, 16 x 1024 scan against a second scan's tree
  ct_64x1024_1m_map   CT-ICP, skewed 64 x 1024 scan against the tree of 20 prior scans of
                      128 x 8192 rays (about 14.6M points, 1.2M surfels, 20+ levels: the
                      large-node partition at scale)

For each: the map and scan trees bit-identical to the oracle's build (node arrays, leaf
lists, point order); one linearization at the initial guess with identical float caches
-- correspondences, status masks, H and b bit-identical; the whole compute() --
pose, velocities, result code and stats bit-identical to the oracle in the product's
semantics (MODE_MIXED), and the pose within 1e-4 m / rad of the all-FP64 oracle.
"""
import numpy as np
import pytest

from conftest import assert_same_tree, pose_err
from oracle import orc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["rigid_16x1024", "ct_64x1024_1m_map"])
def test_named_configuration_parity(name):
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import scans
    wl = getattr(scans, name)()
    ct = wl["kind"] == "ct"
    tp = orc.tree_params(**wl["tree"])
    gen = kds.TreeGeneratorB2003D(**wl["tree"])
    Gm, Gs = gen.make_tree(wl["map_xyz"]), gen.make_tree(wl["xyz"], wl["st"])
    Om, Os = orc.OTree.build(wl["map_xyz"], None, tp), orc.OTree.build(wl["xyz"], wl["st"], tp)
    assert_same_tree(Om, Gm)
    assert_same_tree(Os, Gs)
    if ct:
        assert Gm.num_leaves > 1_000_000 and Gm.info.depth >= 20
    X0, v0 = wl["X0s"][0], wl["v0"]
    a = kds.CTICPB2003D(**wl["params"]) if ct else kds.ICPB2003D(**wl["params"])
    a.set_fixed(Gm)
    a.set_moving(Gs)
    P = orc.align_params(**wl["params"])
    kind = orc.KIND_CT if ct else orc.KIND_ICP
    # one linearization at the initial guess, identical float caches
    c = orc.caches_from(X0)
    v = None if v0 is None else np.asarray(v0, np.float32)
    mg, sg, Hg, bg, stg = a.linearize_debug(c, v=v) if ct else a.linearize_debug(c)
    mo, so, Ho, bo, sto = orc.linearize(kind, Om, Os, c, P, v=v)
    assert np.array_equal(mg, mo) and np.array_equal(sg, so)
    assert np.array_equal(Hg, Ho) and np.array_equal(bg, bo)
    assert stg == sto
    # the whole Gauss-Newton loop
    a.set_x(X0)
    if ct:
        a.set_velocities(v0)
    ret = a.compute()
    ro = orc.align(kind, orc.MODE_MIXED, Om, Os, P, X0, v0=v0)
    assert ret == ro["ret"]
    assert np.array_equal(a.get_x(), ro["X"]), pose_err(a.get_x(), ro["X"])
    assert np.array_equal(a.velocities(), ro["v"])
    r64 = orc.align(kind, orc.MODE_FP64, Om, Os, P, X0, v0=v0)
    assert max(pose_err(a.get_x(), r64["X"])) <= 1e-4
