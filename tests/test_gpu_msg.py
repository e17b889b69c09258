"""Tree wire format (kd_slam2_msgs/msg/KDTree3f with KDNode3f nodes): a device tree
written as a message and read back (toMessage, lib/kd_io/slam_messages.h:47-80;
TreeLoader_::fromTreeMsg, lib/kd_io/tree_loader_impl_.h:59-70) is the same tree --
node for node, with its root frame -- and aligns to bit-identical results as the fixed
and as the moving tree.  Malformed node arrays are refused with a status."""
import numpy as np
import pytest

from conftest import make_scan

pytestmark = pytest.mark.gpu

TREE = dict(leaf_max_points=16)


def test_message_round_trip_is_the_same_tree(scene):
    import kd_slam2_b200 as kds
    xyz, st = make_scan(scene, 4100, beams=32, elev=(-15.0, 15.0), vel=[5.0, 0, 0, 0, 0, 0.2])
    T = kds.TreeGeneratorB2003D(**TREE).make_tree(xyz, st)
    msg = T.to_msg()
    assert msg["nodes"].dtype.itemsize == 56 and len(msg["nodes"]) == T.num_nodes
    U = kds.Tree.from_msg(msg)
    et, eu = T.export(), U.export()
    for k in ("mean", "dir", "dts_mean", "dts_cov", "start", "end", "left", "right", "leaves"):
        assert np.array_equal(et[k], eu[k]), k
    assert eu["ts_start"] == et["ts_start"] and U.info.num_points == 0
    rt, ru = T.root(), U.root()
    for k in rt:
        assert np.array_equal(rt[k], ru[k]), k
    # the message fields themselves: column-major eigenvectors, node records in Node_ order
    assert np.array_equal(msg["root_eigenvectors"].reshape(3, 3).T, rt["root_eigenvectors"])
    assert np.array_equal(msg["nodes"]["mean"], et["mean"])
    assert np.array_equal(msg["nodes"]["idx_left"], et["left"])
    assert np.array_equal(msg["nodes"]["idx_end"].astype(np.int64), et["end"])


def test_message_tree_aligns_like_the_original(scene):
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import synth
    X_true = synth.pose((0.3, -0.2, 1.8), (0.0, 0.0, 0.05))
    m_xyz, m_st = make_scan(scene, 4200, beams=32, elev=(-15.0, 15.0))
    s_xyz, s_st = make_scan(scene, 4201, beams=16, elev=(-15.0, 15.0), pose=X_true,
                            vel=[4.0, 0, 0, 0, 0, 0.3])
    gen = kds.TreeGeneratorB2003D(**TREE)
    M, S = gen.make_tree(m_xyz, m_st), gen.make_tree(s_xyz, s_st)
    M2, S2 = kds.Tree.from_msg(M.to_msg()), kds.Tree.from_msg(S.to_msg())
    X0 = synth.pose((0.2, -0.1, 1.75), (0.0, 0.0, 0.03))
    out = []
    for fixed, moving in ((M, S), (M2, S2), (M, S2), (M2, S)):
        a = kds.CTICPB2003D(max_error=0.5, max_iterations=10, velocity_damping=10.0)
        a.set_fixed(fixed)
        a.set_moving(moving)
        a.set_x(X0)
        a.set_velocities(np.array([3.0, 0, 0, 0, 0, 0.2]))
        r = a.compute()
        out.append((r, np.asarray(a.get_x()).copy(), np.asarray(a.velocities()).copy()))
    for r, X, v in out[1:]:
        assert r == out[0][0]
        assert np.array_equal(X, out[0][1]) and np.array_equal(v, out[0][2])


def test_malformed_messages_are_refused():
    import kd_slam2_b200 as kds
    from kd_slam2_b200.abi import KDNODE3F_DTYPE, KDS_ERR_BAD_TREE, KdsError
    nodes = np.zeros(3, KDNODE3F_DTYPE)
    nodes["idx_left"] = [1, -1, -1]
    nodes["idx_right"] = [2, -1, -1]
    kds.Tree.from_msg({"nodes": nodes}).free()  # a root with two leaves is fine
    bad = nodes.copy()
    bad["idx_left"][1] = 0  # a child before its parent: not BFS
    with pytest.raises(KdsError) as e:
        kds.Tree.from_msg({"nodes": bad})
    assert e.value.code == KDS_ERR_BAD_TREE
    bad = nodes.copy()
    bad["idx_right"][0] = 7  # out of range
    with pytest.raises(KdsError) as e:
        kds.Tree.from_msg({"nodes": bad})
    assert e.value.code == KDS_ERR_BAD_TREE
