"""GPU tree build against the oracle: bit-exact node arrays, leaf lists and point order."""
import numpy as np
import pytest

from conftest import assert_same_tree, make_scan
from oracle import orc

pytestmark = pytest.mark.gpu


def build_both(xyz, st, **params):
    import kd_slam2_b200 as kds
    O = orc.OTree.build(xyz, st, orc.tree_params(**params))
    G = kds.TreeGeneratorB2003D(**params).make_tree(xyz, st)
    return O, G


@pytest.mark.parametrize("seed,beams,params", [
    (2000, 16, dict(leaf_max_points=16)),
    (2001, 16, dict(leaf_max_points=16, propagate_normal=1)),
    (2002, 32, dict()),
    (2003, 64, dict(leaf_max_points=16)),  # 65k points: large-node path
    (2004, 16, dict(leaf_max_points=100, leaf_min_points=5, leaf_min_normal_incidence=0.2, propagate_normal=1,
                    tree_min_good_leaves=50)),
])
def test_tree_build_bit_exact(scene, seed, beams, params):
    xyz, st = make_scan(scene, seed, beams=beams, elev=(-15.0, 15.0) if beams <= 32 else (-22.5, 22.5))
    O, G = build_both(xyz, st, **params)
    assert O.accepted and G is not None
    assert_same_tree(O, G)


def test_forest_build_equals_single_builds(scene):
    """One batched pass over uneven clouds gives each tree bit-identical to its own build."""
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import synth
    clouds = []
    for i, beams in enumerate([16, 32, 16, 64]):
        xyz, st = make_scan(scene, 2300 + i, beams=beams, elev=(-15.0, 15.0),
                            vel=[5.0 * i, 0, 0, 0, 0, 0.1 * i])
        clouds.append((xyz, st + 10.0 * i))
    clouds.insert(2, (np.zeros((3, 3), np.float32), None))  # rejected: fewer than leaf_min_points
    gen = kds.TreeGeneratorB2003D(leaf_max_points=16, propagate_normal=1)
    trees = gen.make_trees(clouds)
    assert trees[2] is None
    for (xyz, st), T in zip(clouds, trees):
        if len(xyz) < 5:
            continue
        O = orc.OTree.build(xyz, st, orc.tree_params(leaf_max_points=16, propagate_normal=1))
        assert_same_tree(O, T)
    # the packed form (kds_tree_build_batch: one array, offsets) gives the same trees
    import ctypes as C
    from kd_slam2_b200 import abi as L
    xyz = np.ascontiguousarray(np.concatenate([c[0] for c in clouds]))
    st = np.ascontiguousarray(np.concatenate([np.zeros(len(c[0])) if c[1] is None else c[1] for c in clouds]))
    off = np.zeros(len(clouds) + 1, np.int64)
    off[1:] = np.cumsum([len(c[0]) for c in clouds])
    hs = (C.c_void_p * len(clouds))()
    status = (C.c_int32 * len(clouds))()
    rc = kds.lib().kds_tree_build_batch(xyz.ctypes.data, st.ctypes.data, off.ctypes.data, len(clouds),
                                        L.KDS_MEM_HOST, C.byref(gen.params), None, hs, status)
    assert rc == L.KDS_OK and status[2] == L.KDS_ERR_TREE_REJECTED
    for i, T in enumerate(trees):
        if T is None:
            continue
        P = kds.Tree(hs[i])
        a, b = T.export(), P.export()
        for k in ("mean", "dir", "dts_mean", "left", "right", "leaves", "perm"):
            assert np.array_equal(a[k], b[k]), (i, k)


def test_tree_build_skewed_scan_with_stamps(scene):
    from kd_slam2_b200 import synth
    xyz, st = make_scan(scene, 2010, beams=32, vel=[10.0, 0, 0, 0, 0, np.deg2rad(30.0)])
    st = st + 1234.5  # absolute stamps: dts relative to the first point
    O, G = build_both(xyz, st, leaf_max_points=16)
    assert_same_tree(O, G)


def test_tree_without_stamps(scene):
    xyz, _ = make_scan(scene, 2011)
    O, G = build_both(xyz, None, leaf_max_points=16)
    assert_same_tree(O, G)


def test_rejected_trees_match_makeTree_nullptr(scene):
    import kd_slam2_b200 as kds
    # fewer points than leaf_min_points
    xyz = np.zeros((3, 3), np.float32)
    assert kds.TreeGeneratorB2003D().make_tree(xyz) is None
    # a tiny patch: too few good leaves for tree_min_good_leaves
    rng = np.random.default_rng(0)
    xyz = (rng.normal(size=(200, 3)) * [1.0, 1.0, 0.01] + [10.0, 0, 0]).astype(np.float32)
    O = orc.OTree.build(xyz, None, orc.tree_params(tree_min_good_leaves=50))
    G = kds.TreeGeneratorB2003D(tree_min_good_leaves=50).make_tree(xyz)
    assert not O.accepted and G is None


def test_degenerate_inputs(scene):
    """duplicated points and collinear runs: deterministic, same as the oracle"""
    xyz, st = make_scan(scene, 2012)
    dup = np.concatenate([xyz, xyz[:3000], np.repeat(xyz[:5], 40, axis=0)]).astype(np.float32)
    std = np.concatenate([st, st[:3000], np.repeat(st[:5], 40)])
    line = np.stack([np.linspace(5, 15, 500), np.full(500, 3.0), np.full(500, 0.5)], 1).astype(np.float32)
    allp = np.concatenate([dup, line]).astype(np.float32)
    alls = np.concatenate([std, np.zeros(500)])
    O, G = build_both(allp, alls, leaf_max_points=16)
    assert_same_tree(O, G)


def test_out_of_range_input_is_rejected_with_status():
    import kd_slam2_b200 as kds
    xyz = np.zeros((100, 3), np.float32)
    xyz[5] = [1e6, 0, 0]
    with pytest.raises(kds.KdsError) as ei:
        kds.TreeGeneratorB2003D().make_tree(xyz)
    assert ei.value.code == kds.abi.KDS_ERR_RANGE


def test_import_export_roundtrip(scene):
    import kd_slam2_b200 as kds
    xyz, st = make_scan(scene, 2013)
    O = orc.OTree.build(xyz, st, orc.tree_params(leaf_max_points=16))
    e = O.export()
    T = kds.Tree.import_nodes(e["mean"], e["dir"], e["left"], e["right"], e["dts_mean"], e["dts_cov"], e["start"],
                              e["end"], ts_start=e["ts_start"])
    g = T.export()
    for k in ("mean", "dir", "left", "right", "dts_mean", "dts_cov", "start", "end", "leaves"):
        assert np.array_equal(e[k], g[k]), k
    # malformed: child index pointing backwards
    bad = e["left"].copy()
    bad[5] = 1
    with pytest.raises(kds.KdsError) as ei:
        kds.Tree.import_nodes(e["mean"], e["dir"], bad, e["right"])
    assert ei.value.code == kds.abi.KDS_ERR_BAD_TREE


def test_morph_and_isometry_match_oracle(scene):
    import kd_slam2_b200 as kds
    xyz, st = make_scan(scene, 2014, vel=[5.0, 0.5, 0, 0.01, 0, 0.4])
    G = kds.TreeGeneratorB2003D(leaf_max_points=16).make_tree(xyz, st)
    e0 = G.export()
    v = np.array([5.0, 0.5, 0.1, 0.01, -0.02, 0.4], np.float32)
    G.apply_velocities_in_place(v)
    e1 = G.export()
    for i in range(0, len(e0["mean"]), 7):
        mo, no = orc.warp_leaf(v, np.float32(e0["dts_mean"][i]), e0["mean"][i], e0["dir"][i])
        assert np.array_equal(mo.view(np.uint32), e1["mean"][i].view(np.uint32))
        assert np.array_equal(no.view(np.uint32), e1["dir"][i].view(np.uint32))
    # leaves only skipped when asked
    G2 = kds.TreeGeneratorB2003D(leaf_max_points=16).make_tree(xyz, st)
    G2.apply_velocities_in_place(v, skip_leaves=True)
    e2 = G2.export()
    assert np.array_equal(e2["mean"][e2["leaves"]], e0["mean"][e0["leaves"]])
    # rigid transform: applyIsometry_ row loop
    from kd_slam2_b200 import synth
    X = synth.pose((1.0, -2.0, 0.3), (0.1, 0.2, -0.3)).astype(np.float32)
    G3 = kds.TreeGeneratorB2003D(leaf_max_points=16).make_tree(xyz, st)
    G3.apply_isometry_in_place(X)
    e3 = G3.export()
    m = e0["mean"][10]
    ref = np.float32(X[:, 3])
    for c in range(3):
        ref = (ref + (X[:, c] * m[c]).astype(np.float32)).astype(np.float32)
    assert np.array_equal(ref.view(np.uint32), e3["mean"][10].view(np.uint32))
    L = G3.extract_compressed_leaves()
    assert np.array_equal(L[:, :3], e3["mean"][e3["leaves"]])
    # into a device buffer: the same values, with and without a morph
    import torch
    D = torch.empty((G3.num_leaves, 6), dtype=torch.float32, device="cuda")
    G3.extract_compressed_leaves_device(D)
    torch.cuda.synchronize()
    assert np.array_equal(D.cpu().numpy(), L)
    G3.extract_compressed_leaves_device(D, v=v)
    torch.cuda.synchronize()
    assert np.array_equal(D.cpu().numpy(), G3.extract_compressed_leaves(v))


def test_tree_build_bit_exact_on_stream_scans():
    """Scans of the served-registration trace (moving sensors, skewed stamps)."""
    from kd_slam2_b200 import streams
    tr = streams.make_trace(7, num_streams=4, scans_per_stream=2, saturate=True, beam_mix=(16, 32), map_scans=2)
    for r in tr.requests:
        O, G = build_both(r.xyz, r.stamps, leaf_max_points=16)
        assert O.accepted and G is not None
        assert_same_tree(O, G)
    for s in tr.streams:  # the initial maps, world frame, no stamps
        O, G = build_both(s.map_xyz, None, leaf_max_points=16)
        assert_same_tree(O, G)


def test_tree_build_bit_exact_near_the_origin():
    """Many tiny products of mixed sign: the fixed-point floor of small negative values
    (where 1 - |v| does not fit a double) must agree between the GPU and the oracle."""
    rng = np.random.default_rng(21)
    n = 20000
    xyz = np.empty((n, 3), np.float32)
    xyz[:, 0] = rng.uniform(-0.05, 0.05, n)
    xyz[:, 1] = rng.uniform(-0.05, 0.05, n)
    xyz[:, 2] = -1.0 + rng.normal(scale=1e-4, size=n)  # a plane 1 m below the sensor
    st = rng.uniform(0.0, 0.1, n)
    O, G = build_both(xyz, st, leaf_max_points=16, leaf_density=0.0)
    assert O.accepted and G is not None
    assert_same_tree(O, G)
