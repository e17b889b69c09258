"""Device assembly of the multi-view bundle-adjustment factors (kds_batch_assemble)
against the restated MultiViewICPFactor_ / MultiViewCTICPFactor_ block updates
(oracle/factors.py) over the same batch's per-pair H, b: identical blocks, b and
enabled flags, with some factors disabled by their inlier ratio."""
import numpy as np
import pytest

import kd_slam2_b200 as kds

pytestmark = pytest.mark.gpu

TREE = dict(leaf_max_points=16)
ICP = dict(max_error=0.5, max_iterations=10)
CT = dict(max_error=0.5, max_iterations=15, velocity_damping=10.0)


def test_assembly_equals_restated_factor_updates():
    from kd_slam2_b200 import ba, synth
    from kd_slam2_b200.streams import compose
    from oracle import factors as OF
    wl = ba.make_workload(seed=9, num_keyframes=8, min_pts=8000, max_pts=30000, beams=64, cols=1024)
    trees = ba.build_trees(wl, TREE)
    rng = np.random.default_rng(5)
    X = [compose(kf.X, synth.pose(0.05 * rng.normal(size=3), np.deg2rad(0.5) * rng.normal(size=3)))
         for kf in wl.keyframes]
    v = [kf.vel + 0.1 * rng.normal(size=6) for kf in wl.keyframes]
    jobs, factors, nv = ba.factor_jobs(wl, trees, ICP, CT, X=X, v=v)
    assert {len(f[1]) for f in factors} == {2, 4}
    B = kds.Batch()
    res = B.run(jobs)
    ratios = np.array([OF.inlier_ratio(j.stats) for j in res])
    thr = float(np.median(ratios))  # about half the factors disabled
    rc, H, b, en = B.assemble(factors, nv, disable_inlier_ratio=thr)
    Hr, br, enr = OF.assemble(res, factors, nv, thr)
    assert np.array_equal(en, enr) and 0 < en.sum() < len(factors)
    assert [tuple(x) for x in rc] == sorted(Hr)
    for k, (r, c) in enumerate(rc):
        assert r <= c
        assert np.array_equal(H[k], Hr[(r, c)]), (r, c)
    assert np.array_equal(b, br)


def test_assembly_rejects_bad_factors():
    from kd_slam2_b200 import ba
    from kd_slam2_b200.abi import KDS_ERR_INVALID_ARG, KdsError
    wl = ba.make_workload(seed=3, num_keyframes=4, min_pts=8000, max_pts=20000, beams=64, cols=1024)
    trees = ba.build_trees(wl, TREE)
    jobs = ba.jobs(wl, trees, ICP, CT)  # plain CT jobs: no dual blocks
    B = kds.Batch()
    B.run(jobs)
    ct = next(k for k, p in enumerate(wl.pairs) if p.kind == 1)
    for bad in ([(ct, [0, 1, 2, 3])], [(len(jobs), [0, 1])], [(0, [0, 99])]):
        with pytest.raises(KdsError) as e:
            B.assemble(bad, 8)
        assert e.value.code == KDS_ERR_INVALID_ARG


def test_assembly_full_ba_step():
    """The full bundle-adjustment configuration (200 keyframes, 894 pairs, each a rigid and a
    CT factor = 1,788 factors over 400 variables): device assembly equals the restatement."""
    from kd_slam2_b200 import ba
    from oracle import factors as OF
    wl = ba.make_workload()
    trees = ba.build_trees(wl, TREE, inputs=ba.device_inputs(wl))
    jobs, factors, nv = ba.factor_jobs(wl, trees, ICP, CT)
    B = kds.Batch()
    res = B.run(jobs)
    rc, H, b, en = B.assemble(factors, nv, disable_inlier_ratio=0.3)
    Hr, br, enr = OF.assemble(res, factors, nv, 0.3)
    assert len(factors) == 1788 and np.array_equal(en, enr)
    assert [tuple(x) for x in rc] == sorted(Hr)
    for k, (r, c) in enumerate(rc):
        assert np.array_equal(H[k], Hr[(r, c)]), (r, c)
    assert np.array_equal(b, br)
