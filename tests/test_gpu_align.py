"""GPU ICP / CT-ICP against the oracle.

Per linearization at identical float caches: fixed-leaf indices, status masks, H and b
are bit-exact (the oracle's MODE_MIXED sums in the product's tile / warp-Kahan order).
Whole compute(): pose, velocities, result code and stats are bit-identical to the
oracle in the product's semantics (MODE_MIXED: float per-leaf terms, FP64 sums,
Cholesky and pose update), and the pose is within the stated POSE_TOL_FP64 of the
all-FP64 oracle.  With a pose prior the prior's FP64 terms are summed in another order
than the oracle's, so that case is held to POSE_TOL.
"""
import numpy as np
import pytest

from conftest import make_scan, perturbation, pose_err
from oracle import orc

pytestmark = pytest.mark.gpu

POSE_TOL = 1e-5         # m and rad, against MODE_MIXED where a pose prior is summed in
POSE_TOL_FP64 = 1e-4    # m and rad, against the all-FP64 oracle


@pytest.fixture(scope="module")
def trees(scene):
    import kd_slam2_b200 as kds
    p = dict(leaf_max_points=16)
    xf, sf = make_scan(scene, 2000)
    xm, sm = make_scan(scene, 2001)
    gen = kds.TreeGeneratorB2003D(**p)
    Gf, Gm = gen.make_tree(xf, sf), gen.make_tree(xm, sm)
    Of = orc.OTree.build(xf, sf, orc.tree_params(**p))
    Om = orc.OTree.build(xm, sm, orc.tree_params(**p))
    return Gf, Gm, Of, Om


@pytest.fixture(scope="module")
def ct_trees(scene):
    """skewed moving scan (10 m/s, 30 deg/s) against a static scan"""
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import synth
    p = dict(leaf_max_points=16)
    xf, sf = make_scan(scene, 2100, beams=32)
    vel = np.array([10.0, 0, 0, 0, 0, np.deg2rad(30.0)])
    xm, sm = make_scan(scene, 2101, beams=32, pose=synth.pose((0.0, 0.0, 1.8)), vel=vel)
    gen = kds.TreeGeneratorB2003D(**p)
    Gf, Gm = gen.make_tree(xf, sf), gen.make_tree(xm, sm)
    Of = orc.OTree.build(xf, sf, orc.tree_params(**p))
    Om = orc.OTree.build(xm, sm, orc.tree_params(**p))
    return Gf, Gm, Of, Om, vel


def hb_equal(Hg, Ho, bg, bo):
    assert np.array_equal(Hg, Ho), np.abs(Hg - Ho).max() / max(1e-300, np.abs(Ho).max())
    assert np.array_equal(bg, bo), np.abs(bg - bo).max() / max(1e-300, np.abs(bo).max())


def same_run(a, ro):
    """GPU aligner state after compute() against an oracle MODE_MIXED result: identical."""
    assert np.array_equal(a.get_x(), ro["X"]), pose_err(a.get_x(), ro["X"])
    assert np.array_equal(a.velocities(), ro["v"]), np.abs(a.velocities() - ro["v"]).max()
    st = a.stats
    for k in ("num_inliers", "num_outliers", "num_bad", "num_err_normal", "num_err_fn", "chi2", "chi2_kernelized"):
        assert st[k] == ro["stats"][k], (k, st[k], ro["stats"][k])


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("stats_mode", [False, True])
def test_icp_linearization_bit_exact_correspondences(trees, seed, stats_mode):
    import kd_slam2_b200 as kds
    Gf, Gm, Of, Om = trees
    rng = np.random.default_rng(seed)
    X = perturbation(rng, 0.3, 3.0)
    c = orc.caches_from(X)
    P = dict(max_error=0.5, kernel_threshold=0.01)
    a = kds.ICPB2003D(**P)
    a.set_fixed(Gf)
    a.set_moving(Gm)
    mg, sg, Hg, bg, stg = a.linearize_debug(c, stats_mode=stats_mode)
    mo, so, Ho, bo, sto = orc.linearize(orc.KIND_ICP, Of, Om, c, orc.align_params(**P), stats_mode=stats_mode)
    assert np.array_equal(mg, mo)
    assert np.array_equal(sg, so)
    for k in ("num_inliers", "num_outliers", "num_bad", "num_err_normal", "num_err_fn"):
        assert stg[k] == sto[k], k
    assert stg["num_outliers"] > 0 and stg["num_bad"] > 0  # every gate is exercised
    hb_equal(Hg, Ho, bg, bo)


@pytest.mark.parametrize("seed", [0, 1])
def test_ct_linearization_bit_exact_correspondences(ct_trees, seed):
    import kd_slam2_b200 as kds
    Gf, Gm, Of, Om, vel = ct_trees
    rng = np.random.default_rng(10 + seed)
    X = perturbation(rng, 0.2, 2.0)
    v = (vel + rng.normal(size=6) * [0.5, 0.5, 0.1, 0.01, 0.01, 0.05]).astype(np.float32)
    c = orc.caches_from(X)
    P = dict(max_error=0.5)
    a = kds.CTICPB2003D(**P)
    a.set_fixed(Gf)
    a.set_moving(Gm)
    mg, sg, Hg, bg, stg = a.linearize_debug(c, v=v)
    mo, so, Ho, bo, sto = orc.linearize(orc.KIND_CT, Of, Om, c, orc.align_params(**P), v=v)
    assert np.array_equal(mg, mo)
    assert np.array_equal(sg, so)
    hb_equal(Hg, Ho, bg, bo)


def test_ct_dual_linearization(ct_trees):
    import kd_slam2_b200 as kds
    Gf, Gm, Of, Om, vel = ct_trees
    c = orc.caches_from(perturbation(np.random.default_rng(3), 0.1, 1.0))
    v = vel.astype(np.float32)
    fv = np.array([0.5, 0.1, 0, 0, 0, 0.05], np.float32)
    a = kds.CTICPB2003D(max_error=0.5)
    a.set_fixed(Gf)
    a.set_moving(Gm)
    mg, sg, Hg, bg, _ = a.linearize_debug(c, v=v, fixed_v=fv, kind=2)
    d = a.dual()
    mo, so, Ho, bo, _ = orc.linearize(orc.KIND_CT_DUAL, Of, Om, c, orc.align_params(max_error=0.5), v=v, fixed_v=fv)
    assert np.array_equal(mg, mo) and np.array_equal(sg, so)
    hb_equal(Hg, Ho[:12, :12], bg, bo[:12])
    assert np.array_equal(d["H_dual_vel_B"], Ho[12:, 12:])
    assert np.array_equal(d["H_dual_cross_pose_vel_B"], Ho[:6, 12:])
    assert np.array_equal(d["H_dual_cross_vel_AB"], Ho[6:12, 12:])
    assert np.array_equal(d["b_dual_vel_B"], bo[12:])


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_icp_compute_matches_oracle(trees, seed):
    import kd_slam2_b200 as kds
    Gf, Gm, Of, Om = trees
    rng = np.random.default_rng(100 + seed)
    X0 = perturbation(rng, 0.2, 2.0)
    P = dict(max_error=0.5, max_iterations=10)
    a = kds.ICPB2003D(**P)
    a.set_fixed(Gf)
    a.set_moving(Gm)
    a.set_x(X0)
    ret = a.compute()
    ro = orc.align(orc.KIND_ICP, orc.MODE_MIXED, Of, Om, orc.align_params(**P), X0)
    r64 = orc.align(orc.KIND_ICP, orc.MODE_FP64, Of, Om, orc.align_params(**P), X0)
    assert ret == ro["ret"] == 10
    same_run(a, ro)
    dt, dr = pose_err(a.get_x(), r64["X"])
    assert dt <= POSE_TOL_FP64 and dr <= POSE_TOL_FP64, (dt, dr)
    assert len(a.stats_log) == 10


def test_ct_compute_matches_oracle(ct_trees):
    import kd_slam2_b200 as kds
    Gf, Gm, Of, Om, vel = ct_trees
    X0 = perturbation(np.random.default_rng(7), 0.1, 1.0)
    P = dict(max_error=0.5, max_iterations=15, velocity_damping=10.0)
    a = kds.CTICPB2003D(**P)
    a.set_fixed(Gf)
    a.set_moving(Gm)
    a.set_x(X0)
    a.set_velocities(np.zeros(6))
    ret = a.compute()
    ro = orc.align(orc.KIND_CT, orc.MODE_MIXED, Of, Om, orc.align_params(**P), X0, v0=np.zeros(6))
    assert ret == ro["ret"]
    same_run(a, ro)
    # CTICP_::poseHessian: the Schur complement over the velocity block of the last
    # iteration's H (bit-identical to the oracle's) against the oracle's restatement
    assert np.array_equal(a.H, ro["H"])
    Hp, Ho = a.get_pose_hessian(), orc.pose_hessian(ro["H"])
    assert np.abs(Hp - Ho).max() <= 1e-9 * np.abs(Ho).max(), np.abs(Hp - Ho).max() / np.abs(Ho).max()
    assert np.allclose(Hp, Hp.T, rtol=1e-9, atol=1e-6)


def test_term_crit_prior_and_result_codes(trees):
    import kd_slam2_b200 as kds
    Gf, Gm, Of, Om = trees
    X0 = perturbation(np.random.default_rng(5), 0.1, 1.0)
    P = dict(max_error=0.5, max_iterations=20)
    a = kds.ICPB2003D(term_crit={"d_pert": 1e-3, "d_score": 1e-3}, **P)
    a.set_fixed(Gf)
    a.set_moving(Gm)
    a.set_x(X0)
    ret = a.compute()
    ro = orc.align(orc.KIND_ICP, orc.MODE_MIXED, Of, Om, orc.align_params(term_crit=1, **P), X0)
    assert 0 < ret < 20 and ret == ro["ret"]
    same_run(a, ro)
    # pose prior pulls the estimate towards Z
    from kd_slam2_b200 import synth
    Z = synth.pose((0.05, 0.0, 0.0))
    info = np.diag([1e4] * 6)
    a2 = kds.ICPB2003D(**P)
    a2.set_fixed(Gf)
    a2.set_moving(Gm)
    a2.set_x(X0)
    a2.set_pose_prior(kds.identity(), Z, info)
    a2.compute()
    ro2 = orc.align(orc.KIND_ICP, orc.MODE_MIXED, Of, Om, orc.align_params(**P), X0, prior=(np.eye(3, 4), Z, info))
    dt, dr = pose_err(a2.get_x(), ro2["X"])
    assert dt <= POSE_TOL and dr <= POSE_TOL
    # too few measurements: round 0 fails -> returns -0
    a3 = kds.ICPB2003D(min_good_measurements=10 ** 6, **P)
    a3.set_fixed(Gf)
    a3.set_moving(Gm)
    a3.set_x(X0)
    assert a3.compute() == 0
    assert np.allclose(a3.get_x(), X0)
    # stats_mode: one round, no update, returns max_iterations
    a.set_x(X0)
    assert a.compute(stats_mode=True) == 20
    assert np.allclose(a.get_x(), X0)


def test_fixed_forest_sums_entries(trees):
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import synth
    Gf, Gm, Of, Om = trees
    X0 = perturbation(np.random.default_rng(9), 0.1, 1.0)
    Xb = synth.pose((0.5, 0.0, 0.0))
    P = dict(max_error=0.5, max_iterations=5)
    a = kds.ICPB2003D(**P)
    a.set_moving(Gm)
    a.add_fixed_entry(Gf, np.eye(3, 4))
    a.add_fixed_entry(Gf, Xb)
    a.set_x(X0)
    a.compute()
    ro = orc.align(orc.KIND_ICP, orc.MODE_MIXED, [(Of, np.eye(3, 4)), (Of, Xb)], Om, orc.align_params(**P), X0)
    same_run(a, ro)


def test_batch_equals_single_alignments(trees, ct_trees):
    """Each job's result is bit-identical alone and inside a mixed batch."""
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import abi
    Gf, Gm, _, _ = trees
    Cf, Cm, _, _, vel = ct_trees
    rng = np.random.default_rng(11)
    P = kds.aligner_params(max_error=0.5, max_iterations=8)
    jobs, singles = [], []
    for i in range(6):
        X0 = perturbation(rng, 0.15, 1.5)
        if i % 2 == 0:
            jobs.append(kds.make_job(abi.KDS_ICP, Gf, Gm, P, X=X0))
        else:
            jobs.append(kds.make_job(abi.KDS_CTICP, Cf, Cm, P, X=X0, v=np.zeros(6)))
    for j in jobs:
        singles.append(kds.Batch().run([j], use_graph=False)[0])
    out = kds.Batch().run(jobs, use_graph=True)
    for s, m in zip(singles, out):
        assert s.result == m.result
        assert list(s.X) == list(m.X)
        assert list(s.v) == list(m.v)
        assert s.stats.num_inliers == m.stats.num_inliers


def test_tree_top_wait_fallback(trees):
    """With the bounded wait for the tree-top TMA copy cut to zero polls, every block of
    compute() reads the fixed tree from global memory: the call reports KDS_ERR_TIMEOUT
    from the runner's own error slot, the results are identical to a normal run, and the
    next compute() with the default limit reports nothing."""
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import abi
    Gf, Gm, _, _ = trees
    X0 = perturbation(np.random.default_rng(31), 0.2, 2.0)

    def run():
        a = kds.ICPB2003D(max_error=0.5, max_iterations=6)
        a.set_fixed(Gf)
        a.set_moving(Gm)
        a.set_x(X0)
        return a

    ref = run()
    ref.compute()
    lib = kds.lib()
    assert lib.kds_set_tma_wait_limit(0) == abi.KDS_OK
    try:
        a = run()
        with pytest.raises(kds.KdsError) as ei:
            a.compute()
    finally:
        assert lib.kds_set_tma_wait_limit(1 << 20) == abi.KDS_OK
    assert ei.value.code == abi.KDS_ERR_TIMEOUT and "valid" in str(ei.value)
    assert np.array_equal(a.get_x(), ref.get_x())
    b = run()
    b.compute()
    assert np.array_equal(b.get_x(), ref.get_x())
