"""kds_linearize_static, the linearization that allocates nothing, against the
aligner's own buildQuadraticForm (kds_aligner_build_quadratic_form + get_hb/get_stats).

Both run the same kernels over the same 128-leaf tiles, so H, b and the stats counters
are expected to agree; the test allows RTOL_HB relative to max|H|, the tolerance the
other linearization tests use.  Each case makes two calls in a row with different
inputs, because every call reuses the same static scratch.  The file name sorts last
so that it also runs after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import make_scan, perturbation

pytestmark = pytest.mark.gpu

RTOL_HB = 2e-5
STATIC_MAX_LEAVES = 65536


def _static(lib, fixed, moving, kind, params, X, Xf, v=None, fv=None, stats_mode=0):
    from kd_slam2_b200 import abi
    D = 6 if kind == abi.KDS_ICP else 12
    H = np.zeros(D * D, np.float64)
    b = np.zeros(D, np.float64)
    st = abi.Stats()
    X = np.ascontiguousarray(np.asarray(X, np.float64).reshape(3, 4)).ravel()
    Xf = np.ascontiguousarray(np.asarray(Xf, np.float64).reshape(3, 4)).ravel()
    vv = None if v is None else np.ascontiguousarray(v, np.float64)
    fvv = None if fv is None else np.ascontiguousarray(fv, np.float64)
    rc = lib.kds_linearize_static(fixed.handle, moving.handle, kind, C.byref(params), X.ctypes.data,
                                  Xf.ctypes.data, None if vv is None else vv.ctypes.data,
                                  None if fvv is None else fvv.ctypes.data, stats_mode, None, H.ctypes.data,
                                  b.ctypes.data, C.byref(st))
    return rc, H.reshape(D, D), b, st.as_dict()


def _reference_form(aligner, X, v=None, stats_mode=False):
    aligner.set_x(X)
    if v is not None:
        aligner.set_velocities(v)
    aligner.build_quadratic_form(stats_mode=stats_mode)
    return aligner.H, aligner.b, aligner.stats


def _close(Hs, bs, ss, Ha, ba, sa):
    s = max(1e-12, np.abs(Ha).max())
    assert np.abs(Hs - Ha).max() <= RTOL_HB * s, np.abs(Hs - Ha).max() / s
    sb = max(1e-12, np.abs(ba).max(), s * 1e-3)
    assert np.abs(bs - ba).max() <= RTOL_HB * sb * 10, np.abs(bs - ba).max() / sb
    for k in ("num_inliers", "num_outliers", "num_bad", "num_err_normal", "num_err_fn"):
        assert ss[k] == sa[k], (k, ss[k], sa[k])
    assert ss["num_inliers"] > 0


@pytest.fixture(scope="module")
def clouds(scene):
    from kd_slam2_b200 import synth
    xf, sf = make_scan(scene, 3000)
    xm, sm = make_scan(scene, 3001)
    vel = np.array([8.0, 0.5, 0, 0, 0, np.deg2rad(20.0)])
    xc, sc = make_scan(scene, 3002, beams=32, pose=synth.pose((0.0, 0.0, 1.8)), vel=vel)
    return (xf, sf), (xm, sm), (xc, sc), vel


def test_icp_two_calls_match_build_quadratic_form(clouds):
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import abi
    (xf, sf), (xm, sm), _, _ = clouds
    gen = kds.TreeGeneratorB2003D(leaf_max_points=16)
    Gf, Gm = gen.make_tree(xf, sf), gen.make_tree(xm, sm)
    assert 0 < Gm.num_leaves <= STATIC_MAX_LEAVES
    P = dict(max_error=0.5, kernel_threshold=0.01)
    a = kds.ICPB2003D(**P)
    a.set_fixed(Gf)
    a.set_moving(Gm)
    params = kds.aligner_params(**P)
    rng = np.random.default_rng(7)
    Xf = kds.identity()
    for call, stats_mode in enumerate((0, 1)):
        X = perturbation(rng, 0.3, 3.0)
        rc, Hs, bs, ss = _static(kds.lib(), Gf, Gm, abi.KDS_ICP, params, X, Xf, stats_mode=stats_mode)
        assert rc == abi.KDS_OK, (call, kds.lib().kds_last_error())
        Ha, ba, sa = _reference_form(a, X, stats_mode=bool(stats_mode))
        _close(Hs, bs, ss, Ha, ba, sa)


def test_ct_two_calls_match_build_quadratic_form(clouds):
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import abi
    (xf, sf), _, (xc, sc), vel = clouds
    gen = kds.TreeGeneratorB2003D(leaf_max_points=16)
    Gf, Gc = gen.make_tree(xf, sf), gen.make_tree(xc, sc)
    assert 0 < Gc.num_leaves <= STATIC_MAX_LEAVES
    P = dict(max_error=0.5, velocity_damping=10.0)
    a = kds.CTICPB2003D(**P)
    a.set_fixed(Gf)
    a.set_moving(Gc)
    params = kds.aligner_params(**P)
    rng = np.random.default_rng(11)
    Xf = kds.identity()
    for call in range(2):
        X = perturbation(rng, 0.2, 2.0)
        v = vel + rng.normal(scale=0.3, size=6) * np.array([1, 1, 1, 0.05, 0.05, 0.05])
        rc, Hs, bs, ss = _static(kds.lib(), Gf, Gc, abi.KDS_CTICP, params, X, Xf, v=v)
        assert rc == abi.KDS_OK, (call, kds.lib().kds_last_error())
        Ha, ba, sa = _reference_form(a, X, v=v)
        _close(Hs, bs, ss, Ha, ba, sa)


def test_rejects_more_leaves_than_the_static_maximum():
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import abi
    # a noisy plane: flat leaves of at most 16 points, well over 65,536 of them
    rng = np.random.default_rng(5)
    n = 1_600_000
    xyz = np.empty((n, 3), np.float32)
    xyz[:, 0] = rng.uniform(-200, 200, n)
    xyz[:, 1] = rng.uniform(-200, 200, n)
    xyz[:, 2] = rng.normal(scale=0.01, size=n)
    gen = kds.TreeGeneratorB2003D(leaf_max_points=16)
    G = gen.make_tree(xyz)
    assert G is not None and G.num_leaves > STATIC_MAX_LEAVES
    params = kds.aligner_params()
    rc, _, _, _ = _static(kds.lib(), G, G, abi.KDS_ICP, params, kds.identity(), kds.identity())
    assert rc == abi.KDS_ERR_CAPACITY
    assert b"65536" in kds.lib().kds_last_error()
