"""kds_linearize_static, the linearization for callers that cannot allocate device memory
(real-time loops that reserve all their memory at start-up, code that must not wait on
cudaMalloc/cudaFree), against the aligner's own buildQuadraticForm and the oracle.

The static call runs the same kernels over the same 128-leaf tiles as
kds_aligner_build_quadratic_form, so H, b and the stats must be bit-identical to it; the
oracle's linearization in the product's summation order, at the caches the product
derives from the same poses, must be bit-identical too.  Each case makes two calls in a
row with different inputs, because every call reuses the same static scratch, and the
second call must leave the device's free memory and the default memory pool's
reservation and use unchanged.  The file name sorts last so that it also runs after the
rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import make_scan, perturbation
from oracle import orc

pytestmark = pytest.mark.gpu

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


def _same(Hs, bs, ss, Ha, ba, sa):
    assert np.array_equal(Hs, Ha), np.abs(Hs - Ha).max()
    assert np.array_equal(bs, ba), np.abs(bs - ba).max()
    for k in ("num_inliers", "num_outliers", "num_bad", "num_err_normal", "num_err_fn", "chi2", "chi2_kernelized"):
        assert ss[k] == sa[k], (k, ss[k], sa[k])
    assert ss["num_inliers"] > 0


def _memory_state():
    """Free device memory and the default pool's reserved and used bytes (current device)."""
    from cuda.bindings import runtime as rt
    err, free, _total = rt.cudaMemGetInfo()
    assert err == rt.cudaError_t.cudaSuccess
    err, dev = rt.cudaGetDevice()
    err, pool = rt.cudaDeviceGetDefaultMemPool(dev)
    assert err == rt.cudaError_t.cudaSuccess
    out = [free]
    for attr in (rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent):
        err, val = rt.cudaMemPoolGetAttribute(pool, attr)
        assert err == rt.cudaError_t.cudaSuccess
        out.append(int(val))
    return tuple(out)


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
    Of = orc.OTree.build(xf, sf, orc.tree_params(leaf_max_points=16))
    Om = orc.OTree.build(xm, sm, orc.tree_params(leaf_max_points=16))
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
        _same(Hs, bs, ss, Ha, ba, sa)
        _, _, Ho, bo, so = orc.linearize(orc.KIND_ICP, Of, Om, orc.product_caches(X, Xf), orc.align_params(**P),
                                         stats_mode=bool(stats_mode))
        _same(Hs, bs, ss, Ho, bo, so)
    # the second static call reserved and used no device memory: nothing changed between
    # the state after the first call and the state after the second (the aligner's own
    # buildQuadraticForm ran before the second call, so compare what it left behind)
    X = perturbation(rng, 0.3, 3.0)
    before = _memory_state()
    rc, _, _, _ = _static(kds.lib(), Gf, Gm, abi.KDS_ICP, params, X, Xf)
    assert rc == abi.KDS_OK
    assert _memory_state() == before


def test_ct_two_calls_match_build_quadratic_form(clouds):
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import abi
    (xf, sf), _, (xc, sc), vel = clouds
    gen = kds.TreeGeneratorB2003D(leaf_max_points=16)
    Gf, Gc = gen.make_tree(xf, sf), gen.make_tree(xc, sc)
    Of = orc.OTree.build(xf, sf, orc.tree_params(leaf_max_points=16))
    Oc = orc.OTree.build(xc, sc, orc.tree_params(leaf_max_points=16))
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
        before = _memory_state()
        rc, Hs, bs, ss = _static(kds.lib(), Gf, Gc, abi.KDS_CTICP, params, X, Xf, v=v)
        assert rc == abi.KDS_OK, (call, kds.lib().kds_last_error())
        if call == 1:  # the first call of a process may load the library's kernels
            assert _memory_state() == before
        Ha, ba, sa = _reference_form(a, X, v=v)
        _same(Hs, bs, ss, Ha, ba, sa)
        _, _, Ho, bo, so = orc.linearize(orc.KIND_CT, Of, Oc, orc.product_caches(X, Xf), orc.align_params(**P),
                                         v=np.asarray(v, np.float32))
        _same(Hs, bs, ss, Ho, bo, so)


def test_tree_top_wait_fallback_reports_own_timeout(clouds):
    """With the bounded wait for the tree-top copy cut to zero polls every block falls back
    to global memory: the call returns KDS_ERR_TIMEOUT from its own error slot, with the
    same H, b and stats; the next call with the default limit returns KDS_OK."""
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import abi
    (xf, sf), (xm, sm), _, _ = clouds
    gen = kds.TreeGeneratorB2003D(leaf_max_points=16)
    Gf, Gm = gen.make_tree(xf, sf), gen.make_tree(xm, sm)
    params = kds.aligner_params(max_error=0.5)
    X = perturbation(np.random.default_rng(21), 0.2, 2.0)
    lib = kds.lib()
    rc0, H0, b0, s0 = _static(lib, Gf, Gm, abi.KDS_ICP, params, X, kds.identity())
    assert rc0 == abi.KDS_OK
    assert lib.kds_set_tma_wait_limit(0) == abi.KDS_OK
    try:
        rc1, H1, b1, s1 = _static(lib, Gf, Gm, abi.KDS_ICP, params, X, kds.identity())
    finally:
        assert lib.kds_set_tma_wait_limit(1 << 20) == abi.KDS_OK
    assert rc1 == abi.KDS_ERR_TIMEOUT
    assert b"valid" in lib.kds_last_error()
    _same(H1, b1, s1, H0, b0, s0)
    rc2, H2, b2, s2 = _static(lib, Gf, Gm, abi.KDS_ICP, params, X, kds.identity())
    assert rc2 == abi.KDS_OK
    _same(H2, b2, s2, H0, b0, s0)


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
