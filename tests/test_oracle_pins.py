"""Pins the CPU oracle against the reference's own known-answer tests.

The reference has no golden vectors; its only asserting tests on this path are
apps/tests/jacobians/motion_jacobian_3d_test.cpp (errorAndJacobianVelocityA/B vs
central differences, 20 cases, srand(42), h = 1e-3, TOL = 5e-3) and
apps/tests/jacobians/pose_error_jacobian_3d_test.cpp (dPoseToPoseError vs numeric,
20 cases, srand(42), h = 1e-4, TOL = 1e-2).  The same checks are run here against
the oracle's float functions, drawing the random inputs from glibc rand() after
srand(42) in the order GCC evaluates the reference's constructor arguments
(right to left).  Also checked: the canonical sine/cosine and the Jacobi eigensolver.
"""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import orc

libc = C.CDLL("libc.so.6")
libc.rand.restype = C.c_int
RAND_MAX = np.float32(2147483647)


def rnd(rng_range=1.0):
    r = np.float32(libc.rand())
    return np.float32(rng_range) * ((np.float32(2) * r) / RAND_MAX - np.float32(1))


def vec3(f):
    z = f(); y = f(); x = f()  # right-to-left evaluation of (f(), f(), f())
    return np.array([x, y, z], np.float32)


def unit():
    v = vec3(rnd)
    return (v / np.linalg.norm(v.astype(np.float64))).astype(np.float32)


def angle_axis(a, n):
    n = np.asarray(n, np.float64)
    K = np.array([[0, -n[2], n[1]], [n[2], 0, -n[0]], [-n[1], n[0], 0]])
    return (np.eye(3) + math.sin(a) * K + (1 - math.cos(a)) * (K @ K)).astype(np.float32)


def random_transform(angle_range):
    n = unit()
    a = rnd(angle_range)
    T = np.zeros((3, 4), np.float32)
    T[:, :3] = angle_axis(float(a), n)
    T[:, 3] = vec3(lambda: rnd(2.0))
    return T


def inv(T):
    R, t = T[:, :3].astype(np.float64), T[:, 3].astype(np.float64)
    out = np.zeros((3, 4))
    out[:, :3] = R.T
    out[:, 3] = -R.T @ t
    return out.astype(np.float32)


def mul(A, B):
    A = A.astype(np.float64); B = B.astype(np.float64)
    out = np.zeros((3, 4))
    out[:, :3] = A[:, :3] @ B[:, :3]
    out[:, 3] = A[:, :3] @ B[:, 3] + A[:, 3]
    return out.astype(np.float32)


def jac_A(Ta, pa, na, pb, nb, va, dt):
    lib = orc.load()
    e = C.c_float()
    J = np.zeros(6, np.float32)
    arrs = [np.ascontiguousarray(x, np.float32) for x in (Ta.reshape(12), pa, na, pb, nb, va)]
    lib.orc_err_jac_vel_A(0, C.byref(e), J.ctypes.data, *(a.ctypes.data for a in arrs), dt)
    return np.float32(e.value), J


def jac_B(Tb, pa, na, pb, nb, vb, dt):
    lib = orc.load()
    e = C.c_float()
    J = np.zeros(6, np.float32)
    arrs = [np.ascontiguousarray(x, np.float32) for x in (Tb.reshape(12), pa, na, pb, nb, vb)]
    lib.orc_err_jac_vel_B(0, C.byref(e), J.ctypes.data, *(a.ctypes.data for a in arrs), dt)
    return np.float32(e.value), J


def test_motion_jacobian_3d_known_answer():
    """motion_jacobian_3d_test.cpp:68-127 restated against the oracle."""
    libc.srand(42)
    H, TOL = np.float32(1e-3), 5e-3
    n_pass = n_total = 0
    worst = 0.0
    for _ in range(20):
        Tb = random_transform(math.pi)
        Ta = random_transform(math.pi)
        pa_l = vec3(lambda: rnd(3.0)); na_l = unit()
        pb_l = vec3(lambda: rnd(3.0)); nb_l = unit()
        pa_g = (Ta[:, :3].astype(np.float64) @ pa_l + Ta[:, 3]).astype(np.float32)
        na_g = (Ta[:, :3].astype(np.float64) @ na_l).astype(np.float32)
        pb_g = (Tb[:, :3].astype(np.float64) @ pb_l + Tb[:, 3]).astype(np.float32)
        nb_g = (Tb[:, :3].astype(np.float64) @ nb_l).astype(np.float32)
        va = np.array([rnd(.5), rnd(.5), rnd(.5), rnd(.3), rnd(.3), rnd(.3)][::-1], np.float32)
        vb = np.array([rnd(.5), rnd(.5), rnd(.5), rnd(.3), rnd(.3), rnd(.3)][::-1], np.float32)
        dt = 0.1
        for which in ("A", "B"):
            if which == "A":
                _, Jan = jac_A(Ta, pa_l, na_l, pb_g, nb_g, va, dt)
                f = lambda v: jac_A(Ta, pa_l, na_l, pb_g, nb_g, v, dt)[0]
                v0 = va
            else:
                _, Jan = jac_B(Tb, pa_g, na_g, pb_l, nb_l, vb, dt)
                f = lambda v: jac_B(Tb, pa_g, na_g, pb_l, nb_l, v, dt)[0]
                v0 = vb
            Jnu = np.zeros(6, np.float32)
            for i in range(6):
                vp = v0.copy(); vp[i] += H
                vm = v0.copy(); vm[i] -= H
                Jnu[i] = (f(vp) - f(vm)) / (np.float32(2) * H)
            err = float(np.max(np.abs(Jan - Jnu)))
            worst = max(worst, err)
            n_pass += err < TOL
            n_total += 1
    assert n_pass == n_total, f"{n_pass}/{n_total} passed, worst {worst}"


def test_pose_error_jacobian_3d_known_answer():
    """pose_error_jacobian_3d_test.cpp:37-71 restated against the oracle."""
    lib = orc.load()
    libc.srand(42)
    H, TOL = np.float32(1e-4), 1e-2
    worst = 0.0
    for _ in range(20):
        B = random_transform(math.pi * 0.4)
        A = random_transform(math.pi * 0.4)
        ZXi = mul(inv(A), inv(B))
        Xm = random_transform(math.pi * 0.4)
        J = np.zeros(36, np.float32)
        lib.orc_dpose_to_pose_error(0, np.ascontiguousarray(ZXi.reshape(12)).ctypes.data,
                                    np.ascontiguousarray(Xm.reshape(12)).ctypes.data, J.ctypes.data)
        J = J.reshape(6, 6)
        Jnu = np.zeros((6, 6), np.float32)
        for i in range(6):
            cols = []
            for sgn in (1, -1):
                v = np.zeros(6, np.float32); v[i] = sgn * H
                dX = np.zeros(12, np.float32)
                lib.orc_expmap(0, v.ctypes.data, dX.ctypes.data)
                P = mul(dX.reshape(3, 4), Xm)
                e = np.zeros(6, np.float32)
                lib.orc_pose_to_pose_error(0, np.ascontiguousarray(ZXi.reshape(12)).ctypes.data,
                                           np.ascontiguousarray(P.reshape(12)).ctypes.data, e.ctypes.data)
                cols.append(e)
            Jnu[:, i] = (cols[0] - cols[1]) / (np.float32(2) * H)
        err = float(np.max(np.abs(J - Jnu)))
        worst = max(worst, err)
        assert err < TOL, f"case error {err}"


def test_canonical_sincos_accuracy():
    """The canonical sin/cos that replaces sinf/cosf on the CT warp: <= 2 ulp on [-400, 400]."""
    xs = np.concatenate([np.linspace(-400, 400, 20001, dtype=np.float32),
                         np.linspace(-1e-3, 1e-3, 2001, dtype=np.float32),
                         np.float32([0.0, 1e-9, 1e-30, math.pi / 4, math.pi / 2, math.pi, 3.0e-2])])
    worst = 0.0
    for x in xs:
        s, c = orc.sincosf(float(x))
        rs, rc = math.sin(float(x)), math.cos(float(x))
        for got, ref in ((s, rs), (c, rc)):
            ulp = float(np.spacing(np.float32(abs(ref)))) if ref != 0 else 1e-45
            err = abs(got - ref) / max(ulp, float(np.spacing(np.float32(1.0))) * 2 ** -24)
            worst = max(worst, err)
    assert worst <= 2.0, worst


def test_jacobi3_matches_eigh():
    lib = orc.load()
    rng = np.random.default_rng(7)
    for _ in range(200):
        A = rng.normal(size=(3, 3))
        A = A @ A.T * rng.uniform(1e-6, 1e2)
        if rng.uniform() < 0.3:  # nearly flat (surfel-like)
            U, _, _ = np.linalg.svd(rng.normal(size=(3, 3)))
            A = U @ np.diag([1e-8, 0.5, 2.0]) @ U.T
        ev = np.zeros(3)
        V = np.zeros(9)
        lib.orc_jacobi3(np.ascontiguousarray(A.reshape(9)).ctypes.data, ev.ctypes.data, V.ctypes.data)
        V = V.reshape(3, 3)
        w, _ = np.linalg.eigh(A)
        scale = max(1e-300, abs(w).max())
        assert np.all(np.diff(ev) >= 0)
        assert np.allclose(ev, w, atol=1e-12 * scale, rtol=1e-10)
        assert np.allclose(V.T @ V, np.eye(3), atol=1e-12)
        assert np.allclose(A @ V, V * ev, atol=1e-10 * scale)


def test_fixed_point_floor_is_exact():
    """The moment sums put every float product on a 2^-64 grid by flooring; the floor
    must be exact for every sign and magnitude -- in particular for small negative
    products, where 1 - |v| does not fit a double (checked against exact rationals)."""
    from fractions import Fraction
    rng = np.random.default_rng(11)
    f32 = lambda a: np.float32(a)
    vals = [0.0, -0.0, 1.0, -1.0, 2.0 ** -70, -(2.0 ** -70), -(2.0 ** -64), 2.0 ** -64, -3.25, 3599.9]
    for _ in range(3000):
        a = f32(rng.choice([rng.normal() * 30.0, rng.normal() * 1e-3, rng.normal() * 1e-7]))
        b = f32(rng.choice([rng.normal() * 30.0, rng.normal() * 1e-3, 1.0]))
        vals.append(float(a) * float(b))  # exact in double: 24 x 24 bit mantissas
    for v in vals:
        want = math.floor(Fraction(v) * (1 << 64))
        assert orc.fx_floor(v) == want, v


def test_voxel_restatement_known_answer():
    """Two points in one 1 m voxel and one alone; the mean is the float sum times the
    float reciprocal of the count; a voxel whose mean falls inside range_min is dropped."""
    from oracle import voxel as OV
    xyz = np.array([[2.25, 0.5, 0.0], [2.75, 0.25, 0.0], [5.5, 5.5, 1.0], [0.1, 0.1, 0.0]], np.float32)
    st = np.array([1.0, 2.0, 3.0, 4.0])
    p, t = OV.voxelize(xyz, st, range_min=0.5, range_max=20.0, space_res=1.0)
    assert p.tolist() == [[2.5, 0.375, 0.0], [5.5, 5.5, 1.0]]
    assert t.tolist() == [1.5, 3.0]
    p, t = OV.voxelize(xyz, st, range_min=0.5, range_max=20.0)  # no grid: range filter only
    assert len(p) == 3 and t.tolist() == [1.0, 2.0, 3.0]


def test_tracker_geometry_restatement():
    """The tracker oracle's FP64 pose helpers: expmap/logmap invert each other (below
    pi), the Shepperd-quaternion rotation angle equals acos((tr R - 1) / 2) on both of
    its branches, and iso_inv is the inverse of iso_mul."""
    from oracle import tracker as T
    rng = np.random.default_rng(5)
    for k in range(200):
        ang = [0.0, 1e-8, 1e-3, 0.5, 2.0, 3.1][k % 6]
        a = rng.normal(size=3)
        a *= ang / np.linalg.norm(a)
        v = list(rng.normal(size=3)) + list(a)
        X = T.expmap(v)
        assert np.allclose(T.logmap(X), v, atol=1e-7 if ang > 1e-7 else 1e-12)
        R = np.array(X).reshape(3, 4)[:, :3]
        want = math.acos(max(-1.0, min(1.0, (np.trace(R) - 1) / 2)))
        assert abs(T.rotation_angle(X) - want) <= 1e-6, (ang, T.rotation_angle(X), want)
        Y = T.expmap(list(rng.normal(size=6)))
        I = T.iso_mul(T.iso_inv(Y), Y)
        assert np.allclose(I, [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], atol=1e-12)
    # ConstVelMotionModel_ arithmetic on a known sequence: two updates by the same
    # delta from zero give (1 - alpha^2) log(delta) (alpha = (float)0.9)
    alpha = float(np.float32(0.9))
    d = T.expmap([0.2, 0.01, 0.0, 0.0, 0.0, 0.01])
    dv = T.logmap(d)
    s = [0.0] * 6
    for _ in range(2):
        s = [alpha * s[i] + (1.0 - alpha) * dv[i] for i in range(6)]
    assert np.allclose(s, np.array(dv) * (1 - alpha ** 2), rtol=1e-12)
