"""ctypes binding of the CPU oracle (liborc.so) -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg, always
as the checker or the timed CPU baseline, never as part of the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborc.so")

MODE_REF32, MODE_MIXED, MODE_FP64 = 0, 1, 2
KIND_ICP, KIND_CT, KIND_CT_DUAL = 0, 1, 2


class TreeParams(C.Structure):
    _fields_ = [("propagate_normal", C.c_int32), ("tree_min_good_leaves", C.c_int32),
                ("leaf_min_points", C.c_int32), ("leaf_max_points", C.c_int32), ("leaf_density", C.c_float),
                ("leaf_min_normal_incidence", C.c_float), ("leaf_eigenvalue_threshold", C.c_float),
                ("leaf_normal_eigenratio", C.c_float), ("prune_min_normal_incidence", C.c_float),
                ("max_level", C.c_int32)]


class AlignParams(C.Structure):
    _fields_ = [("kernel_threshold", C.c_float), ("damping", C.c_float), ("max_error", C.c_float),
                ("min_normal_cos", C.c_float), ("min_good_measurements", C.c_int32), ("max_iterations", C.c_int32),
                ("velocity_damping", C.c_float), ("term_crit", C.c_int32), ("d_pert", C.c_float),
                ("d_score", C.c_float)]


class OStats(C.Structure):
    _fields_ = [("num_inliers", C.c_int32), ("num_outliers", C.c_int32), ("num_bad", C.c_int32),
                ("num_err_normal", C.c_int32), ("num_err_fn", C.c_int32), ("chi2", C.c_float),
                ("chi2_kernelized", C.c_float), ("pert_pose_norm", C.c_float), ("pert_vel_norm", C.c_float)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class OPrior(C.Structure):
    _fields_ = [("enabled", C.c_int32), ("X_ref", C.c_double * 12), ("Z", C.c_double * 12),
                ("info", C.c_double * 36)]


class OResult(C.Structure):
    _fields_ = [("ret", C.c_int32), ("iterations", C.c_int32), ("H", C.c_double * 144), ("b", C.c_double * 12),
                ("dx", C.c_double * 12), ("stats", OStats), ("log", OStats * 64)]


def tree_params(**kw) -> TreeParams:
    p = TreeParams(0, 10, 5, 30, 100.0, 0.1, 1e-3, 0.1, 0.1, 48)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def align_params(**kw) -> AlignParams:
    p = AlignParams(0.1, 1.0, 1.0, float(np.float32(np.cos(25.0 / 180.0 * np.pi))), 10, 20, 100.0, 0, 1e-3, 1e-3)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


_LIB = None


def load() -> C.CDLL:
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    sig = {
        "orc_tree_build": (P, [P, P, C.c_int64, C.POINTER(TreeParams)]),
        "orc_tree_build_ref32": (P, [P, P, C.c_int64, C.POINTER(TreeParams), C.c_int32]),
        "orc_tree_from_nodes": (P, [P, P, P, P, P, C.c_int64]),
        "orc_tree_num_nodes": (C.c_int64, [P]),
        "orc_tree_num_leaves": (C.c_int64, [P]),
        "orc_tree_num_points": (C.c_int64, [P]),
        "orc_tree_num_unpruned": (C.c_int64, [P]),
        "orc_tree_accepted": (C.c_int32, [P]),
        "orc_tree_ts_start": (C.c_double, [P]),
        "orc_tree_export": (None, [P] * 12),
        "orc_tree_root": (None, [P, P, P, P]),
        "orc_tree_free": (None, [P]),
        "orc_align": (C.c_int32, [C.c_int32, C.c_int32, P, P, C.c_int32, P, C.POINTER(AlignParams),
                                  C.POINTER(OPrior), P, P, P, C.c_int32, C.c_int32, C.POINTER(OResult)]),
        "orc_linearize": (None, [C.c_int32, P, P, P, P, P, C.POINTER(AlignParams), C.c_int32, P, P, P, P,
                                 C.POINTER(OStats)]),
        "orc_align_recorded": (C.c_int32, [C.c_int32, P, P, C.c_int32, P, C.POINTER(AlignParams), P, P, P,
                                           C.POINTER(OResult), P, P]),
        "orc_align_replay64": (None, [C.c_int32, P, P, C.c_int32, P, C.POINTER(AlignParams), P, P, P, C.c_int32,
                                      P, P]),
        "orc_sincos_canon_d": (None, [C.c_double, P, P]),
        "orc_product_caches": (None, [P, P, P]),
        "orc_pose_hessian": (C.c_int32, [P, P]),
        "orc_sincosf": (None, [C.c_float, P, P]),
        "orc_err_jac_vel_A": (None, [C.c_int32, P, P, P, P, P, P, P, P, C.c_double]),
        "orc_err_jac_vel_B": (None, [C.c_int32, P, P, P, P, P, P, P, P, C.c_double]),
        "orc_pose_to_pose_error": (None, [C.c_int32, P, P, P]),
        "orc_dpose_to_pose_error": (None, [C.c_int32, P, P, P]),
        "orc_expmap": (None, [C.c_int32, P, P]),
        "orc_iso_mul": (None, [P, P, P]),
        "orc_jacobi3": (None, [P, P, P]),
        "orc_fx_floor": (None, [C.c_double, C.POINTER(C.c_int64), C.POINTER(C.c_uint64)]),
        "orc_warp_leaf": (None, [P, C.c_float, P, P, P, P]),
        "orc_tree_apply_velocities": (None, [P, P]),
        "orc_tree_apply_isometry": (None, [P, P]),
        "orc_tree_clone": (P, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _LIB = lib
    return lib


class OTree:
    """Oracle tree handle (canonical build or a node array)."""

    def __init__(self, h):
        self.h = h

    def __del__(self):
        if self.h:
            load().orc_tree_free(self.h)
            self.h = None

    @staticmethod
    def build(xyz, stamps=None, params: TreeParams | None = None) -> "OTree":
        lib = load()
        xyz = np.ascontiguousarray(xyz, np.float32)
        st = None if stamps is None else np.ascontiguousarray(stamps, np.float64)
        p = params or tree_params()
        h = lib.orc_tree_build(xyz.ctypes.data, None if st is None else st.ctypes.data, len(xyz), C.byref(p))
        return OTree(h)

    @staticmethod
    def build_ref32(xyz, stamps=None, params: TreeParams | None = None, parallel_level: int = -1) -> "OTree":
        """The reference's float build arithmetic (timed CPU baseline; not bit-comparable)."""
        lib = load()
        xyz = np.ascontiguousarray(xyz, np.float32)
        st = None if stamps is None else np.ascontiguousarray(stamps, np.float64)
        p = params or tree_params()
        h = lib.orc_tree_build_ref32(xyz.ctypes.data, None if st is None else st.ctypes.data, len(xyz), C.byref(p),
                                     int(parallel_level))
        return OTree(h)

    @staticmethod
    def from_nodes(mean, dir, dts_mean, left, right) -> "OTree":
        lib = load()
        mean = np.ascontiguousarray(mean, np.float32)
        dir = np.ascontiguousarray(dir, np.float32)
        dm = np.ascontiguousarray(dts_mean, np.float64)
        left = np.ascontiguousarray(left, np.int32)
        right = np.ascontiguousarray(right, np.int32)
        return OTree(lib.orc_tree_from_nodes(mean.ctypes.data, dir.ctypes.data, dm.ctypes.data, left.ctypes.data,
                                             right.ctypes.data, len(mean)))

    @property
    def num_nodes(self) -> int:
        return load().orc_tree_num_nodes(self.h)

    @property
    def num_leaves(self) -> int:
        return load().orc_tree_num_leaves(self.h)

    @property
    def accepted(self) -> bool:
        return bool(load().orc_tree_accepted(self.h))

    def export(self) -> dict:
        lib = load()
        n, nl, npnt = self.num_nodes, self.num_leaves, lib.orc_tree_num_points(self.h)
        out = {"mean": np.zeros((n, 3), np.float32), "dir": np.zeros((n, 3), np.float32),
               "dts_mean": np.zeros(n), "dts_cov": np.zeros(n), "start": np.zeros(n, np.int64),
               "end": np.zeros(n, np.int64), "left": np.zeros(n, np.int32), "right": np.zeros(n, np.int32),
               "level": np.zeros(n, np.int32), "leaves": np.zeros(nl, np.int64), "perm": np.zeros(npnt, np.int64)}
        lib.orc_tree_export(self.h, *(out[k].ctypes.data for k in ("mean", "dir", "dts_mean", "dts_cov", "start",
                                                                    "end", "left", "right", "level", "leaves",
                                                                    "perm")))
        out["ts_start"] = lib.orc_tree_ts_start(self.h)
        out["num_unpruned"] = lib.orc_tree_num_unpruned(self.h)
        out["accepted"] = self.accepted
        out.update(self.root())
        return out

    def apply_velocities_in_place(self, v) -> None:
        """Tree_::applyVelocitiesInPlace: every node warped by v * (float)dts_mean."""
        vv = np.ascontiguousarray(v, np.float32)
        load().orc_tree_apply_velocities(self.h, vv.ctypes.data)

    def apply_isometry_in_place(self, X) -> None:
        """Tree_::applyIsometryInPlace with a 3x4 float isometry."""
        XX = np.ascontiguousarray(np.asarray(X, np.float32).reshape(12))
        load().orc_tree_apply_isometry(self.h, XX.ctypes.data)

    def clone(self) -> "OTree":
        return OTree(load().orc_tree_clone(self.h))

    def root(self) -> dict:
        """Tree_::root_mean / root_eigenvalues / root_eigenvectors (3x3, columns = vectors)."""
        m, ev, V = np.zeros(3, np.float32), np.zeros(3, np.float32), np.zeros(9, np.float32)
        load().orc_tree_root(self.h, m.ctypes.data, ev.ctypes.data, V.ctypes.data)
        return {"root_mean": m, "root_eigenvalues": ev, "root_eigenvectors": V.reshape(3, 3).T.copy()}


def align(kind: int, mode: int, fixed, moving: OTree, params: AlignParams, X0, v0=None, fixed_X=None,
          fixed_v=None, prior=None, stats_mode: bool = False, num_threads: int = 1):
    """Runs TreeAlignerBase_::compute.  fixed: OTree or list of (OTree, X) entries."""
    lib = load()
    if isinstance(fixed, OTree):
        fixed = [(fixed, np.eye(3, 4) if fixed_X is None else fixed_X)]
    hs = (C.c_void_p * len(fixed))(*[f.h for f, _ in fixed])
    FX = np.ascontiguousarray(np.stack([np.asarray(x, np.float64).reshape(12) for _, x in fixed]))
    X = np.ascontiguousarray(np.asarray(X0, np.float64).reshape(12)).copy()
    v = np.zeros(6) if v0 is None else np.ascontiguousarray(v0, np.float64).copy()
    fv = np.zeros(6) if fixed_v is None else np.ascontiguousarray(fixed_v, np.float64)
    res = OResult()
    pr = None
    if prior is not None:
        pr = OPrior()
        pr.enabled = 1
        pr.X_ref[:] = list(np.asarray(prior[0], np.float64).reshape(12))
        pr.Z[:] = list(np.asarray(prior[1], np.float64).reshape(12))
        pr.info[:] = list(np.asarray(prior[2], np.float64).reshape(36))
    ret = lib.orc_align(kind, mode, hs, FX.ctypes.data, len(fixed), moving.h, C.byref(params),
                        C.byref(pr) if pr is not None else None, X.ctypes.data, v.ctypes.data, fv.ctypes.data,
                        1 if stats_mode else 0, num_threads, C.byref(res))
    D = 6 if kind == KIND_ICP else 12
    return {"ret": ret, "X": X.reshape(3, 4), "v": v, "iterations": res.iterations,
            "H": np.array(res.H[:D * D]).reshape(D, D), "b": np.array(res.b[:D]), "dx": np.array(res.dx[:D]),
            "stats": res.stats.as_dict(), "log": [res.log[i].as_dict() for i in range(min(res.iterations, 64))]}


def _fixed_entries(fixed, fixed_X):
    if isinstance(fixed, OTree):
        fixed = [(fixed, np.eye(3, 4) if fixed_X is None else fixed_X)]
    hs = (C.c_void_p * len(fixed))(*[f.h for f, _ in fixed])
    FX = np.ascontiguousarray(np.stack([np.asarray(x, np.float64).reshape(12) for _, x in fixed]))
    return fixed, hs, FX


def align_recorded(kind: int, fixed, moving: OTree, params: AlignParams, X0, v0=None, fixed_X=None, fixed_v=None):
    """MODE_MIXED compute() (the product's semantics and summation order) that also
    returns every iteration's correspondences and status, shape (iterations, entries,
    moving leaves), for align_replay64."""
    lib = load()
    fixed, hs, FX = _fixed_entries(fixed, fixed_X)
    X = np.ascontiguousarray(np.asarray(X0, np.float64).reshape(12)).copy()
    v = np.zeros(6) if v0 is None else np.ascontiguousarray(v0, np.float64).copy()
    fv = np.zeros(6) if fixed_v is None else np.ascontiguousarray(fixed_v, np.float64)
    nl = moving.num_leaves
    cap = max(1, params.max_iterations) * len(fixed) * nl
    match = np.zeros(cap, np.int32)
    status = np.zeros(cap, np.int32)
    res = OResult()
    ret = lib.orc_align_recorded(kind, hs, FX.ctypes.data, len(fixed), moving.h, C.byref(params), X.ctypes.data,
                                 v.ctypes.data, fv.ctypes.data, C.byref(res), match.ctypes.data, status.ctypes.data)
    it = res.iterations
    shape = (it, len(fixed), nl)
    return {"ret": ret, "X": X.reshape(3, 4), "v": v, "iterations": it,
            "match": match[:it * len(fixed) * nl].reshape(shape), "status": status[:it * len(fixed) * nl].reshape(shape)}


def align_replay64(kind: int, fixed, moving: OTree, params: AlignParams, X0, match, status, v0=None, fixed_X=None,
                   fixed_v=None):
    """All-FP64 Gauss-Newton steps that reuse recorded correspondences and inlier sets
    (one step per recorded iteration): the arithmetic error of the FP32 per-leaf terms
    with every branch held fixed.  Returns (X, v)."""
    lib = load()
    fixed, hs, FX = _fixed_entries(fixed, fixed_X)
    X = np.ascontiguousarray(np.asarray(X0, np.float64).reshape(12)).copy()
    v = np.zeros(6) if v0 is None else np.ascontiguousarray(v0, np.float64).copy()
    fv = np.zeros(6) if fixed_v is None else np.ascontiguousarray(fixed_v, np.float64)
    m = np.ascontiguousarray(match, np.int32)
    st = np.ascontiguousarray(status, np.int32)
    lib.orc_align_replay64(kind, hs, FX.ctypes.data, len(fixed), moving.h, C.byref(params), X.ctypes.data,
                           v.ctypes.data, fv.ctypes.data, int(m.shape[0]), m.ctypes.data, st.ctypes.data)
    return X.reshape(3, 4), v


def sincos_canon_d(x: float):
    s, c = C.c_double(), C.c_double()
    load().orc_sincos_canon_d(float(x), C.byref(s), C.byref(c))
    return s.value, c.value


def linearize(kind: int, fixed: OTree, moving: OTree, caches36, params: AlignParams, v=None, fixed_v=None,
              stats_mode: bool = False):
    lib = load()
    n = moving.num_leaves
    c = np.ascontiguousarray(caches36, np.float32)
    vv = np.zeros(6, np.float32) if v is None else np.ascontiguousarray(v, np.float32)
    fv = np.zeros(6, np.float32) if fixed_v is None else np.ascontiguousarray(fixed_v, np.float32)
    match = np.zeros(n, np.int32)
    status = np.zeros(n, np.int32)
    D = {KIND_ICP: 6, KIND_CT: 12, KIND_CT_DUAL: 18}[kind]
    H = np.zeros(D * D)
    b = np.zeros(D)
    st = OStats()
    lib.orc_linearize(kind, fixed.h, moving.h, c.ctypes.data, vv.ctypes.data, fv.ctypes.data, C.byref(params),
                      1 if stats_mode else 0, match.ctypes.data, status.ctypes.data, H.ctypes.data, b.ctypes.data,
                      C.byref(st))
    return match, status, H.reshape(D, D), b, st.as_dict()


def fx_floor(v: float) -> int:
    """floor(v * 2^64) as computed by the oracle's moment sums (a Python int)."""
    hi, lo = C.c_int64(), C.c_uint64()
    load().orc_fx_floor(float(v), C.byref(hi), C.byref(lo))
    return hi.value * (1 << 64) + lo.value


def sincosf(x: float):
    s, c = C.c_float(), C.c_float()
    load().orc_sincosf(x, C.byref(s), C.byref(c))
    return s.value, c.value


def pose_hessian(H12) -> np.ndarray:
    """CTICP_::poseHessian: Schur complement of a 12x12 CT-ICP H over its velocity block."""
    H = np.ascontiguousarray(np.asarray(H12, np.float64).reshape(144))
    out = np.zeros(36)
    if not load().orc_pose_hessian(H.ctypes.data, out.ctypes.data):
        raise ValueError("velocity block is singular")
    return out.reshape(6, 6)


def product_caches(X, Xf=None) -> np.ndarray:
    """Float caches Xm, Xf, Xmf exactly as the product derives them from FP64 poses."""
    X = np.ascontiguousarray(np.asarray(X, np.float64).reshape(12))
    Xf = np.ascontiguousarray(np.eye(3, 4) if Xf is None else np.asarray(Xf, np.float64).reshape(12))
    out = np.zeros(36, np.float32)
    load().orc_product_caches(X.ctypes.data, Xf.ctypes.data, out.ctypes.data)
    return out


def caches_from(X, Xf=None) -> np.ndarray:
    """Float caches Xm, Xf, Xmf computed in double and rounded, as the product does."""
    X = np.asarray(X, np.float64).reshape(3, 4)
    Xf = np.eye(3, 4) if Xf is None else np.asarray(Xf, np.float64).reshape(3, 4)
    R, t = Xf[:, :3], Xf[:, 3]
    iXf = np.zeros((3, 4))
    iXf[:, :3] = R.T
    iXf[:, 3] = -(R.T @ t)
    Xmf = np.zeros((3, 4))
    Xmf[:, :3] = iXf[:, :3] @ X[:, :3]
    Xmf[:, 3] = iXf[:, :3] @ X[:, 3] + iXf[:, 3]
    return np.concatenate([X.reshape(12), Xf.reshape(12), Xmf.reshape(12)]).astype(np.float32)


def warp_leaf(v6, dt, m, n):
    lib = load()
    v = np.ascontiguousarray(v6, np.float32)
    m = np.ascontiguousarray(m, np.float32)
    n = np.ascontiguousarray(n, np.float32)
    mo = np.zeros(3, np.float32)
    no = np.zeros(3, np.float32)
    lib.orc_warp_leaf(v.ctypes.data, float(np.float32(dt)), m.ctypes.data, n.ctypes.data, mo.ctypes.data,
                      no.ctypes.data)
    return mo, no
