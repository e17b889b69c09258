"""Precision study of the product's numerics: per-surfel residuals, Jacobians and H,b
terms in FP32 with Kahan-compensated warp sums, FP64 block partials, FP64 cross-block
sums, Cholesky solve, SE(3) exp and pose composition -- against the all-FP64 oracle, for
seeded CT-ICP perturbations of 0-0.5 m and 0-5 degrees about random axes.

Default: a 64 x 1024 scan against a map of 6 prior scans, 24 perturbations (minutes of
CPU at most).  With KDS_PRECISION_FULL=1: the 128 x 2048 scan against a 4M-surfel map
and 1000 perturbations; KDS_PRECISION_OUT=<path> writes the summary there as JSON.
All perturbations run on the GPU in one batch (kds_batch_run); the oracle runs them in
a process pool.
"""
import json
import multiprocessing as mp
import os
import tempfile

import numpy as np
import pytest

from conftest import pose_err

pytestmark = pytest.mark.gpu

FULL = os.environ.get("KDS_PRECISION_FULL", "0") == "1"
TREE = dict(leaf_max_points=16)
CT = dict(max_error=0.5, max_iterations=15, velocity_damping=10.0)
VEL = np.array([10.0, 0.0, 0.0, 0.0, 0.0, np.deg2rad(30.0)])


def _oracle_worker(args):
    """One oracle alignment, all-FP64 (mode 64) or in the product's semantics (runs in a
    spawned process)."""
    path, X0, v0, mode = args
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    from oracle import orc
    g = globals()
    if g.get("_cache_path") != path:
        d = np.load(path)
        g["_M"] = orc.OTree.from_nodes(d["mean"], d["dir"], d["dts_mean"], d["left"], d["right"])
        g["_T"] = orc.OTree.build(d["xyz"], d["st"], orc.tree_params(**TREE))
        g["_cache_path"] = path
    r = orc.align(orc.KIND_CT, orc.MODE_FP64 if mode == 64 else orc.MODE_MIXED, g["_M"], g["_T"],
                  orc.align_params(**CT), X0, v0=v0)
    return r["X"], r["ret"]


def _setup():
    from kd_slam2_b200 import synth
    boxes = synth.scene(1003)
    if FULL:
        map_scans, map_cols, beams, cols, n = 68, 8192, 128, 2048, 1000
    else:
        map_scans, map_cols, beams, cols, n = 6, 2048, 64, 1024, 24
    pts = []
    for k in range(map_scans):
        P = synth.pose((-34.0 + k if FULL else -6.0 + k, 0.0, 1.8))
        xyz, _ = synth.scan(boxes, P, beams=128, cols=map_cols, elev=(-22.5, 22.5), seed=5000 + k, threads=16)
        pts.append(synth.transform(xyz, P))
    map_xyz = np.ascontiguousarray(np.concatenate(pts))
    X_true = synth.pose((0.0, 0.0, 1.8))
    xyz, st = synth.scan(boxes, X_true, vel=VEL, beams=beams, cols=cols, elev=(-22.5, 22.5), seed=5999, threads=16)
    rng = np.random.default_rng(3000)
    X0s = []
    for _ in range(n):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        a = rng.normal(size=3)
        a /= np.linalg.norm(a)
        X0s.append(synth.pose(X_true[:, 3] + rng.uniform(0, 0.5) * d, np.deg2rad(rng.uniform(0, 5.0)) * a))
    return map_xyz, xyz, st, X_true, X0s


def test_fp32_kahan_fp64_solve_against_fp64_oracle():
    import kd_slam2_b200 as kds
    from kd_slam2_b200.abi import KDS_CTICP
    map_xyz, xyz, st, X_true, X0s = _setup()
    gen = kds.TreeGeneratorB2003D(**TREE)
    M = gen.make_tree(map_xyz)
    T = gen.make_tree(xyz, st)
    v0 = VEL * 0.9
    params = kds.aligner_params(**CT)
    jobs = [kds.make_job(KDS_CTICP, M, T, params, X=X0, v=v0) for X0 in X0s]
    res = kds.Batch().run(jobs)
    me = M.export()
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "study.npz")
        np.savez(path, mean=me["mean"], dir=me["dir"], dts_mean=me["dts_mean"], left=me["left"],
                 right=me["right"], xyz=xyz, st=st)
        ctx = mp.get_context("spawn")
        with ctx.Pool(min(16, os.cpu_count() or 1)) as pool:
            ref = pool.map(_oracle_worker, [(path, X0, v0, 64) for X0 in X0s], chunksize=1)
            mix = pool.map(_oracle_worker, [(path, X0, v0, 32) for X0 in X0s], chunksize=1)
    et, er, tt, tr_, conv = [], [], [], [], []
    for j, (X64, ret64) in zip(res, ref):
        X = np.array(j.X[:]).reshape(3, 4)
        a, b = pose_err(X, X64)
        et.append(a)
        er.append(b)
        c, d = pose_err(X, X_true)
        tt.append(c)
        tr_.append(d)
        g, h = pose_err(X64, X_true)
        conv.append(g < 0.05 and h < np.deg2rad(0.5))  # the FP64 run converged near the truth
    et, er, conv = np.array(et), np.array(er), np.array(conv)
    ok = (et <= 1e-5) & (er <= 1e-5)
    em = np.array([max(pose_err(np.array(j.X[:]).reshape(3, 4), Xm)) for j, (Xm, _) in zip(res, mix)])
    summary = {
        "scan_points": int(len(xyz)), "scan_leaves": int(T.num_leaves), "map_points": int(len(map_xyz)),
        "map_leaves": int(M.num_leaves), "perturbations": len(X0s),
        "t_err_vs_fp64_m": {"median": float(np.median(et)), "p99": float(np.percentile(et, 99)), "max": float(et.max())},
        "r_err_vs_fp64_rad": {"median": float(np.median(er)), "p99": float(np.percentile(er, 99)), "max": float(er.max())},
        "within_1e-5": int(np.sum(ok)),
        "fp64_converged": int(np.sum(conv)),
        "within_1e-5_of_converged": int(np.sum(ok & conv)),
        "t_err_vs_fp64_m_converged_p99": float(np.percentile(et[conv], 99)) if conv.any() else None,
        "t_err_vs_truth_m_median": float(np.median(tt)), "r_err_vs_truth_rad_median": float(np.median(tr_)),
        "vs_product_semantics_oracle": {"within_1e-5": int(np.sum(em <= 1e-5)), "median": float(np.median(em)),
                                        "max": float(em.max())},
    }
    out = os.environ.get("KDS_PRECISION_OUT")
    if out:
        with open(out, "w") as f:
            json.dump(summary, f, indent=1)
    # The descent and the gates run in FP32, as in the reference, so a query within an ulp
    # of a split plane or a gate can take another branch than in FP64; one changed
    # correspondence moves the path, and over 15 iterations from up to 0.5 m / 5 deg the
    # runs can end apart.  The same happens, more rarely, against the oracle in the
    # product's own semantics, whose FP64 sums run in another order than the GPU's
    # Kahan-compensated tiles: a last-bit difference in H,b changes the next float cache.
    assert np.median(et) <= 1e-5 and np.median(er) <= 1e-5, summary
    assert np.sum(em <= 1e-5) >= 0.9 * len(X0s), summary
