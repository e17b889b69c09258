"""Seeded single-alignment workloads of the plain drop-in, one per named configuration.

Scene: the box scene of `synth` (ground plane and 40 axis-aligned boxes 2-15 m tall),
scans cast by the spinning-LiDAR model with 2 cm Gaussian range noise, 1-60 m ranges.

  rigid_16x1024        rigid point-to-plane ICP: a 16 x 1024 scan (16,384 rays) against
                       the tree of a second scan at the true pose; initial guess 0.2 m /
                       2 deg off; 10 Gauss-Newton iterations, 0.5 m max error
                       (the reference demo apps/tests/icp/kd_icp_main.cpp:52-64)
  ct_64x1024_1m_map    CT-ICP with deskew: a 64 x 1024 scan (65,536 rays) taken while
                       moving at 10 m/s and 30 deg/s over a 0.1 s sweep, against the tree of
                       20 prior static scans of 128 x 8192 rays (about 1.2M surfels);
                       15 iterations (apps/tests/cticp/kd_cticp_main.cpp:62-81)
  ct_128x2048_4m_map   the precision study: a 128 x 2048 scan (262,144 rays) with the same
                       motion against 68 prior scans (about 4.2M surfels), perturbations of
                       0-0.5 m and 0-5 deg about random axes

Each returns a dict with the map points (world frame), the scan points and stamps
(sensor frame, stamps in seconds), the true pose, the initial guesses and velocities,
the aligner kind and its parameters.
"""
from __future__ import annotations

import numpy as np

from . import synth

TREE = dict(leaf_max_points=16)
VEL = np.array([10.0, 0.0, 0.0, 0.0, 0.0, np.deg2rad(30.0)])
ELEV = (-22.5, 22.5)


def _unit(rng):
    d = rng.normal(size=3)
    return d / np.linalg.norm(d)


def rigid_16x1024(seed: int = 1001) -> dict:
    boxes = synth.scene(seed)
    X_true = synth.pose((0.0, 0.0, 1.8))
    map_xyz, _ = synth.scan(boxes, X_true, beams=16, cols=1024, elev=(-15.0, 15.0), seed=seed + 10)
    xyz, st = synth.scan(boxes, X_true, beams=16, cols=1024, elev=(-15.0, 15.0), seed=seed + 11)
    rng = np.random.default_rng(seed)
    X0 = synth.pose(0.2 * _unit(rng), np.deg2rad(2.0) * _unit(rng))
    # the map is a scan at the true pose: the moving scan aligns onto its sensor frame
    return dict(name="rigid_16x1024", kind="icp", map_xyz=map_xyz, xyz=xyz, st=st, X_true=np.eye(3, 4),
                X0s=[X0], v0=None, params=dict(max_error=0.5, max_iterations=10), tree=TREE)


def _static_map(boxes, scans: int, x0: float, seed0: int, cols: int = 8192) -> np.ndarray:
    pts = []
    for k in range(scans):
        P = synth.pose((x0 + k, 0.0, 1.8))
        xyz, _ = synth.scan(boxes, P, beams=128, cols=cols, elev=ELEV, seed=seed0 + k, threads=16)
        pts.append(synth.transform(xyz, P))
    return np.ascontiguousarray(np.concatenate(pts))


def ct_64x1024_1m_map(seed: int = 1003, map_scans: int = 20) -> dict:
    boxes = synth.scene(seed)
    map_xyz = _static_map(boxes, map_scans, -20.0, 3000)
    X_true = synth.pose((0.0, 0.0, 1.8))
    xyz, st = synth.scan(boxes, X_true, vel=VEL, beams=64, cols=1024, elev=ELEV, seed=2000, threads=16)
    rng = np.random.default_rng(3000)
    X0 = synth.pose(X_true[:, 3] + 0.1 * _unit(rng), np.deg2rad(1.0) * _unit(rng))
    v0 = VEL + rng.normal(size=6) * np.array([0.5, 0.5, 0.1, 0.01, 0.01, 0.05])
    return dict(name="ct_64x1024_1m_map", kind="ct", map_xyz=map_xyz, xyz=xyz, st=st, X_true=X_true, X0s=[X0],
                v0=v0, params=dict(max_error=0.5, max_iterations=15, velocity_damping=10.0), tree=TREE)


def ct_128x2048_4m_map(perturbations: int = 1000, seed: int = 1003, map_scans: int = 68) -> dict:
    boxes = synth.scene(seed)
    map_xyz = _static_map(boxes, map_scans, -34.0, 5000)
    X_true = synth.pose((0.0, 0.0, 1.8))
    xyz, st = synth.scan(boxes, X_true, vel=VEL, beams=128, cols=2048, elev=ELEV, seed=5999, threads=16)
    rng = np.random.default_rng(3000)
    X0s = []
    for _ in range(perturbations):
        d, a = _unit(rng), _unit(rng)
        X0s.append(synth.pose(X_true[:, 3] + rng.uniform(0, 0.5) * d, np.deg2rad(rng.uniform(0, 5.0)) * a))
    return dict(name="ct_128x2048_4m_map", kind="ct", map_xyz=map_xyz, xyz=xyz, st=st, X_true=X_true, X0s=X0s,
                v0=VEL * 0.9, params=dict(max_error=0.5, max_iterations=15, velocity_damping=10.0), tree=TREE)
