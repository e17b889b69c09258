"""toPointsVector + Voxelizer_::voxelize restated in numpy / Python -- TEST
INFRASTRUCTURE ONLY (the checker of kds_points_voxelize; tests/ use it).

toPointsVector (lib/kd_io/scan_utils_impl_.h:9-33): per-point stamps, else azimuth
stamps msg_t + (atan2(y, x) + pi) / (2 pi) * scan_duration, else msg_t.
Voxelizer_::voxelize (kd/utils/voxelizer_impl_.h:111-145) with add() (:68-109) and the
Accumulator (:11-58): without a voxel grid, the points with range_min^2 <= |p|^2 <=
range_max^2 (double bounds) in input order; with one, the points inside add()'s float
bounds binned by (int)(coord * (1 / space_res)) per axis (and the time bin), each
voxel's coordinates summed in float and stamps in double in input order, the mean
scaled by the float reciprocal of the count, and kept if within the double bounds.
The reference emits voxels in its hash map's order; this restatement, like the
library, sorts them by their integer index (x, y, z, t).
"""
import math

import numpy as np

f32 = np.float32


def stamps_of(xyz, stamps, msg_t, scan_duration):
    if stamps is not None:
        return np.asarray(stamps, np.float64).copy()
    if scan_duration > 0.0:
        return np.array([msg_t + (math.atan2(float(p[1]), float(p[0])) + math.pi) / (2.0 * math.pi) * scan_duration
                         for p in xyz])
    return np.full(len(xyz), msg_t)


def sq_norm(x, y, z):
    return (f32(x) * f32(x) + f32(y) * f32(y)) + f32(z) * f32(z)


def voxelize(xyz, stamps=None, msg_t=0.0, scan_duration=0.0, range_min=0.0, range_max=100.0, space_res=0.0,
             time_res=0.0, use_boundary=False):
    xyz = np.asarray(xyz, np.float32).reshape(-1, 3)
    st = stamps_of(xyz, stamps, msg_t, scan_duration)
    rmin, rmax, res, tres = f32(range_min), f32(range_max), f32(space_res), f32(time_res)
    rmin2, rmax2 = float(rmin) ** 2, float(rmax) ** 2
    if res <= 0:
        keep = [i for i in range(len(xyz)) if not (float(sq_norm(*xyz[i])) < rmin2 or float(sq_norm(*xyz[i])) > rmax2)]
        return xyz[keep].copy(), st[keep].copy()
    b = f32(math.sqrt(float(res * f32(3)))) if use_boundary else f32(0)
    hi2 = f32(float(rmax + b) ** 2)
    lo2 = f32(float(max(f32(0), rmin - b)) ** 2)
    inv = f32(1) / res
    inv_t = f32(1) / tres if tres > 0 else f32(0)
    t0 = st.min()
    acc = {}
    for i in range(len(xyz)):
        x, y, z = xyz[i]
        n2 = sq_norm(x, y, z)
        if n2 > hi2 or n2 < lo2:
            continue
        key = (int(f32(x) * inv), int(f32(y) * inv), int(f32(z) * inv),
               int((st[i] - t0) * float(inv_t)) if tres > 0 else 0)
        a = acc.setdefault(key, [f32(0), f32(0), f32(0), 0.0, 0])
        a[0] = f32(a[0] + x)
        a[1] = f32(a[1] + y)
        a[2] = f32(a[2] + z)
        a[3] = a[3] + float(st[i])
        a[4] += 1
    out_p, out_t = [], []
    for key in sorted(acc):
        sx, sy, sz, ss, c = acc[key]
        r = f32(1) / f32(c)
        m = (f32(sx * r), f32(sy * r), f32(sz * r))
        n2 = float(sq_norm(*m))
        if n2 > rmax2 or n2 < rmin2:
            continue
        out_p.append(m)
        out_t.append(ss * float(r))
    return np.array(out_p, np.float32).reshape(-1, 3), np.array(out_t, np.float64)
