"""Multi-view bundle-adjustment factor assembly, restated in numpy -- TEST
INFRASTRUCTURE ONLY (the checker of kds_batch_assemble; tests/ use it).

MultiViewICPFactor_::compute (kd/map/multiview_icp_factor_impl_.h:30-62) and
MultiViewCTICPFactor_::compute (kd/map/multiview_cticp_factor_impl_.h:33-83): a factor
is enabled when ICPStats_::inlierRatio() (kd/icp/icp_stats_.h:28-31, float) exceeds
disable_inlier_ratio; an enabled factor adds its upper-triangular blocks (factor-local
variable order) and its b blocks.  Here the global system is kept as the upper block
triangle over the caller's variable numbers (row <= column, transposed where the
factor's order is the other way round), summed in FP64 in factor order.
"""
import numpy as np


def inlier_ratio(stats) -> np.float32:
    leaves = (stats.num_inliers + stats.num_outliers + stats.num_bad + stats.num_err_normal + stats.num_err_fn)
    if not leaves:
        return np.float32(0.0)
    return np.float32(stats.num_inliers) / np.float32(leaves)


def factor_blocks(job):
    """The (r, c, M) block updates and (r, v) b updates of one factor, factor-local order."""
    if job.type == 0:  # ICP: x0 = fixed pose, x1 = moving pose
        H = np.array(job.H[:36]).reshape(6, 6)
        b = np.array(job.b[:6])
        return [(0, 0, H), (0, 1, -H), (1, 1, H)], [(0, b), (1, -b)]
    H = np.array(job.H[:144]).reshape(12, 12)  # CT dual: x0 pose_A, v0 vel_A, x1 pose_B, v1 vel_B
    b = np.array(job.b[:12])
    Hpp, Hpv, Hvv = H[:6, :6], H[:6, 6:], H[6:, 6:]
    HpVb = np.array(job.H_cross_pose_vel_B[:]).reshape(6, 6)
    HvAb = np.array(job.H_cross_vel_AB[:]).reshape(6, 6)
    HVbVb = np.array(job.H_vel_B[:]).reshape(6, 6)
    bVb = np.array(job.b_vel_B[:])
    hb = [(0, 0, Hpp), (0, 1, -HpVb), (0, 2, -Hpp), (0, 3, -Hpv), (1, 1, HVbVb), (1, 2, HpVb.T),
          (1, 3, HvAb.T), (2, 2, Hpp), (2, 3, Hpv), (3, 3, Hvv)]
    bb = [(0, b[:6]), (1, -bVb), (2, -b[:6]), (3, -b[6:])]
    return hb, bb


def assemble(jobs, factors, num_vars: int, disable_inlier_ratio: float):
    """jobs: kds_job outputs; factors: (job, vars).  Returns ({(row, col): 6x6}, b, enabled)."""
    H, b = {}, np.zeros((num_vars, 6))
    enabled = []
    for job_i, vs in factors:
        job = jobs[job_i]
        en = bool(inlier_ratio(job.stats) > np.float32(disable_inlier_ratio))
        enabled.append(en)
        hb, bb = factor_blocks(job)
        for r, c, M in hb:
            gr, gc = vs[r], vs[c]
            adds = [M] if gr != gc or r == c else [M, M.T]
            if gr > gc:
                gr, gc, adds = gc, gr, [A.T for A in adds]
            blk = H.setdefault((gr, gc), np.zeros((6, 6)))
            for A in adds:
                if en:
                    blk += A
        for r, v in bb:
            if en:
                b[vs[r]] += v
    return H, b, np.array(enabled)
