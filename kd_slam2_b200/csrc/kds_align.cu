// Fused ICP / CT-ICP linearization and on-device Gauss-Newton.
//
// One launch = one Gauss-Newton iteration for every job of a batch.  A job is one
// alignment (ICP_::compute / CTICP_::compute, kd/icp/tree_aligner_base_.h:100-115)
// or one buildQuadraticForm; it has one moving leaf set and one or more fixed
// entries (the _fixed_forest of kd/icp/icp_impl_.h:55-71).  The grid is a flat list of
// tiles (job, entry, 128 moving leaves); each block:
//   1. runs quadraticTerm for its leaves (kd/icp/icp_impl_.h:102-152,
//      kd/cticp/cticp_impl_.h:105-293): optional CT warp, greedy descent through the
//      fixed tree, gates, symmetric error, Jacobian, robust weight -- the gating path in
//      exact single roundings so matches and masks equal the CPU oracle bit for bit;
//   2. reduces gamma*J^T J and gamma*J^T e over its leaves warp-cooperatively: each
//      lane owns a few of the D(D+1)/2+D entries and sums them over the warp's 32
//      leaves with Kahan compensation; warps are combined in FP64 into one block
//      partial (no per-leaf workspace, replacing ICP_kernel + ~2x14 _reduce1 passes,
//      kd/icp/icp_cuda_impl_.cuh:68-132, kd/cuda/reduce_impl_.cuh:9-78);
//   3. the last block of a job to finish sums the job's partials in tile order (FP64,
//      deterministic: the result of a job does not depend on what else is in the
//      batch), adds the pose prior, solves (H + damping) dx = -b by FP64 LDL^T, applies
//      X <- expmap(dx) X, v += dx_v, runs the termination test and refreshes the
//      float caches for the next launch.  No host round trip inside compute().
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "kds_align.cuh"
#include "kds_internal.cuh"

namespace kds {

// Every float operation of the per-leaf path -- gates, errors and Jacobians -- rounds
// once, in the operation order of the CPU oracle (itself the reference's order,
// kd/d3/icp_.h:40-60, kd/d3/cticp_impl_.h:10-73, kd/utils/geometry_3d_impl_.h:143-174):
// 3-term sums as x0 + (x1 + x2), as Eigen reduces a fixed-size-3 dot product.  So the
// per-leaf terms, and with the fixed summation order below H and b, are bit-identical
// to the oracle's.
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
  return f3(fs(fm(a.y, b.z), fm(a.z, b.y)), fs(fm(a.z, b.x), fm(a.x, b.z)), fs(fm(a.x, b.y), fm(a.y, b.x)));
}

// C = A * B (3x3 row-major), each coefficient a dot3x of a row and a column
__device__ __forceinline__ void mm3(const float* A, const float* B, float* C) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      C[i * 3 + j] = fa(fm(A[i * 3], B[j]), fa(fm(A[i * 3 + 1], B[3 + j]), fm(A[i * 3 + 2], B[6 + j])));
}
__device__ __forceinline__ F3 mv3(const float* A, F3 p) { return mat_vec_x(A, p); }
// column c of a row-major 3x3
__device__ __forceinline__ F3 col3(const float* A, int c) { return f3(A[c], A[3 + c], A[6 + c]); }

// Pieces of dRxp (kd/utils/geometry_3d_impl_.h:143-174) shared by both of its calls:
// R = rodrigues(w) and Q = n n^T + (R^T - I) S / angle, so that
// d(R u)/dw = -R skew(u) Q.  small = angle < 1e-9 (then dR = -skew(u)).
struct DRxp {
  float R[9];
  float Q[9];
  bool small;
};
__device__ __forceinline__ void drxp_setup(F3 w, DRxp& d) {
  float angle = __fsqrt_rn(dot3x(w, w));
  d.small = angle < 1e-9f;
  if (d.small) {
#pragma unroll
    for (int i = 0; i < 9; ++i) { d.R[i] = (i % 4 == 0) ? 1.f : 0.f; d.Q[i] = 0.f; }
    return;
  }
  rodrigues_x(w, d.R);
  float inv = __fdiv_rn(1.0f, angle);
  F3 n = f3(fm(w.x, inv), fm(w.y, inv), fm(w.z, inv));
  float S[9] = {0.f, -n.z, n.y, n.z, 0.f, -n.x, -n.y, n.x, 0.f};
  float RtmI[9] = {fs(d.R[0], 1.f), d.R[3], d.R[6], d.R[1], fs(d.R[4], 1.f), d.R[7], d.R[2], d.R[5], fs(d.R[8], 1.f)};
  float A[9];
  mm3(RtmI, S, A);
  float nn[3] = {n.x, n.y, n.z};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) d.Q[i * 3 + j] = fa(fm(nn[i], nn[j]), fm(A[i * 3 + j], inv));
}
// out = Ra * d(R u)/dw  (3x3)
__device__ __forceinline__ void ra_drxp(const DRxp& d, const float* Ra, F3 u, float* out) {
  float su[9] = {0.f, -u.z, u.y, u.z, 0.f, -u.x, -u.y, u.x, 0.f};
  float dR[9];
  if (d.small) {
#pragma unroll
    for (int i = 0; i < 9; ++i) dR[i] = -su[i];
  } else {
    float Rs[9], P[9];
    mm3(d.R, su, Rs);
    mm3(Rs, d.Q, P);
#pragma unroll
    for (int i = 0; i < 9; ++i) dR[i] = -P[i];
  }
  mm3(Ra, dR, out);
}

// errorAndJacobianVelocityA (kd/d3/cticp_impl_.h:10-39) -> J[0..5]
__device__ __forceinline__ void jac_vel_A(const float* Xm, F3 pa_l, F3 na_l, F3 pb_g, F3 nb_g, const float* va, float dt,
                                          float* J) {
  F3 tm = f3(fm(va[0], dt), fm(va[1], dt), fm(va[2], dt));
  F3 wa = f3(fm(va[3], dt), fm(va[4], dt), fm(va[5], dt));
  DRxp d;
  drxp_setup(wa, d);
  float Ra[9] = {Xm[0], Xm[1], Xm[2], Xm[4], Xm[5], Xm[6], Xm[8], Xm[9], Xm[10]};
  F3 pam = add3x(mv3(d.R, pa_l), tm);
  F3 nam = mv3(d.R, na_l);
  F3 pag = add3x(mv3(Ra, pam), f3(Xm[3], Xm[7], Xm[11]));
  F3 nag = mv3(Ra, nam);
  F3 n = add3x(nag, nb_g);
  F3 dp = sub3x(pag, pb_g);
  float A[9], B[9];
  ra_drxp(d, Ra, pa_l, A);
  ra_drxp(d, Ra, na_l, B);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    J[c] = fm(dot3x(n, col3(Ra, c)), dt);
    J[3 + c] = fm(fa(dot3x(n, col3(A, c)), dot3x(dp, col3(B, c))), dt);
  }
}

// errorAndJacobianVelocityB (kd/d3/cticp_impl_.h:43-73) -> J[0..5]
__device__ __forceinline__ void jac_vel_B(const float* Xf, F3 pa_g, F3 na_g, F3 pb_l, F3 nb_l, const float* vb, float dt,
                                          float* J) {
  F3 tm = f3(fm(vb[0], dt), fm(vb[1], dt), fm(vb[2], dt));
  F3 wb = f3(fm(vb[3], dt), fm(vb[4], dt), fm(vb[5], dt));
  DRxp d;
  drxp_setup(wb, d);
  float Rb[9] = {Xf[0], Xf[1], Xf[2], Xf[4], Xf[5], Xf[6], Xf[8], Xf[9], Xf[10]};
  F3 pbm = add3x(mv3(d.R, pb_l), tm);
  F3 nbm = mv3(d.R, nb_l);
  F3 pbg = add3x(mv3(Rb, pbm), f3(Xf[3], Xf[7], Xf[11]));
  F3 nbg = mv3(Rb, nbm);
  F3 n = add3x(na_g, nbg);
  F3 nn = f3(-n.x, -n.y, -n.z);
  F3 dp = sub3x(pa_g, pbg);
  float A[9], B[9];
  ra_drxp(d, Rb, pb_l, A);
  ra_drxp(d, Rb, nb_l, B);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    J[c] = fm(dot3x(nn, col3(Rb, c)), dt);
    J[3 + c] = fm(fa(dot3x(nn, col3(A, c)), dot3x(dp, col3(B, c))), dt);
  }
}

enum { ST_INLIER = 0, ST_OUTLIER = 1, ST_BAD = 2, ST_ERR_NORMAL = 3, ST_ERR_FN = 4, ST_NONE = 5 };

template <int KIND> struct KindDim;
template <> struct KindDim<0> { static constexpr int D = 6; };
template <> struct KindDim<1> { static constexpr int D = 12; };
template <> struct KindDim<2> { static constexpr int D = 18; };

// The query of one moving leaf: optional CT warp (applyVelocities) and the moving-to-
// fixed transform Xmf.
template <int KIND>
__device__ __forceinline__ void leaf_query(const CacheF& C, float4 md, float4 nr, F3& m, F3& n, F3& mw, F3& nw,
                                           F3& q) {
  m = f3(md.x, md.y, md.z);
  n = f3(nr.x, nr.y, nr.z);
  mw = m;
  nw = n;
  if (KIND != 0) warp_x(C.v, md.w, m, n, mw, nw);
  q = apply_iso_x(C.Xmf, mw);
}

// Greedy descent (kd/icp/icp_impl_.h:116-121): no backtracking.  idx = the leaf reached,
// or -1 where the descent steps into a pruned child; nd = its record.
__device__ __forceinline__ void descend(const DNode* F, int fnn, const DNode* staged, int nstaged, F3 q, int& idx,
                                        DNode& nd) {
  idx = fnn > 0 ? 0 : -1;
  while (idx >= 0) {
    nd = (idx < nstaged) ? staged[idx] : load_node(F + idx);
    int l = node_left(nd), r = node_right(nd);
    if (l < 0 && r < 0) break;
    bool side = dot3x(node_dir(nd), sub3x(q, node_mean(nd))) > 0.0f;
    idx = side ? l : r;
  }
}

// Two descents through the same tree in lockstep: both chains' node loads are issued
// before either is used, so a thread keeps two dependent load chains in flight.  Each
// chain takes exactly the steps of descend().
__device__ __forceinline__ void descend2(const DNode* F, int fnn, const DNode* staged, int nstaged, bool va, F3 qa,
                                         int& ia, DNode& na, bool vb, F3 qb, int& ib, DNode& nb) {
  ia = (va && fnn > 0) ? 0 : -1;
  ib = (vb && fnn > 0) ? 0 : -1;
  bool ra = ia >= 0, rb = ib >= 0;  // still descending
  while (ra || rb) {
    if (ra) na = (ia < nstaged) ? staged[ia] : load_node(F + ia);
    if (rb) nb = (ib < nstaged) ? staged[ib] : load_node(F + ib);
    if (ra) {
      const int l = node_left(na), r = node_right(na);
      if (l < 0 && r < 0) {
        ra = false;
      } else {
        ia = dot3x(node_dir(na), sub3x(qa, node_mean(na))) > 0.0f ? l : r;
        ra = ia >= 0;
      }
    }
    if (rb) {
      const int l = node_left(nb), r = node_right(nb);
      if (l < 0 && r < 0) {
        rb = false;
      } else {
        ib = dot3x(node_dir(nb), sub3x(qb, node_mean(nb))) > 0.0f ? l : r;
        rb = ib >= 0;
      }
    }
  }
}

// Gates, error, Jacobian and robust weight of one leaf whose descent ended at idx / nd.
template <int KIND>
__device__ __forceinline__ void leaf_math(const CacheF& C, F3 m, F3 n, float dt, F3 mw, F3 nw, int idx,
                                          const DNode& nd, const float* fdts, const ParamsF& P, bool stats_mode,
                                          int& status, int& match, float& e_out, float& gamma_out, float* J) {
  constexpr int D = KindDim<KIND>::D;
#pragma unroll
  for (int i = 0; i < D; ++i) J[i] = 0.f;
  e_out = 0.f;
  gamma_out = 0.f;
  match = idx;
  if (idx < 0) { status = ST_BAD; return; }
  F3 pf = node_mean(nd), nf = node_dir(nd);
  F3 pm = apply_iso_x(C.Xm, mw);
  F3 nm = apply_rot_x(C.Xm, nw);
  F3 pfx = apply_iso_x(C.Xf, pf);
  F3 nfx = apply_rot_x(C.Xf, nf);
  // ICP_3D_Traits::errorAndJacobian (kd/d3/icp_.h:40-60)
  if (dot3x(nfx, nm) < P.min_normal_cos) { status = ST_ERR_NORMAL; return; }
  F3 ns = add3x(nm, nfx);
  float e = dot3x(sub3x(pm, pfx), ns);
  if (fabsf(e) > P.max_error) { status = ST_ERR_FN; return; }
  F3 c1 = cross3(pm, nfx), c2 = cross3(pfx, nm);
  J[0] = ns.x; J[1] = ns.y; J[2] = ns.z;
  J[3] = fa(c1.x, c2.x); J[4] = fa(c1.y, c2.y); J[5] = fa(c1.z, c2.z);
  if (KIND != 0) jac_vel_A(C.Xm, m, n, pfx, nfx, C.v, dt, J + 6);
  float chi2 = fm(e, e);
  float kt = P.kernel_threshold;
  float gamma;
  if (KIND == 2) {
    gamma = stats_mode ? 0.f : 1.f;
    if (chi2 > kt) { status = ST_OUTLIER; gamma = __fsqrt_rn(__fdiv_rn(kt, chi2)); }
    else status = ST_INLIER;
    jac_vel_B(C.Xf, pm, nm, pf, nf, C.fv, fdts[idx], J + 12);
  } else {
    gamma = 1.f;
    if (chi2 > kt) { status = ST_OUTLIER; gamma = stats_mode ? 0.f : __fsqrt_rn(__fdiv_rn(kt, chi2)); }
    else status = ST_INLIER;
  }
  e_out = e;
  gamma_out = gamma;
}

template <int KIND>
__device__ __forceinline__ void leaf_term(const CacheF& C, const DNode* F, int fnn, const float* fdts,
                                          const DNode* staged, int nstaged, float4 md,
                                          float4 nr, const ParamsF& P, bool stats_mode, int& status, int& match,
                                          float& e_out, float& gamma_out, float* J) {
  F3 m, n, mw, nw, q;
  leaf_query<KIND>(C, md, nr, m, n, mw, nw, q);
  int idx;
  DNode nd;
  descend(F, fnn, staged, nstaged, q, idx, nd);
  leaf_math<KIND>(C, m, n, md.w, mw, nw, idx, nd, fdts, P, stats_mode, status, match, e_out, gamma_out, J);
}

// entry k of the packed D(D+1)/2 + D vector -> (row, col); col == D means "e"
__device__ __forceinline__ void entry_rc(int D, int k, int& r, int& c) {
  int T = D * (D + 1) / 2;
  if (k >= T) { r = k - T; c = D; return; }
  int rr = 0, off = 0;
  while (off + (D - rr) <= k) { off += D - rr; ++rr; }
  r = rr;
  c = rr + (k - off);
}

constexpr int kBlock = 128;
constexpr int kWarps = kBlock / 32;
constexpr int kMaxFS = 21;  // factor row stride (D + 2, padded to odd)

// One warp's share of a tile partial from its 32 leaves' terms (leaf = lane): stats by
// ballots, chi2 sums by xor butterfly, and gamma J^T J, gamma J^T e as float Kahan sums
// over the lanes (lane k owns packed entries k, k + 32, ...) stored as s - comp in FP64.
template <int KIND>
__device__ __forceinline__ void tile_reduce(int status, float e, float gamma, const float* J, double* wpart,
                                            float* fac) {
  constexpr int D = KindDim<KIND>::D;
  constexpr int M = D * (D + 1) / 2 + D;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  bool contrib = status == ST_INLIER || status == ST_OUTLIER;
  float* row = fac + (w * 32 + lane) * kMaxFS;
#pragma unroll
  for (int k = 0; k < D; ++k) row[k] = contrib ? J[k] : 0.f;
  row[D] = contrib ? e : 0.f;
  row[D + 1] = contrib ? gamma : 0.f;
  // stats (ICPStats_::pack, kd/icp/icp_stats_.h:57-59)
  unsigned full = 0xffffffffu;
  int c_in = __popc(__ballot_sync(full, status == ST_INLIER));
  int c_out = __popc(__ballot_sync(full, status == ST_OUTLIER));
  int c_bad = __popc(__ballot_sync(full, status == ST_BAD));
  int c_nrm = __popc(__ballot_sync(full, status == ST_ERR_NORMAL));
  int c_fn = __popc(__ballot_sync(full, status == ST_ERR_FN));
  double chi2 = contrib ? (double)fm(e, e) : 0.0;
  double chi2k = contrib ? (double)fm(fm(e, e), gamma) : 0.0;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    chi2 += __shfl_xor_sync(full, chi2, off);
    chi2k += __shfl_xor_sync(full, chi2k, off);
  }
  __syncwarp();
  // warp-cooperative outer products: lane owns entries lane, lane+32, ...
  const float* wf = fac + w * 32 * kMaxFS;
  double* wp = wpart + w * kPStride;
  for (int k = lane; k < M; k += 32) {
    int r, c;
    entry_rc(D, k, r, c);
    float s = 0.f, comp = 0.f;
#pragma unroll 8
    for (int l = 0; l < 32; ++l) {
      const float* fr = wf + l * kMaxFS;
      float val = fm(fm(fr[r], fr[c]), fr[D + 1]);
      float y = fs(val, comp);
      float t = fa(s, y);
      comp = fs(fs(t, s), y);
      s = t;
    }
    wp[k] = (double)s - (double)comp;
  }
  if (lane == 0) {
    wp[kPStats + 0] = c_in;
    wp[kPStats + 1] = c_out;
    wp[kPStats + 2] = c_bad;
    wp[kPStats + 3] = c_nrm;
    wp[kPStats + 4] = c_fn;
    wp[kPStats + 5] = chi2;
    wp[kPStats + 6] = chi2k;
  }
  __syncwarp();  // the warp's rows may be rewritten after this
}

template <int KIND>
__device__ __forceinline__ void tile_body(const JobIn& Jn, const LinDev& L, const CacheF& C, const TileDev& T,
                                          const DNode* staged, int nstaged,
                                          double* wpart /* [kWarps][kPStride] */, float* fac /* [kWarps][32][kMaxFS] */,
                                          int32_t* dbg_match, int32_t* dbg_status) {
  constexpr int D = KindDim<KIND>::D;
  const int i = T.leaf_begin + threadIdx.x;
  int status = ST_NONE, match = -1;
  float e = 0.f, gamma = 0.f;
  float J[D];
#pragma unroll
  for (int k = 0; k < D; ++k) J[k] = 0.f;
  if (i < T.leaf_end) {
    float4 md = __ldg(Jn.m_md + i);
    float4 nr = __ldg(Jn.m_nrm + i);
    leaf_term<KIND>(C, L.fnodes, L.f_num_nodes, L.fdts, staged, nstaged, md, nr, Jn.P, Jn.stats_mode != 0, status,
                    match, e, gamma, J);
    if (dbg_match) { dbg_match[i] = match; dbg_status[i] = status; }
  }
  tile_reduce<KIND>(status, e, gamma, J, wpart, fac);
}

// Two tiles of one (job, fixed entry) per block: thread t takes leaf t of both, runs the
// two descents in lockstep, then reduces tile A and tile B one after the other with
// tile_body's arithmetic, so each tile's partial is bit-identical to one-tile blocks.
template <int KIND>
__device__ __forceinline__ void tile_body_pair(const JobIn& Jn, const LinDev& L, const CacheF& C, const TileDev& TA,
                                               const TileDev& TB, bool has_b, const DNode* staged, int nstaged,
                                               double* wpa, double* wpb, float* fac, int32_t* dbg_match,
                                               int32_t* dbg_status) {
  constexpr int D = KindDim<KIND>::D;
  const int ia = TA.leaf_begin + threadIdx.x, ib = TB.leaf_begin + threadIdx.x;
  const bool va = ia < TA.leaf_end, vb = has_b && ib < TB.leaf_end;
  F3 ma, na, mwa, nwa, qa, mb, nb, mwb, nwb, qb;
  float dta = 0.f, dtb = 0.f;
  if (va) {
    const float4 md = __ldg(Jn.m_md + ia), nr = __ldg(Jn.m_nrm + ia);
    leaf_query<KIND>(C, md, nr, ma, na, mwa, nwa, qa);
    dta = md.w;
  }
  if (vb) {
    const float4 md = __ldg(Jn.m_md + ib), nr = __ldg(Jn.m_nrm + ib);
    leaf_query<KIND>(C, md, nr, mb, nb, mwb, nwb, qb);
    dtb = md.w;
  }
  int xa, xb;
  DNode nda, ndb;
  descend2(L.fnodes, L.f_num_nodes, staged, nstaged, va, qa, xa, nda, vb, qb, xb, ndb);
  {
    int status = ST_NONE, match = -1;
    float e = 0.f, gamma = 0.f, J[D];
#pragma unroll
    for (int k = 0; k < D; ++k) J[k] = 0.f;
    if (va) {
      leaf_math<KIND>(C, ma, na, dta, mwa, nwa, xa, nda, L.fdts, Jn.P, Jn.stats_mode != 0, status, match, e, gamma, J);
      if (dbg_match) { dbg_match[ia] = match; dbg_status[ia] = status; }
    }
    tile_reduce<KIND>(status, e, gamma, J, wpa, fac);
  }
  {
    int status = ST_NONE, match = -1;
    float e = 0.f, gamma = 0.f, J[D];
#pragma unroll
    for (int k = 0; k < D; ++k) J[k] = 0.f;
    if (vb) {
      leaf_math<KIND>(C, mb, nb, dtb, mwb, nwb, xb, ndb, L.fdts, Jn.P, Jn.stats_mode != 0, status, match, e, gamma, J);
      if (dbg_match) { dbg_match[ib] = match; dbg_status[ib] = status; }
    }
    tile_reduce<KIND>(status, e, gamma, J, wpb, fac);
  }
}

// ---------------------------------------------------------------------------
// FP64 finalize (one thread) -- ICP_::oneRound / CTICP_::oneRound.
// Pose algebra in FP64 with one rounding per operation and 3-term sums as
// x0 + (x1 + x2), the CPU oracle's order for Eigen's Transform product and inverse.
__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddot3(double a0, double a1, double a2, double b0, double b1, double b2) {
  return da(dm(a0, b0), da(dm(a1, b1), dm(a2, b2)));
}
__device__ void iso_mul_d(const double* A, const double* B, double* C) {
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) C[i * 4 + j] = ddot3(A[i * 4], A[i * 4 + 1], A[i * 4 + 2], B[j], B[4 + j], B[8 + j]);
    C[i * 4 + 3] = da(ddot3(A[i * 4], A[i * 4 + 1], A[i * 4 + 2], B[3], B[7], B[11]), A[i * 4 + 3]);
  }
}
__device__ void iso_inv_d(const double* A, double* B) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) B[i * 4 + j] = A[j * 4 + i];
  for (int i = 0; i < 3; ++i) B[i * 4 + 3] = -ddot3(A[i], A[4 + i], A[8 + i], A[3], A[7], A[11]);
}

// Canonical FP64 sine/cosine (this project's own, shared with the CPU oracle so that the
// pose update is bit-identical there): Cody-Waite reduction by pi/2 with a three-part
// constant (Cody & Waite 1980; parts of 33, 33 and 53 bits, so q * C1 and q * C2 are
// exact for |q| < 2^20), then the Taylor series of sin to r^17 and of cos to r^18 on
// [-pi/4, pi/4] in Horner form (truncation below 1e-19).
__device__ void sincos_canon_d(double x, double* s_out, double* c_out) {
  const double q = rint(dm(x, 0x1.45f306dc9c883p-1));
  const long long j = (long long)q;
  double r = ds(x, dm(q, 0x1.921fb54400000p+0));
  r = ds(r, dm(q, 0x1.0b4611a600000p-34));
  r = ds(r, dm(q, 0x1.3198a2e037073p-69));
  const double r2 = dm(r, r);
  double t = 0x1.952c77030ad4ap-49;             // 1/17!
  t = da(-0x1.ae7f3e733b81fp-41, dm(r2, t));    // 1/15!
  t = da(0x1.6124613a86d09p-33, dm(r2, t));     // 1/13!
  t = da(-0x1.ae64567f544e4p-26, dm(r2, t));    // 1/11!
  t = da(0x1.71de3a556c734p-19, dm(r2, t));     // 1/9!
  t = da(-0x1.a01a01a01a01ap-13, dm(r2, t));    // 1/7!
  t = da(0x1.1111111111111p-7, dm(r2, t));      // 1/5!
  t = da(-0x1.5555555555555p-3, dm(r2, t));     // 1/3!
  const double sn = da(r, dm(r, dm(r2, t)));
  double u = -0x1.6827863b97d97p-53;            // 1/18!
  u = da(0x1.ae7f3e733b81fp-45, dm(r2, u));     // 1/16!
  u = da(-0x1.93974a8c07c9dp-37, dm(r2, u));    // 1/14!
  u = da(0x1.1eed8eff8d898p-29, dm(r2, u));     // 1/12!
  u = da(-0x1.27e4fb7789f5cp-22, dm(r2, u));    // 1/10!
  u = da(0x1.a01a01a01a01ap-16, dm(r2, u));     // 1/8!
  u = da(-0x1.6c16c16c16c17p-10, dm(r2, u));    // 1/6!
  u = da(0x1.5555555555555p-5, dm(r2, u));      // 1/4!
  u = da(-0.5, dm(r2, u));
  const double cs = da(1.0, dm(r2, u));
  switch ((int)(j & 3)) {
    case 0: *s_out = sn; *c_out = cs; break;
    case 1: *s_out = cs; *c_out = -sn; break;
    case 2: *s_out = -sn; *c_out = -cs; break;
    default: *s_out = -cs; *c_out = sn; break;
  }
}

// rodrigues (kd/utils/geometry_3d_impl_.h:37-46) in FP64: I + sin(a) S + (1 - cos(a)) S^2
__device__ void rodrigues_d(const double* w, double* R) {
  const double a = sqrt(ddot3(w[0], w[1], w[2], w[0], w[1], w[2]));
  if (a < 1e-9) {
    for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1.0 : 0.0;
    return;
  }
  const double inv = 1.0 / a;
  const double n[3] = {dm(w[0], inv), dm(w[1], inv), dm(w[2], inv)};
  const double S[9] = {0, -n[2], n[1], n[2], 0, -n[0], -n[1], n[0], 0};
  double s, c;
  sincos_canon_d(a, &s, &c);
  const double omc = ds(1.0, c);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const double s2 = ddot3(S[i * 3], S[i * 3 + 1], S[i * 3 + 2], S[j], S[3 + j], S[6 + j]);
      R[i * 3 + j] = da(da((i == j) ? 1.0 : 0.0, dm(s, S[i * 3 + j])), dm(omc, s2));
    }
}
__device__ void expmap_d(const double* v, double* X) {
  double R[9];
  rodrigues_d(v + 3, R);
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) X[i * 4 + j] = R[i * 3 + j];
    X[i * 4 + 3] = v[i];
  }
}
__device__ void logso3_d(const double* X, double* w) {
  double tr = X[0] + X[5] + X[10];
  double ca = fmin(1.0, fmax(-1.0, 0.5 * (tr - 1.0)));
  double a = acos(ca);
  double ax[3] = {X[9] - X[6], X[2] - X[8], X[4] - X[1]};
  double f = (a < 1e-7) ? 0.5 : a / (2.0 * sin(a));
  for (int i = 0; i < 3; ++i) w[i] = ax[i] * f;
}
// dPoseToPoseError (kd/utils/geometry_3d_impl_.h:125-140) in FP64
__device__ void dpose_d(const double* ZXi, const double* Xm, double* e, double J[6][6]) {
  double P[12];
  iso_mul_d(ZXi, Xm, P);
  for (int i = 0; i < 3; ++i) e[i] = P[i * 4 + 3];
  logso3_d(P, e + 3);
  double R[9] = {ZXi[0], ZXi[1], ZXi[2], ZXi[4], ZXi[5], ZXi[6], ZXi[8], ZXi[9], ZXi[10]};
  double B[12][6];
  for (int i = 0; i < 12; ++i) for (int j = 0; j < 6; ++j) B[i][j] = 0.0;
  auto skewmul = [&](const double* v, double* out) {  // out = R * skew(v)
    double S[9] = {0, -v[2], v[1], v[2], 0, -v[0], -v[1], v[0], 0};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) out[i * 3 + j] = R[i * 3] * S[j] + R[i * 3 + 1] * S[3 + j] + R[i * 3 + 2] * S[6 + j];
  };
  double t[3] = {Xm[3], Xm[7], Xm[11]};
  double RS[9];
  skewmul(t, RS);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) { B[i][j] = R[i * 3 + j]; B[i][3 + j] = -RS[i * 3 + j]; }
  for (int k = 0; k < 3; ++k) {
    double col[3] = {Xm[k], Xm[4 + k], Xm[8 + k]};
    skewmul(col, RS);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) B[3 + 3 * k + i][3 + j] = -RS[i * 3 + j];
  }
  // dlogSO3 of P's rotation (column-major coefficient order)
  double ax[3] = {P[9] - P[6], P[2] - P[8], P[4] - P[1]};
  double tr = P[0] + P[5] + P[10];
  double ca = fmin(1.0, fmax(-1.0, 0.5 * (tr - 1.0)));
  double a = acos(ca);
  bool small = a < 1e-7;
  double f = small ? 0.5 : a / (2.0 * sin(a));
  double Js[3][9];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 9; ++j) Js[i][j] = 0.0;
  Js[0][5] = f; Js[0][7] = -f;
  Js[1][6] = f; Js[1][2] = -f;
  Js[2][1] = f; Js[2][3] = -f;
  if (!small) {
    double s = sin(a);
    double c = (s - a * cos(a)) / (4.0 * s * s * s);
    for (int k = 0; k < 3; ++k) { Js[k][0] -= c * ax[k]; Js[k][4] -= c * ax[k]; Js[k][8] -= c * ax[k]; }
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      double acc = 0.0;
      if (i < 3) acc = B[i][j];
      else for (int k = 0; k < 9; ++k) acc += Js[i - 3][k] * B[3 + k][j];
      J[i][j] = acc;
    }
}

__device__ void refresh_caches(const JobState& S, LinDev* lins, int lb, int lc) {
  for (int l = lb; l < lb + lc; ++l) {
    LinDev& L = lins[l];
    double iXf[12], Xmf[12];
    iso_inv_d(L.Xf, iXf);
    iso_mul_d(iXf, S.X, Xmf);
    for (int k = 0; k < 12; ++k) {
      L.cache.Xm[k] = (float)S.X[k];
      L.cache.Xf[k] = (float)L.Xf[k];
      L.cache.Xmf[k] = (float)Xmf[k];
    }
    for (int k = 0; k < 6; ++k) {
      L.cache.v[k] = (float)S.v[k];
      L.cache.fv[k] = (float)L.fv[k];
    }
  }
}

// Pose prior (posePriorBuildQuadraticForm, kd/icp/tree_aligner_base_.h:139-152): adds
// J^T Omega J and J^T Omega e to the pose block.  Single thread, used by the localizer.
__device__ __noinline__ void add_pose_prior(const JobIn& Jn, const double* X, double* H, double* b, int D) {
  double e6[6], Jp[6][6];
  dpose_d(Jn.prior_ZXi, X, e6, Jp);
  const double* Om = Jn.prior_info;
  double OJ[6][6], Oe[6];
  for (int i = 0; i < 6; ++i) {
    for (int j = 0; j < 6; ++j) {
      double a = 0;
      for (int k = 0; k < 6; ++k) a += Om[i * 6 + k] * Jp[k][j];
      OJ[i][j] = a;
    }
    double a = 0;
    for (int k = 0; k < 6; ++k) a += Om[i * 6 + k] * e6[k];
    Oe[i] = a;
  }
  for (int i = 0; i < 6; ++i) {
    for (int j = 0; j < 6; ++j) {
      double a = 0;
      for (int k = 0; k < 6; ++k) a += Jp[k][i] * OJ[k][j];
      H[i * D + j] += a;
    }
    double a = 0;
    for (int k = 0; k < 6; ++k) a += Jp[k][i] * Oe[k];
    b[i] += a;
  }
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// ---------------------------------------------------------------------------
// The last block of a job: FP64 sum of the job's partials in tile order, then warp 0
// runs ICP_::oneRound / CTICP_::oneRound (kd/icp/icp_impl_.h:72-89,
// kd/cticp/cticp_impl_.h:67-91) with the D x D system in shared memory: Cholesky of
// H + damping (SPD), warp-parallel trailing updates and triangular solves.
__device__ void tail_warp(const JobIn& Jn, JobState& S, JobOut& O, kds_stats* log, LinDev* lins, double* red, int M);

// Phase stamps (clock64) of the last launch, recorded only when profiling is on:
// [0..3] block 0: entry, staged, tile done, partial published; [8..15] tail block:
// entry, partials summed, state staged, solve start, factorized, solved, updated, done.
__device__ int g_phase_on;
__device__ unsigned long long g_phase[16];
// Error bits of a k_linearize launch whose caller passed no error slot of its own (the
// served loop): 1 = a bounded wait for the tree-top copy gave up and the block read the
// tree from global memory (results valid); 2 = the copy was still not seen complete when
// the block was about to exit (the CUDA context is suspect).
__device__ int g_kernel_error;
// Polls of the first bounded wait for the tree-top copy (kds_set_tma_wait_limit).  The
// wait a block makes before it exits always allows 2^20 polls.
__device__ int g_wait_spins = 1 << 20;

// Bounded wait for the phase with the given parity of an mbarrier to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, int spins = 1 << 20) {
  for (int i = 0; i < spins; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

constexpr int kTailJobOff = 560;    // doubles into the tail's shared scratch
constexpr int kTailStateOff = 680;
static_assert(kTailJobOff + sizeof(JobIn) / 8 + 1 <= kTailStateOff, "tail scratch layout");
static_assert(kTailStateOff + sizeof(JobState) / 8 + 1 <= 4 * kPStride, "tail scratch layout");

__device__ __noinline__ void job_tail(const JobIn& JnG, JobState& SG, JobOut& O, kds_stats* log, LinDev* lins,
                                      const double* partials, double* red, int M) {
  const bool stamp = g_phase_on && threadIdx.x == 0;
  if (stamp) g_phase[8] = clock64();
  for (int k = threadIdx.x; k < kPStride; k += blockDim.x) {
    if (k >= M && k < kPStats) { red[k] = 0.0; continue; }
    double acc = 0.0;
    const double* src = partials + (size_t)JnG.tile_begin * kPStride + k;
    const int nt = JnG.tile_count;
    double a4[4] = {0.0, 0.0, 0.0, 0.0};
    int t = 0;
    for (; t + 4 <= nt; t += 4) {
#pragma unroll
      for (int u = 0; u < 4; ++u) a4[u] += __ldcg(src + (size_t)(t + u) * kPStride);
    }
    for (; t < nt; ++t) a4[0] += __ldcg(src + (size_t)t * kPStride);
    acc = (a4[0] + a4[1]) + (a4[2] + a4[3]);
    red[k] = acc;
  }
  __syncthreads();
  if (stamp) g_phase[9] = clock64();
  if (threadIdx.x >= 32) return;
  // the job's inputs and state move to shared memory in one parallel round trip
  JobIn* sJn = reinterpret_cast<JobIn*>(red + kTailJobOff);
  JobState* sS = reinterpret_cast<JobState*>(red + kTailStateOff);
  {
    typedef unsigned long long u64;
    constexpr int NJ = sizeof(JobIn) / 8, NS = sizeof(JobState) / 8;
    static_assert(sizeof(JobIn) % 8 == 0 && sizeof(JobState) % 8 == 0 && NJ <= 96 && NS <= 32, "staging");
    const u64* a = reinterpret_cast<const u64*>(&JnG);
    const u64* c = reinterpret_cast<const u64*>(&SG);
    const int l = threadIdx.x;
    u64 r0 = 0, r1 = 0, r2 = 0, r3 = 0;  // all loads issued before any store
    if (l < NJ) r0 = a[l];
    if (l + 32 < NJ) r1 = a[l + 32];
    if (l + 64 < NJ) r2 = a[l + 64];
    if (l < NS) r3 = c[l];
    u64* b = reinterpret_cast<u64*>(sJn);
    u64* d = reinterpret_cast<u64*>(sS);
    if (l < NJ) b[l] = r0;
    if (l + 32 < NJ) b[l + 32] = r1;
    if (l + 64 < NJ) b[l + 64] = r2;
    if (l < NS) d[l] = r3;
  }
  __syncwarp();
  if (stamp) g_phase[10] = clock64();
  tail_warp(*sJn, *sS, O, log, lins, red, M);
  __syncwarp();
  {
    const unsigned long long* c = reinterpret_cast<const unsigned long long*>(sS);
    unsigned long long* d = reinterpret_cast<unsigned long long*>(&SG);
    if (threadIdx.x < (int)(sizeof(JobState) / 8)) d[threadIdx.x] = c[threadIdx.x];
  }
  if (stamp) g_phase[15] = clock64();
}

// Warp 0 of the last block: unpack, prior, solve, update, termination test.
__device__ void tail_warp(const JobIn& Jn, JobState& S, JobOut& O, kds_stats* log, LinDev* lins, double* red, int M) {
  const int lane = threadIdx.x;
  const int kind = Jn.kind;
  const int Dk = kind == 0 ? 6 : (kind == 1 ? 12 : 18);
  const int D = kind == 0 ? 6 : 12;
  double* sH = red + kPStride;  // D*D
  double* sA = sH + 144;        // D*D
  double* sb = sA + 144;        // D
  double* sy = sb + 12;         // D
  double* sx = sy + 12;         // D
  // unpack the packed upper triangle
  for (int k = lane; k < M; k += 32) {
    int r, c;
    entry_rc(Dk, k, r, c);
    double v = red[k];
    if (c == Dk) {
      if (r < D) sb[r] = v;
      else O.b_vel_B[r - 12] = v;
    } else if (c < D) {
      sH[r * D + c] = v;
      sH[c * D + r] = v;
    } else {  // dual blocks, c >= 12
      if (r < 6) O.H_cross_pose_vel_B[r * 6 + (c - 12)] = v;
      else if (r < 12) O.H_cross_vel_AB[(r - 6) * 6 + (c - 12)] = v;
      else { O.H_vel_B[(r - 12) * 6 + (c - 12)] = v; O.H_vel_B[(c - 12) * 6 + (r - 12)] = v; }
    }
  }
  kds_stats st;
  st.num_inliers = (int32_t)red[kPStats + 0];
  st.num_outliers = (int32_t)red[kPStats + 1];
  st.num_bad = (int32_t)red[kPStats + 2];
  st.num_err_normal = (int32_t)red[kPStats + 3];
  st.num_err_fn = (int32_t)red[kPStats + 4];
  st.chi2 = (float)red[kPStats + 5];
  st.chi2_kernelized = (float)red[kPStats + 6];
  st.pert_pose_norm = 0.f;
  st.pert_vel_norm = 0.f;
  const int it = S.iter;
  __syncwarp();
  if (Jn.mode != KDS_JOB_COMPUTE) {
    for (int i = lane; i < D * D; i += 32) O.H[i] = sH[i];
    if (lane < D) O.b[lane] = sb[lane];
    if (lane == 0) {
      O.stats = st;
      O.result = 0;
      O.iterations = 1;
      S.done = 1;
      S.arrive = 0u;
    }
    return;
  }
  if (Jn.prior_enabled && lane == 0) add_pose_prior(Jn, S.X, sH, sb, D);
  __syncwarp();
  for (int i = lane; i < D * D; i += 32) {
    O.H[i] = sH[i];
    sA[i] = sH[i];
  }
  if (lane < D) {
    O.b[lane] = sb[lane];
    sA[lane * D + lane] += (lane < 6) ? (double)Jn.P.damping : (double)Jn.P.velocity_damping;
  }
  if (st.num_inliers + st.num_outliers < Jn.P.min_good_measurements) {
    if (lane == 0) {
      if (log && it < kMaxLog) log[it] = st;
      O.stats = st;
      O.iterations = it + 1;
      S.done = 1;
      S.result = -it;
      O.result = S.result;
      S.arrive = 0u;
    }
    return;
  }
  __syncwarp();
  if (g_phase_on && lane == 0) g_phase[11] = clock64();
  // Cholesky of the lower triangle of sA: per pivot one square root and reciprocal,
  // the column scaled by the lanes, the trailing update spread over all lanes.
  double* sinv = sx + 12;  // reciprocals of diag(L)
  bool ok = true;
  for (int k = 0; k < D; ++k) {
    double d = sA[k * D + k];
    ok = ok && (d > 0.0);
    double lkk = sqrt(fmax(d, 1e-300));
    double inv = 1.0 / lkk;
    __syncwarp();
    if (lane > k && lane < D) sA[lane * D + k] *= inv;
    if (lane == k) {
      sA[k * D + k] = lkk;
      sinv[k] = inv;
    }
    __syncwarp();
    // pairs (i, j), k < j <= i < D, enumerated row-major over the trailing triangle
    const int m = D - k - 1;
    const int npair = m * (m + 1) / 2;
    for (int p = lane; p < npair; p += 32) {
      int ii = 0;
      while ((ii + 1) * (ii + 2) / 2 <= p) ++ii;
      const int i = k + 1 + ii, j = k + 1 + (p - ii * (ii + 1) / 2);
      sA[i * D + j] -= sA[i * D + k] * sA[j * D + k];
    }
    __syncwarp();
  }
  if (g_phase_on && lane == 0) g_phase[12] = clock64();
  // L y = -b and L^T x = y by column sweeps
  if (lane < D) sy[lane] = -sb[lane];
  __syncwarp();
  for (int k = 0; k < D; ++k) {
    const double yk = sy[k] * sinv[k];
    __syncwarp();
    if (lane == k) sy[k] = yk;
    if (lane > k && lane < D) sy[lane] -= sA[lane * D + k] * yk;
    __syncwarp();
  }
  if (lane < D) sx[lane] = sy[lane];
  __syncwarp();
  for (int k = D - 1; k >= 0; --k) {
    const double xk = sx[k] * sinv[k];
    __syncwarp();
    if (lane == k) sx[k] = xk;
    if (lane < k) sx[lane] -= sA[k * D + lane] * xk;
    __syncwarp();
  }
  if (lane != 0) return;
  if (g_phase_on) g_phase[13] = clock64();
  double dx[12];
  for (int i = 0; i < D; ++i) dx[i] = ok ? sx[i] : 0.0;
  double pp = 0.0, pv = 0.0;
  for (int i = 0; i < 6; ++i) pp += dx[i] * dx[i];
  st.pert_pose_norm = (float)sqrt(pp);
  if (D == 12) {
    for (int i = 6; i < 12; ++i) pv += dx[i] * dx[i];
    st.pert_vel_norm = (float)sqrt(pv);
  }
  for (int i = 0; i < D; ++i) O.dx[i] = dx[i];
  if (log && it < kMaxLog) log[it] = st;
  O.stats = st;
  O.iterations = it + 1;
  if (!Jn.stats_mode) {
    double dX[12], Xn[12];
    expmap_d(dx, dX);
    iso_mul_d(dX, S.X, Xn);
    for (int i = 0; i < 12; ++i) S.X[i] = Xn[i];
    if (D == 12)
      for (int i = 0; i < 6; ++i) S.v[i] += dx[6 + i];
  }
  bool stop = false;
  if (Jn.P.term_crit) {
    // ICPTerminationCriteriaScore_::hasToStop (kd/icp/icp_stats_.h:91-101)
    int nl = st.num_inliers + st.num_outliers + st.num_bad + st.num_err_normal + st.num_err_fn;
    float ratio = nl ? (float)st.num_inliers / (float)nl : 0.f;
    float score = ratio / (st.chi2_kernelized / (float)st.num_inliers + 1e-6f);
    if (it > 0) {
      bool pert_ok = st.pert_pose_norm < Jn.P.d_pert;
      float dsc = score - S.prev_score;
      bool score_ok = (dsc > 0.f) && ((double)dsc / ((double)S.prev_score + 1e-6) < (double)Jn.P.d_score);
      if (pert_ok && score_ok) stop = true;
    }
    S.prev_score = score;
  }
  S.iter = it + 1;
  if (stop) {
    S.done = 1;
    S.result = it;
  } else if (S.iter >= S.max_iter) {
    S.done = 1;
    S.result = Jn.P.max_iterations;
  }
  O.result = S.result;
  for (int i = 0; i < 12; ++i) O.X[i] = S.X[i];
  for (int i = 0; i < 6; ++i) O.v[i] = S.v[i];
  if (!S.done) refresh_caches(S, lins, Jn.lin_begin, Jn.lin_count);
  if (g_phase_on) g_phase[14] = clock64();
  S.arrive = 0u;
}

// One Gauss-Newton iteration over the tiles [tile0, tile0 + gridDim.x) of one kind.
__device__ __forceinline__ void report_error(int32_t* err, int bits) { atomicOr(err ? err : &g_kernel_error, bits); }

template <int KIND>
__global__ void __launch_bounds__(kBlock, 4) k_linearize(const JobIn* __restrict__ jobs, JobState* states, JobOut* outs,
                                                      kds_stats* logs, LinDev* lins, const TileDev* __restrict__ tiles,
                                                      int tile0, int stage, double* partials, int32_t* dbg_match,
                                                      int32_t* dbg_status, int32_t* err) {
  constexpr int D = KindDim<KIND>::D;
  constexpr int M = D * (D + 1) / 2 + D;
  __shared__ CacheF sC;
  __shared__ float sfac[kWarps * 32 * kMaxFS];
  __shared__ double swp[kWarps * kPStride];
  __shared__ int s_last;
  __shared__ __align__(8) unsigned long long s_mbar;
  const bool stamp = g_phase_on && blockIdx.x == 0 && threadIdx.x == 0;
  if (stamp) g_phase[0] = clock64();
  const int tile = tile0 + blockIdx.x;
  const TileDev T = tiles[tile];
  JobState& S = states[T.job];
  if (*(volatile int32_t*)&S.done) return;
  const JobIn& Jn = jobs[T.job];
  const LinDev& L = lins[T.lin];
  // Top of the fixed tree: in BFS order the first nodes are the shallowest levels.
  // One thread issues a TMA bulk copy (cp.async.bulk, no multicast) of them into
  // shared memory while the block loads the rest of its inputs.
  extern __shared__ float4 sDyn[];
  const DNode* sN = reinterpret_cast<const DNode*>(sDyn);
  int nst = min(stage, L.f_num_nodes);
  const uint32_t bytes = (uint32_t)nst * (uint32_t)sizeof(DNode);
  const uint32_t mbar = (uint32_t)__cvta_generic_to_shared(&s_mbar);
  if (threadIdx.x == 0 && bytes > 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(sDyn)),
                 "l"(L.fnodes), "r"(bytes), "r"(mbar)
                 : "memory");
  }
  if (threadIdx.x < (int)(sizeof(CacheF) / 4))
    reinterpret_cast<float*>(&sC)[threadIdx.x] = reinterpret_cast<const float*>(&L.cache)[threadIdx.x];
  __syncthreads();
  if (bytes > 0 && !mbar_wait(mbar, 0u, g_wait_spins)) {
    // copy not observed complete: record it and read the whole tree from global memory
    report_error(err, 1);
    nst = 0;
  }
  // Before the block exits, thread 0 waits (bounded) for the copy to land, so that no
  // bulk copy into this block's shared memory outlives the block.
  auto settle = [&]() {
    if (threadIdx.x == 0 && bytes > 0 && !mbar_wait(mbar, 0u)) report_error(err, 2);
  };
  if (stamp) g_phase[1] = clock64();
  tile_body<KIND>(Jn, L, sC, T, sN, nst, swp, sfac, dbg_match, dbg_status);
  __syncthreads();
  if (stamp) g_phase[2] = clock64();
  double* P = partials + (size_t)tile * kPStride;
  for (int k = threadIdx.x; k < kPStride; k += blockDim.x) {
    if (k >= M && k < kPStats) continue;
    double acc = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) acc += swp[w * kPStride + k];
    P[k] = acc;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned prev = atomicAdd(&S.arrive, 1u);
    s_last = (prev == (unsigned)(Jn.tile_count - 1)) ? 1 : 0;
  }
  __syncthreads();
  if (stamp) g_phase[3] = clock64();
  if (!s_last) {
    settle();
    return;
  }
  __threadfence();
  job_tail(Jn, S, outs[T.job], logs ? logs + (size_t)T.job * kMaxLog : nullptr, lins, partials, swp, M);
  settle();
}

// One Gauss-Newton iteration with two tiles per block: the block list pairs consecutive
// tiles of the same (job, fixed entry) (the second index is -1 for a job's odd last
// tile).  Each thread keeps two descents in flight; the partials, the arrival count and
// the job's step are those of k_linearize.
template <int KIND>
__global__ void __launch_bounds__(kBlock, 4) k_linearize_pair(const JobIn* __restrict__ jobs, JobState* states,
                                                           JobOut* outs, kds_stats* logs, LinDev* lins,
                                                           const TileDev* __restrict__ tiles,
                                                           const int2* __restrict__ pairs, int pair0, int stage,
                                                           double* partials, int32_t* dbg_match, int32_t* dbg_status,
                                                           int32_t* err) {
  constexpr int D = KindDim<KIND>::D;
  constexpr int M = D * (D + 1) / 2 + D;
  __shared__ CacheF sC;
  __shared__ float sfac[kWarps * 32 * kMaxFS];
  __shared__ double swp[2][kWarps * kPStride];
  __shared__ int s_last;
  __shared__ __align__(8) unsigned long long s_mbar;
  const int2 pr = pairs[pair0 + blockIdx.x];
  const TileDev TA = tiles[pr.x];
  const bool has_b = pr.y >= 0;
  const TileDev TB = has_b ? tiles[pr.y] : TA;
  JobState& S = states[TA.job];
  if (*(volatile int32_t*)&S.done) return;
  const JobIn& Jn = jobs[TA.job];
  const LinDev& L = lins[TA.lin];
  extern __shared__ float4 sDyn[];
  const DNode* sN = reinterpret_cast<const DNode*>(sDyn);
  int nst = min(stage, L.f_num_nodes);
  const uint32_t bytes = (uint32_t)nst * (uint32_t)sizeof(DNode);
  const uint32_t mbar = (uint32_t)__cvta_generic_to_shared(&s_mbar);
  if (threadIdx.x == 0 && bytes > 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(sDyn)),
                 "l"(L.fnodes), "r"(bytes), "r"(mbar)
                 : "memory");
  }
  if (threadIdx.x < (int)(sizeof(CacheF) / 4))
    reinterpret_cast<float*>(&sC)[threadIdx.x] = reinterpret_cast<const float*>(&L.cache)[threadIdx.x];
  __syncthreads();
  if (bytes > 0 && !mbar_wait(mbar, 0u, g_wait_spins)) {
    report_error(err, 1);  // read the whole tree from global memory
    nst = 0;
  }
  auto settle = [&]() {
    if (threadIdx.x == 0 && bytes > 0 && !mbar_wait(mbar, 0u)) report_error(err, 2);
  };
  tile_body_pair<KIND>(Jn, L, sC, TA, TB, has_b, sN, nst, swp[0], swp[1], sfac, dbg_match, dbg_status);
  __syncthreads();
  for (int h = 0; h < (has_b ? 2 : 1); ++h) {
    double* P = partials + (size_t)(h ? pr.y : pr.x) * kPStride;
    for (int k = threadIdx.x; k < kPStride; k += blockDim.x) {
      if (k >= M && k < kPStats) continue;
      double acc = 0.0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) acc += swp[h][w * kPStride + k];
      P[k] = acc;
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned nt = has_b ? 2u : 1u;
    unsigned prev = atomicAdd(&S.arrive, nt);
    s_last = (prev + nt == (unsigned)Jn.tile_count) ? 1 : 0;
  }
  __syncthreads();
  if (!s_last) {
    settle();
    return;
  }
  __threadfence();
  job_tail(Jn, S, outs[TA.job], logs ? logs + (size_t)TA.job * kMaxLog : nullptr, lins, partials, swp[0], M);
  settle();
}

// ---------------------------------------------------------------------------
// Persistent form of a batch: one launch runs every Gauss-Newton iteration of every job.
// The work items are (iteration, tile) pairs in iteration-major order, handed out by one
// atomic counter (queue[0]).  Before an item of iteration i runs, its job's iteration
// i - 1 must have finished: the last tile of that iteration ran the job's FP64 step and
// then published ready[job] = i (after a fence).  Items are claimed in order, so every
// earlier item belongs to a running block and every wait ends; the waits are bounded all
// the same (an expired wait sets error bit 4 and queue[1], and every later wait gives up
// at once).  A job that has finished skips its remaining items.  The arithmetic of a
// tile and of the step is k_linearize's, so each job's result is bit-identical to the
// per-iteration launches.  A block re-stages the fixed tree's top only when its next tile
// reads another tree.
constexpr int kWaitPolls = 1 << 22;

template <int KIND>
__device__ __forceinline__ void persistent_tile(const JobIn& Jn, const LinDev& L, const CacheF& C, const TileDev& T,
                                                const DNode* staged, int nst, double* swp, float* sfac, double* P) {
  constexpr int D = KindDim<KIND>::D;
  constexpr int M = D * (D + 1) / 2 + D;
  tile_body<KIND>(Jn, L, C, T, staged, nst, swp, sfac, nullptr, nullptr);
  __syncthreads();
  for (int k = threadIdx.x; k < kPStride; k += blockDim.x) {
    if (k >= M && k < kPStats) continue;
    double acc = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) acc += swp[w * kPStride + k];
    P[k] = acc;
  }
}

__global__ void __launch_bounds__(kBlock, 4) k_linearize_persistent(const JobIn* __restrict__ jobs, JobState* states,
                                                                 JobOut* outs, kds_stats* logs, LinDev* lins,
                                                                 const TileDev* __restrict__ tiles, int num_tiles,
                                                                 int max_iter, int stage, double* partials,
                                                                 int32_t* ready, unsigned int* queue, int32_t* err) {
  __shared__ CacheF sC;
  __shared__ float sfac[kWarps * 32 * kMaxFS];
  __shared__ double swp[kWarps * kPStride];
  __shared__ int s_item, s_skip, s_last, s_fail;
  __shared__ __align__(8) unsigned long long s_mbar;
  extern __shared__ float4 sDyn[];
  const DNode* sN = reinterpret_cast<const DNode*>(sDyn);
  const uint32_t mbar = (uint32_t)__cvta_generic_to_shared(&s_mbar);
  const DNode* staged_for = nullptr;  // tree whose top is in shared memory
  int nst = 0;                        // nodes staged (0: read global memory)
  uint32_t phase = 0;                 // parity of the next mbarrier phase
  bool copies = false;                // a copy was issued (settle before exit)
  bool fallback = false;              // a wait gave up: read global memory from here on
  const int items = max_iter * num_tiles;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  for (;;) {
    if (threadIdx.x == 0) {
      s_item = (int)atomicAdd(&queue[0], 1u);
      s_fail = 0;
    }
    __syncthreads();
    const int item = s_item;
    if (item >= items) break;
    const int it = item / num_tiles;
    const int tile = item - it * num_tiles;
    const TileDev T = tiles[tile];
    JobState& S = states[T.job];
    if (threadIdx.x == 0) {
      int skip = 0;
      for (int polls = 0;; ++polls) {
        if (*(volatile int32_t*)&S.done) { skip = 1; break; }
        if (*(volatile int32_t*)&ready[T.job] >= it) {
          __threadfence();
          skip = *(volatile int32_t*)&S.done;  // the step that published may have finished the job
          break;
        }
        if (*(volatile unsigned int*)&queue[1]) { skip = 1; break; }
        if (polls >= kWaitPolls) {
          report_error(err, 4);
          atomicExch(&queue[1], 1u);
          skip = 1;
          break;
        }
        __nanosleep(128);
      }
      s_skip = skip;
    }
    __syncthreads();
    if (s_skip) continue;
    const JobIn& Jn = jobs[T.job];
    const LinDev& L = lins[T.lin];
    const int want = fallback ? 0 : min(stage, L.f_num_nodes);
    if (want > 0 && (L.fnodes != staged_for || want != nst)) {
      const uint32_t bytes = (uint32_t)want * (uint32_t)sizeof(DNode);
      if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(sDyn)),
                     "l"(L.fnodes), "r"(bytes), "r"(mbar)
                     : "memory");
      }
      copies = true;
      if (!mbar_wait(mbar, phase, g_wait_spins)) atomicOr(&s_fail, 1);
      phase ^= 1u;
      __syncthreads();  // one block-wide outcome
      if (s_fail) {
        if (threadIdx.x == 0) report_error(err, 1);
        fallback = true;  // the copy may still land: never stage again, settle at exit
        staged_for = nullptr;
        nst = 0;
      } else {
        staged_for = L.fnodes;
        nst = want;
      }
    } else if (want == 0) {
      nst = 0;
      staged_for = nullptr;
    }
    if (threadIdx.x < (int)(sizeof(CacheF) / 4))
      reinterpret_cast<float*>(&sC)[threadIdx.x] = reinterpret_cast<const float*>(&L.cache)[threadIdx.x];
    __syncthreads();
    double* P = partials + (size_t)tile * kPStride;
    const int use = (L.fnodes == staged_for) ? nst : 0;
    if (Jn.kind == 0) persistent_tile<0>(Jn, L, sC, T, sN, use, swp, sfac, P);
    else if (Jn.kind == 1) persistent_tile<1>(Jn, L, sC, T, sN, use, swp, sfac, P);
    else persistent_tile<2>(Jn, L, sC, T, sN, use, swp, sfac, P);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned prev = atomicAdd(&S.arrive, 1u);
      s_last = (prev == (unsigned)(Jn.tile_count - 1)) ? 1 : 0;
    }
    __syncthreads();
    if (s_last) {
      __threadfence();
      const int Mk = Jn.kind == 0 ? 27 : (Jn.kind == 1 ? 90 : 189);
      job_tail(Jn, S, outs[T.job], logs ? logs + (size_t)T.job * kMaxLog : nullptr, lins, partials, swp, Mk);
      if (threadIdx.x < 32) {  // every lane that wrote the job's state makes it visible, then publish
        __threadfence();
        __syncwarp();
        if (threadIdx.x == 0) atomicExch(&ready[T.job], it + 1);
      }
    }
  }
  if (threadIdx.x == 0 && copies) {
    // the last copy's phase: wait (bounded) until it has landed before the block exits
    if (!mbar_wait(mbar, phase ^ 1u)) report_error(err, 2);
  }
}

// Resets control state, seeds state from the job inputs and writes the first caches.
__device__ void init_job(int j, const JobIn* jobs, JobState* states, JobOut* outs, LinDev* lins) {
  const JobIn& Jn = jobs[j];
  JobState& S = states[j];
  for (int i = 0; i < 12; ++i) S.X[i] = Jn.X0[i];
  for (int i = 0; i < 6; ++i) S.v[i] = Jn.v0[i];
  S.iter = 0;
  S.done = 0;
  S.result = 0;
  S.arrive = 0u;
  S.prev_score = 0.f;
  S.max_iter = Jn.stats_mode ? 1 : Jn.P.max_iterations;
  JobOut& O = outs[j];
  for (int i = 0; i < 12; ++i) O.X[i] = S.X[i];
  for (int i = 0; i < 6; ++i) O.v[i] = S.v[i];
  O.result = Jn.P.max_iterations;
  O.iterations = 0;
  if (Jn.tile_count == 0 || S.max_iter <= 0) {
    // no moving leaves: the round sees zero measurements and fails at iteration 0
    kds_stats z;
    memset(&z, 0, sizeof(z));
    O.stats = z;
    for (int i = 0; i < 144; ++i) O.H[i] = 0.0;
    for (int i = 0; i < 12; ++i) { O.b[i] = 0.0; O.dx[i] = 0.0; }
    S.done = 1;
    O.result = (Jn.mode == KDS_JOB_COMPUTE && S.max_iter > 0 && Jn.P.min_good_measurements > 0) ? 0
                                                                                                  : Jn.P.max_iterations;
    if (Jn.mode != KDS_JOB_COMPUTE) O.result = 0;
    return;
  }
  if (!Jn.keep_cache) refresh_caches(S, lins, Jn.lin_begin, Jn.lin_count);
}

__global__ void k_init_jobs(const JobIn* jobs, JobState* states, JobOut* outs, LinDev* lins, int num_jobs,
                            int32_t* err, int32_t* ready = nullptr, unsigned int* queue = nullptr) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j == 0 && err) *err = 0;
  if (j == 0 && queue) { queue[0] = 0u; queue[1] = 0u; }
  if (j < num_jobs && ready) ready[j] = 0;
  if (j >= num_jobs) return;
  init_job(j, jobs, states, outs, lins);
}

// ---------------------------------------------------------------------------
// Traffic model helper: marks every fixed node that the greedy descents visit.
template <int KIND>
__global__ void k_touch(const JobIn* jobs, const LinDev* lins, uint32_t* bitmap) {
  const JobIn& Jn = jobs[0];
  const LinDev& L = lins[Jn.lin_begin];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Jn.m_num_leaves || L.f_num_nodes <= 0) return;
  const CacheF& C = L.cache;
  float4 md = Jn.m_md[i], nr = Jn.m_nrm[i];
  F3 m = f3(md.x, md.y, md.z), n = f3(nr.x, nr.y, nr.z);
  F3 mw = m, nw = n;
  if (KIND != 0) warp_x(C.v, md.w, m, n, mw, nw);
  F3 q = apply_iso_x(C.Xmf, mw);
  int idx = 0;
  while (idx >= 0) {
    atomicOr(&bitmap[idx >> 5], 1u << (idx & 31));
    DNode nd = load_node(L.fnodes + idx);
    int l = node_left(nd), r = node_right(nd);
    if (l < 0 && r < 0) break;
    idx = dot3x(node_dir(nd), sub3x(q, node_mean(nd))) > 0.0f ? l : r;
  }
}
__global__ void k_popc(const uint32_t* bitmap, int64_t words, unsigned long long* count) {
  unsigned long long c = 0;
  for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < words; w += (int64_t)gridDim.x * blockDim.x)
    c += __popc(bitmap[w]);
  atomicAdd(count, c);
}

int count_touched(Runner& R, int kind, int64_t fixed_nodes, int64_t* out, cudaStream_t s) {
  *out = 0;
  if (R.num_jobs < 1 || fixed_nodes <= 0) return KDS_OK;
  k_init_jobs<<<1, 128, 0, s>>>(R.d_jobs, R.d_states, R.d_outs, R.d_lins, 1, R.d_err); ::kds::count_launch();
  int64_t words = (fixed_nodes + 31) / 32;
  uint32_t* bm = nullptr;
  unsigned long long* cnt = nullptr;
  KDS_CK(cudaMalloc(&bm, words * 4 + 64));
  cnt = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(bm) + ((words * 4 + 7) & ~7ll));
  cudaMemsetAsync(bm, 0, words * 4 + 64, s);
  int nl = R.h_jobs[0].m_num_leaves;
  int g = (nl + 255) / 256;
  if (g > 0) {
    if (kind == 0) k_touch<0><<<g, 256, 0, s>>>(R.d_jobs, R.d_lins, bm);
    else k_touch<1><<<g, 256, 0, s>>>(R.d_jobs, R.d_lins, bm);
    ::kds::count_launch();
  }
  k_popc<<<64, 256, 0, s>>>(bm, words, cnt); ::kds::count_launch();
  unsigned long long h = 0;
  cudaMemcpyAsync(&h, cnt, 8, cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(bm);
  if (e != cudaSuccess) return cuda_status(e, "count_touched", __FILE__, __LINE__);
  *out = (int64_t)h;
  return KDS_OK;
}

// ---------------------------------------------------------------------------
// Host runner
int Runner::reserve(int nj, int nl, int nt) {
  if (nj <= cap_jobs && nl <= cap_lins && nt <= cap_tiles) return KDS_OK;
  // grow by at least half of the old capacity: callers whose job sets vary from call to
  // call (a tracker's frames, served ticks) reallocate -- a device-wide synchronisation in
  // cudaFree -- a logarithmic number of times instead of at every new maximum
  const int oj = cap_jobs, ol = cap_lins, ot = cap_tiles;
  release();
  cap_jobs = std::max({nj, oj + oj / 2, 1});
  cap_lins = std::max({nl, ol + ol / 2, 1});
  cap_tiles = std::max({nt, ot + ot / 2, 1});
  size_t bytes = sizeof(JobIn) * cap_jobs + sizeof(JobState) * cap_jobs + sizeof(JobOut) * cap_jobs +
                 sizeof(kds_stats) * kMaxLog * cap_jobs + sizeof(LinDev) * cap_lins + sizeof(TileDev) * cap_tiles +
                 sizeof(double) * kPStride * cap_tiles + sizeof(int32_t) * cap_jobs + sizeof(int2) * cap_tiles +
                 12 * 256;
  cudaError_t e = cudaMalloc(&block, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    block = nullptr;
    cap_jobs = cap_lins = cap_tiles = 0;
    set_error("cudaMalloc of %zu bytes for the aligner workspace failed", bytes);
    return KDS_ERR_OOM;
  }
  char* p = (char*)block;
  auto carve = [&](size_t sz) {
    char* r = p;
    p += (sz + 255) & ~(size_t)255;
    return (void*)r;
  };
  d_jobs = (JobIn*)carve(sizeof(JobIn) * cap_jobs);
  d_states = (JobState*)carve(sizeof(JobState) * cap_jobs);
  d_outs = (JobOut*)carve(sizeof(JobOut) * cap_jobs);
  d_logs = (kds_stats*)carve(sizeof(kds_stats) * kMaxLog * cap_jobs);
  d_lins = (LinDev*)carve(sizeof(LinDev) * cap_lins);
  d_tiles = (TileDev*)carve(sizeof(TileDev) * cap_tiles);
  d_partials = (double*)carve(sizeof(double) * kPStride * cap_tiles);
  d_err = (int32_t*)carve(sizeof(int32_t));
  d_ready = (int32_t*)carve(sizeof(int32_t) * cap_jobs);
  d_queue = (unsigned int*)carve(2 * sizeof(unsigned int));
  d_pairs = (int2*)carve(sizeof(int2) * cap_tiles);
  return KDS_OK;
}

void Runner::release() {
  drop_graph();
  for (cudaEvent_t e : prof_ev) cudaEventDestroy(e);
  prof_ev.clear();
  if (block) cudaFree(block);
  block = nullptr;
  cap_jobs = cap_lins = cap_tiles = 0;
}

void Runner::drop_graph() {
  if (gexec) cudaGraphExecDestroy(gexec);
  if (graph) cudaGraphDestroy(graph);
  gexec = nullptr;
  graph = nullptr;
  graph_key.clear();
}

// Builds the tile list and device inputs for `jobs` (host descriptions).
int Runner::setup(const std::vector<JobIn>& jobs_in, const std::vector<LinDev>& lins_in, cudaStream_t s) {
  h_jobs = jobs_in;
  h_lins = lins_in;
  h_tiles.clear();
  std::vector<int> order(h_jobs.size());
  for (size_t j = 0; j < order.size(); ++j) order[j] = (int)j;
  if (order_by_size)
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return h_jobs[a].m_num_leaves > h_jobs[b].m_num_leaves; });
  for (int kind = 0; kind < 3; ++kind) {
    kind_begin[kind] = (int)h_tiles.size();
    for (int j : order) {
      JobIn& Jn = h_jobs[j];
      if (Jn.kind != kind) continue;
      Jn.tile_begin = (int32_t)h_tiles.size();
      for (int l = Jn.lin_begin; l < Jn.lin_begin + Jn.lin_count; ++l) {
        for (int b = 0; b < Jn.m_num_leaves; b += kBlock) {
          TileDev t;
          t.job = (int32_t)j;
          t.lin = l;
          t.leaf_begin = b;
          t.leaf_end = std::min(b + kBlock, Jn.m_num_leaves);
          h_tiles.push_back(t);
        }
      }
      Jn.tile_count = (int32_t)h_tiles.size() - Jn.tile_begin;
    }
    kind_count[kind] = (int)h_tiles.size() - kind_begin[kind];
  }
  // blocks of two consecutive tiles of one (job, fixed entry), per kind
  h_pairs.clear();
  for (int kind = 0; kind < 3; ++kind) {
    kind_pair_begin[kind] = (int)h_pairs.size();
    const int e = kind_begin[kind] + kind_count[kind];
    for (int t = kind_begin[kind]; t < e;) {
      const bool two = t + 1 < e && h_tiles[t + 1].job == h_tiles[t].job && h_tiles[t + 1].lin == h_tiles[t].lin;
      h_pairs.push_back(make_int2(t, two ? t + 1 : -1));
      t += two ? 2 : 1;
    }
    kind_pair_count[kind] = (int)h_pairs.size() - kind_pair_begin[kind];
  }
  int rc = reserve((int)h_jobs.size(), (int)h_lins.size(), (int)h_tiles.size());
  if (rc) return rc;
  num_jobs = (int)h_jobs.size();
  num_tiles = (int)h_tiles.size();
  KDS_CK(cudaMemcpyAsync(d_jobs, h_jobs.data(), sizeof(JobIn) * h_jobs.size(), cudaMemcpyHostToDevice, s));
  KDS_CK(cudaMemcpyAsync(d_lins, h_lins.data(), sizeof(LinDev) * h_lins.size(), cudaMemcpyHostToDevice, s));
  if (num_tiles) {
    KDS_CK(cudaMemcpyAsync(d_tiles, h_tiles.data(), sizeof(TileDev) * h_tiles.size(), cudaMemcpyHostToDevice, s));
    KDS_CK(cudaMemcpyAsync(d_pairs, h_pairs.data(), sizeof(int2) * h_pairs.size(), cudaMemcpyHostToDevice, s));
  }
  return KDS_OK;
}

int Runner::max_launches() const {
  int m = 0;
  for (const JobIn& J : h_jobs) {
    int it = (J.mode == KDS_JOB_COMPUTE) ? (J.stats_mode ? 1 : J.P.max_iterations) : 1;
    m = std::max(m, it);
  }
  return m;
}

int phase_stamps(int on, unsigned long long* out16) {
  if (on >= 0) KDS_CK(cudaMemcpyToSymbol(g_phase_on, &on, sizeof(int)));
  if (out16) KDS_CK(cudaMemcpyFromSymbol(out16, g_phase, sizeof(unsigned long long) * 16));
  return KDS_OK;
}

int set_wait_spins(int32_t spins) {
  if (spins < 0) { set_error("kds_set_tma_wait_limit: negative limit %d", spins); return KDS_ERR_INVALID_ARG; }
  KDS_CK(cudaMemcpyToSymbol(g_wait_spins, &spins, sizeof(int32_t)));
  return KDS_OK;
}

int Runner::ensure_events(int n) {
  while ((int)prof_ev.size() < n) {
    cudaEvent_t e;
    KDS_CK(cudaEventCreate(&e));
    prof_ev.push_back(e);
  }
  return KDS_OK;
}

double Runner::profile_mean_ms(int* launches) const {
  double sum = 0.0;
  int n = 0;
  for (int i = 0; i < prof_launches; ++i) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, prof_ev[2 * i], prof_ev[2 * i + 1]) == cudaSuccess) {
      sum += ms;
      ++n;
    } else {
      cudaGetLastError();
    }
  }
  if (launches) *launches = n;
  return n ? sum / n : 0.0;
}

// A profiling event on s: inside a stream capture it becomes an external event node of
// the graph (recorded at every replay); outside one it is a plain record.
static cudaError_t record_profile_event(cudaEvent_t e, cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaError_t r = cudaStreamIsCapturing(s, &cs);
  if (r != cudaSuccess) return r;
  return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(e, s, cudaEventRecordExternal)
                                             : cudaEventRecord(e, s);
}

// Blocks of the persistent kernel: every SM full at its occupancy for `smem` bytes of
// dynamic shared memory, at most one block per work item.
static int persistent_grid(size_t smem, int64_t items) {
  int nsm = 0, dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm <= 0)
    nsm = 148;
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_linearize_persistent, kBlock, smem) != cudaSuccess ||
      per < 1) {
    cudaGetLastError();
    per = 1;
  }
  return (int)std::max<int64_t>(1, std::min<int64_t>(items, (int64_t)nsm * per));
}

int Runner::enqueue(cudaStream_t s, int32_t* dbg_match, int32_t* dbg_status) {
  if (num_jobs == 0) return KDS_OK;
  if (persistent && !dbg_match) {
    k_init_jobs<<<(num_jobs + 127) / 128, 128, 0, s>>>(d_jobs, d_states, d_outs, d_lins, num_jobs, d_err, d_ready,
                                                       d_queue);
    ::kds::count_launch();
    const int L = max_launches();
    prof_launches = profiling ? 1 : 0;
    if (profiling) {
      int rc = ensure_events(2);
      if (rc) return rc;
    }
    const size_t stage_bytes = (size_t)stage_nodes * sizeof(DNode);
    if (!persistent_attr_set) {
      KDS_CK(cudaFuncSetAttribute((const void*)k_linearize_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  200 * 1024));
      persistent_attr_set = true;
    }
    if (num_tiles > 0 && L > 0) {
      const int grid = persistent_grid(stage_bytes, (int64_t)num_tiles * L);
      if (profiling) KDS_CK(record_profile_event(prof_ev[0], s));
      k_linearize_persistent<<<grid, kBlock, stage_bytes, s>>>(d_jobs, d_states, d_outs, d_logs, d_lins, d_tiles,
                                                               num_tiles, L, stage_nodes, d_partials, d_ready,
                                                               d_queue, d_err);
      ::kds::count_launch();
      if (profiling) KDS_CK(record_profile_event(prof_ev[1], s));
    }
    KDS_CK(cudaGetLastError());
    return KDS_OK;
  }
  k_init_jobs<<<(num_jobs + 127) / 128, 128, 0, s>>>(d_jobs, d_states, d_outs, d_lins, num_jobs, d_err);
  ::kds::count_launch();
  int L = max_launches();
  int nk = (kind_count[0] ? 1 : 0) + (kind_count[1] ? 1 : 0) + (kind_count[2] ? 1 : 0);
  prof_launches = profiling ? L * nk : 0;
  if (profiling) {
    int rc = ensure_events(2 * prof_launches);
    if (rc) return rc;
  }
  int ev = 0;
  const int stage = stage_nodes;
  const size_t stage_bytes = (size_t)stage * sizeof(DNode);
  if (stage_bytes > 0 && !smem_attr_set) {  // static + dynamic shared memory can pass 48 KB
    const void* fs[6] = {(const void*)k_linearize<0>, (const void*)k_linearize<1>, (const void*)k_linearize<2>,
                         (const void*)k_linearize_pair<0>, (const void*)k_linearize_pair<1>,
                         (const void*)k_linearize_pair<2>};
    for (int k = 0; k < 6; ++k) KDS_CK(cudaFuncSetAttribute(fs[k], cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    smem_attr_set = true;
  }
  for (int i = 0; i < L; ++i) {
    for (int kind = 0; kind < 3; ++kind) {
      if (!kind_count[kind]) continue;
      if (profiling) KDS_CK(record_profile_event(prof_ev[ev++], s));
      if (pair_tiles) {
        const int nb = kind_pair_count[kind], p0 = kind_pair_begin[kind];
        if (kind == 0)
          k_linearize_pair<0><<<nb, kBlock, stage_bytes, s>>>(d_jobs, d_states, d_outs, d_logs, d_lins, d_tiles,
                                                              d_pairs, p0, stage, d_partials, dbg_match, dbg_status,
                                                              d_err);
        else if (kind == 1)
          k_linearize_pair<1><<<nb, kBlock, stage_bytes, s>>>(d_jobs, d_states, d_outs, d_logs, d_lins, d_tiles,
                                                              d_pairs, p0, stage, d_partials, dbg_match, dbg_status,
                                                              d_err);
        else
          k_linearize_pair<2><<<nb, kBlock, stage_bytes, s>>>(d_jobs, d_states, d_outs, d_logs, d_lins, d_tiles,
                                                              d_pairs, p0, stage, d_partials, dbg_match, dbg_status,
                                                              d_err);
      } else if (kind == 0)
        k_linearize<0><<<kind_count[0], kBlock, stage_bytes, s>>>(d_jobs, d_states, d_outs, d_logs, d_lins,
                                                                     d_tiles, kind_begin[0], stage, d_partials,
                                                                     dbg_match, dbg_status, d_err);
      else if (kind == 1)
        k_linearize<1><<<kind_count[1], kBlock, stage_bytes, s>>>(d_jobs, d_states, d_outs, d_logs, d_lins,
                                                                     d_tiles, kind_begin[1], stage, d_partials,
                                                                     dbg_match, dbg_status, d_err);
      else
        k_linearize<2><<<kind_count[2], kBlock, stage_bytes, s>>>(d_jobs, d_states, d_outs, d_logs, d_lins,
                                                                     d_tiles, kind_begin[2], stage, d_partials,
                                                                     dbg_match, dbg_status, d_err);
      ::kds::count_launch();
      if (profiling) KDS_CK(record_profile_event(prof_ev[ev++], s));
    }
  }
  KDS_CK(cudaGetLastError());
  return KDS_OK;
}

int Runner::run(cudaStream_t s, bool use_graph, int32_t* dbg_match, int32_t* dbg_status) {
  if (!use_graph || dbg_match) return enqueue(s, dbg_match, dbg_status);
  // graph key: everything the captured launches depend on
  std::vector<int64_t> key;
  key.push_back((int64_t)(uintptr_t)block);
  key.push_back(num_jobs);
  key.push_back(num_tiles);
  key.push_back(max_launches());
  for (int k = 0; k < 3; ++k) { key.push_back(kind_begin[k]); key.push_back(kind_count[k]); }
  key.push_back(profiling ? 1 : 0);
  key.push_back(stage_nodes);
  key.push_back(order_by_size);
  key.push_back(persistent);
  key.push_back(pair_tiles);
  if (key != graph_key) {
    // capture only a shape that repeats: a one-off shape (every call of a stream of
    // different scans) costs less launched directly than captured and instantiated
    if (key != last_key) {
      last_key = key;
      return enqueue(s, nullptr, nullptr);
    }
    drop_graph();
    cudaStream_t cs;
    KDS_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    int rc = KDS_OK;
    if (e == cudaSuccess) {
      rc = enqueue(cs, nullptr, nullptr);
      e = cudaStreamEndCapture(cs, &graph);
    }
    cudaStreamDestroy(cs);
    if (e != cudaSuccess || rc) {
      graph = nullptr;
      return rc ? rc : cuda_status(e, "graph capture", __FILE__, __LINE__);
    }
    KDS_CK(cudaGraphInstantiate(&gexec, graph, 0));
    graph_key = key;
  }
  KDS_CK(cudaGraphLaunch(gexec, s));
  return KDS_OK;
}

int Runner::fetch(cudaStream_t s, std::vector<JobOut>& outs, std::vector<kds_stats>* logs) {
  outs.resize(num_jobs);
  if (num_jobs == 0) return KDS_OK;
  KDS_CK(cudaMemcpyAsync(outs.data(), d_outs, sizeof(JobOut) * num_jobs, cudaMemcpyDeviceToHost, s));
  if (logs) {
    logs->resize((size_t)num_jobs * kMaxLog);
    KDS_CK(cudaMemcpyAsync(logs->data(), d_logs, sizeof(kds_stats) * kMaxLog * num_jobs, cudaMemcpyDeviceToHost, s));
  }
  int32_t err = 0;
  KDS_CK(cudaMemcpyAsync(&err, d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  KDS_CK(cudaStreamSynchronize(s));
  return timeout_status(err);
}

// KDS_OK, or KDS_ERR_TIMEOUT with a message for the error bits of a launch sequence.
int timeout_status(int32_t err) {
  if (!err) return KDS_OK;
  if (err & 2)
    set_error("a bounded wait for a tree-top copy gave up and the copy was still not seen complete when its block "
              "exited: the results were computed from global memory, but the CUDA context should be considered "
              "unusable");
  else
    set_error("a bounded wait for a tree-top copy gave up; the results were computed from global memory and are "
              "valid");
  return KDS_ERR_TIMEOUT;
}

// ---------------------------------------------------------------------------
// Served-loop helpers (kds_serve.cu): jobs addressed by slot.
namespace {

__global__ void k_admit_slots(const int32_t* slots, int n, const JobIn* new_jobs, const LinDev* new_lins,
                              JobIn* jobs, JobState* states, JobOut* outs, LinDev* lins) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int slot = slots[i];
  jobs[slot] = new_jobs[i];
  lins[slot] = new_lins[i];
  init_job(slot, jobs, states, outs, lins);
}

__global__ void k_collect(int n, const JobState* states, const JobOut* outs, const unsigned long long* touched,
                          SlotResult* res) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int done = *(const volatile int32_t*)&states[j].done;
  res[j].done = done;
  if (!done) return;
  res[j].touched = touched ? touched[j] : 0ull;
  const JobOut& O = outs[j];
  res[j].result = O.result;
  res[j].iterations = O.iterations;
  res[j].stats = O.stats;
  for (int k = 0; k < 12; ++k) res[j].X[k] = O.X[k];
  for (int k = 0; k < 6; ++k) res[j].v[k] = O.v[k];
}

}  // namespace

static_assert(kBlock == kTileSurfels, "tile size");

int linearize_smem_setup() {
  const int bytes = kStageNodes * (int)sizeof(DNode);
  KDS_CK(cudaFuncSetAttribute((const void*)k_linearize<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  KDS_CK(cudaFuncSetAttribute((const void*)k_linearize<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  KDS_CK(cudaFuncSetAttribute((const void*)k_linearize<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  KDS_CK(cudaFuncSetAttribute((const void*)k_linearize_pair<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  KDS_CK(cudaFuncSetAttribute((const void*)k_linearize_pair<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  KDS_CK(cudaFuncSetAttribute((const void*)k_linearize_pair<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  return KDS_OK;
}

int launch_admit_slots(const int32_t* d_slots, int n, const JobIn* new_jobs, const LinDev* new_lins, JobIn* jobs,
                       JobState* states, JobOut* outs, LinDev* lins, cudaStream_t s) {
  if (n <= 0) return KDS_OK;
  k_admit_slots<<<(n + 127) / 128, 128, 0, s>>>(d_slots, n, new_jobs, new_lins, jobs, states, outs, lins);
  count_launch();
  KDS_CK(cudaGetLastError());
  return KDS_OK;
}

int launch_linearize(int kind, int ntiles, const JobIn* jobs, JobState* states, JobOut* outs, LinDev* lins,
                     const TileDev* tiles, double* partials, cudaStream_t s) {
  if (ntiles <= 0) return KDS_OK;
  const size_t stage_bytes = (size_t)kServeStage * sizeof(DNode);
  if (kind == 0)
    k_linearize<0><<<ntiles, kBlock, stage_bytes, s>>>(jobs, states, outs, nullptr, lins, tiles, 0, kServeStage,
                                                       partials, nullptr, nullptr, nullptr);
  else if (kind == 1)
    k_linearize<1><<<ntiles, kBlock, stage_bytes, s>>>(jobs, states, outs, nullptr, lins, tiles, 0, kServeStage,
                                                       partials, nullptr, nullptr, nullptr);
  else
    k_linearize<2><<<ntiles, kBlock, stage_bytes, s>>>(jobs, states, outs, nullptr, lins, tiles, 0, kServeStage,
                                                       partials, nullptr, nullptr, nullptr);
  count_launch();
  KDS_CK(cudaGetLastError());
  return KDS_OK;
}

int launch_linearize_pairs(int kind, int npairs, const JobIn* jobs, JobState* states, JobOut* outs, LinDev* lins,
                           const TileDev* tiles, const int2* pairs, double* partials, cudaStream_t s) {
  if (npairs <= 0) return KDS_OK;
  const size_t stage_bytes = (size_t)kServeStage * sizeof(DNode);
  if (kind == 0)
    k_linearize_pair<0><<<npairs, kBlock, stage_bytes, s>>>(jobs, states, outs, nullptr, lins, tiles, pairs, 0,
                                                            kServeStage, partials, nullptr, nullptr, nullptr);
  else if (kind == 1)
    k_linearize_pair<1><<<npairs, kBlock, stage_bytes, s>>>(jobs, states, outs, nullptr, lins, tiles, pairs, 0,
                                                            kServeStage, partials, nullptr, nullptr, nullptr);
  else
    k_linearize_pair<2><<<npairs, kBlock, stage_bytes, s>>>(jobs, states, outs, nullptr, lins, tiles, pairs, 0,
                                                            kServeStage, partials, nullptr, nullptr, nullptr);
  count_launch();
  KDS_CK(cudaGetLastError());
  return KDS_OK;
}

int launch_collect(int n, const JobState* states, const JobOut* outs, const unsigned long long* touched,
                   SlotResult* res, cudaStream_t s) {
  if (n <= 0) return KDS_OK;
  k_collect<<<(n + 127) / 128, 128, 0, s>>>(n, states, outs, touched, res);
  count_launch();
  KDS_CK(cudaGetLastError());
  return KDS_OK;
}

int launch_touch(int kind, const JobIn* jobs, const LinDev* lins, int slot, int num_leaves, uint32_t* bitmap,
                 int64_t words, unsigned long long* count, cudaStream_t s) {
  KDS_CK(cudaMemsetAsync(bitmap, 0, (size_t)words * 4, s));
  KDS_CK(cudaMemsetAsync(count, 0, sizeof(unsigned long long), s));
  const int g = (num_leaves + 255) / 256;
  if (g > 0) {
    if (kind == 0) k_touch<0><<<g, 256, 0, s>>>(jobs + slot, lins, bitmap);
    else k_touch<1><<<g, 256, 0, s>>>(jobs + slot, lins, bitmap);
    count_launch();
  }
  k_popc<<<64, 256, 0, s>>>(bitmap, words, count);
  count_launch();
  KDS_CK(cudaGetLastError());
  return KDS_OK;
}

// ---------------------------------------------------------------------------
// One linearization (buildQuadraticForm) that allocates nothing.
//
// Some callers cannot allocate device memory when they linearize: a real-time
// odometry or bundle-adjustment loop that reserves all of its memory at start-up and
// must not call cudaMalloc/cudaFree afterwards (they can block on the device and on
// allocator locks), or code that must not touch the allocator while it enqueues work.
// For them the scratch of k_linearize -- the job, state and output records, the
// fixed-entry record, the tile list and one FP64 partial per tile -- lives in one
// file-scope device array.  Every call on a device shares that array: calls that
// overlap on the GPU (other streams, other host threads) race on it, and it keeps the
// last call's contents.  The tile list is rebuilt and the job state reset by every
// call; each tile writes its own partial before the last tile reads them.
namespace {

constexpr int kStaticMaxTiles = 512;  // 512 tiles x 128 = 65,536 moving surfels per call
constexpr int kStaticStage = 2047;    // fixed-tree nodes staged per block (64 KB)

// What the call reads back: the job's outputs and the launch's own error bits.
struct StaticResult {
  JobOut out;
  int32_t err;
  int32_t pad_[3];
};

struct StaticScratch {
  JobIn job;
  JobState state;
  StaticResult res;
  LinDev lin;
  TileDev tiles[kStaticMaxTiles];
  double partials[(size_t)kStaticMaxTiles * kPStride];
};

__device__ __align__(256) unsigned char g_static_scratch[sizeof(StaticScratch)];

std::mutex g_static_mu;
StaticScratch* g_static_ptr[64] = {nullptr};

// Writes the job and fixed-entry records and the tile list into the scratch.
__global__ void k_static_setup(StaticScratch* scr, JobIn job, LinDev lin, int ntiles) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    scr->job = job;
    scr->lin = lin;
    scr->res.err = 0;
  }
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
    TileDev d;
    d.job = 0;
    d.lin = 0;
    d.leaf_begin = t * kBlock;
    d.leaf_end = min((t + 1) * kBlock, job.m_num_leaves);
    scr->tiles[t] = d;
  }
}

// First call on a device, with that device current: resolves the array's device
// address and raises the kernels' dynamic shared-memory limit.
int static_setup(StaticScratch** out) {
  int dev = 0;
  KDS_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) { set_error("device ordinal %d out of range", dev); return KDS_ERR_INVALID_ARG; }
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || p == nullptr) return cuda_status(e, "cudaGetSymbolAddress(g_static_scratch)", __FILE__, __LINE__);
    const int bytes = kStaticStage * (int)sizeof(DNode);
    KDS_CK(cudaFuncSetAttribute((const void*)k_linearize<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    KDS_CK(cudaFuncSetAttribute((const void*)k_linearize<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    g_static_ptr[dev] = reinterpret_cast<StaticScratch*>(p);
  }
  *out = g_static_ptr[dev];
  return KDS_OK;
}

}  // namespace

int linearize_static(const TreeDev& fixed, const TreeDev& moving, int32_t type, const kds_aligner_params& P,
                     const double* X, const double* Xf, const double* v, const double* fv, int32_t stats_mode,
                     cudaStream_t s, double* H, double* b, kds_stats* stats) {
  const int64_t nl = moving.num_leaves;
  const int64_t ntiles = (nl + kBlock - 1) / kBlock;
  if (ntiles > kStaticMaxTiles) {
    set_error("kds_linearize_static: %lld moving leaves exceed the static maximum of %d", (long long)nl,
              kStaticMaxTiles * kBlock);
    return KDS_ERR_CAPACITY;
  }
  StaticScratch* scr = nullptr;
  int rc = static_setup(&scr);
  if (rc) return rc;
  JobIn J;
  memset(&J, 0, sizeof(J));
  J.m_md = moving.leaf_md;
  J.m_nrm = moving.leaf_nrm;
  J.m_num_leaves = (int32_t)nl;
  J.kind = type == KDS_ICP ? 0 : 1;
  J.mode = KDS_JOB_LINEARIZE;
  J.stats_mode = stats_mode;
  J.lin_begin = 0;
  J.lin_count = 1;
  J.tile_begin = 0;
  J.tile_count = (int32_t)ntiles;
  J.P.kernel_threshold = P.kernel_threshold;
  J.P.damping = P.damping;
  J.P.max_error = P.max_error;
  J.P.min_normal_cos = P.min_normal_cos;
  J.P.min_good_measurements = P.min_good_measurements;
  J.P.max_iterations = P.max_iterations;
  J.P.velocity_damping = P.velocity_damping;
  J.P.term_crit = P.term_crit;
  J.P.d_pert = P.d_pert;
  J.P.d_score = P.d_score;
  for (int i = 0; i < 12; ++i) J.X0[i] = X[i];
  for (int i = 0; i < 6; ++i) J.v0[i] = (type == KDS_ICP || !v) ? 0.0 : v[i];
  LinDev L;
  memset(&L, 0, sizeof(L));
  L.fnodes = fixed.nodes;
  L.fdts = fixed.dts_f;
  L.f_num_nodes = (int32_t)fixed.num_nodes;
  L.job = 0;
  for (int i = 0; i < 12; ++i) L.Xf[i] = Xf[i];
  for (int i = 0; i < 6; ++i) L.fv[i] = fv ? fv[i] : 0.0;
  k_static_setup<<<1, 256, 0, s>>>(scr, J, L, (int)ntiles);
  count_launch();
  k_init_jobs<<<1, 128, 0, s>>>(&scr->job, &scr->state, &scr->res.out, &scr->lin, 1, &scr->res.err);
  count_launch();
  if (ntiles > 0) {
    const size_t stage_bytes = (size_t)kStaticStage * sizeof(DNode);
    if (J.kind == 0)
      k_linearize<0><<<(unsigned)ntiles, kBlock, stage_bytes, s>>>(&scr->job, &scr->state, &scr->res.out, nullptr,
                                                                  &scr->lin, scr->tiles, 0, kStaticStage,
                                                                  scr->partials, nullptr, nullptr, &scr->res.err);
    else
      k_linearize<1><<<(unsigned)ntiles, kBlock, stage_bytes, s>>>(&scr->job, &scr->state, &scr->res.out, nullptr,
                                                                  &scr->lin, scr->tiles, 0, kStaticStage,
                                                                  scr->partials, nullptr, nullptr, &scr->res.err);
    count_launch();
  }
  KDS_CK(cudaGetLastError());
  // outputs and error bits in one copy on the caller's stream
  StaticResult R;
  KDS_CK(cudaMemcpyAsync(&R, &scr->res, sizeof(StaticResult), cudaMemcpyDeviceToHost, s));
  KDS_CK(cudaStreamSynchronize(s));
  const int D = type == KDS_ICP ? 6 : 12;
  if (H) memcpy(H, R.out.H, sizeof(double) * D * D);
  if (b) memcpy(b, R.out.b, sizeof(double) * D);
  if (stats) *stats = R.out.stats;
  return timeout_status(R.err);
}

}  // namespace kds
