// CPU oracle: ICP / CT-ICP Gauss-Newton -- TEST INFRASTRUCTURE ONLY.
//
// Restates, per moving leaf:
//   ICP_::quadraticTerm            kd/icp/icp_impl_.h:102-152
//   ICP_3D_Traits::errorAndJacobian kd/d3/icp_.h:40-60
//   CTICP_::quadraticTerm          kd/cticp/cticp_impl_.h:105-181
//   CTICP_::quadraticTermDual      kd/cticp/cticp_impl_.h:183-293
//   CTICP_3D_Traits::applyVelocities / errorAndJacobianVelocityA/B  kd/d3/cticp_impl_.h:10-96
//   ICPWsItemDiag_/Cross_::pack    kd/icp/icp_ws_item_.h:27-34,73-75
// and per iteration:
//   ICP_CPU_/CTICP_CPU_::_buildQuadraticForm  kd/icp/icp_cpu_impl_.h:27-98,
//                                             kd/cticp/cticp_cpu_impl_.h:26-126
//   StableAdder_                   kd/utils/stable_adder_.h:21-74
//   ICP_::oneRound / CTICP_::oneRound  kd/icp/icp_impl_.h:52-90, kd/cticp/cticp_impl_.h:47-92
//   posePriorBuildQuadraticForm    kd/icp/tree_aligner_base_.h:139-152
//   TreeAlignerBase_::compute      kd/icp/tree_aligner_base_.h:100-115
//   ICPTerminationCriteriaScore_   kd/icp/icp_stats_.h:84-102
//
// Three modes:
//   MODE_REF32  float everywhere, StableAdder_ sums over num_threads chunks, float LDLT
//               and pose update -- the reference CPU path as written.
//   MODE_MIXED  float per-leaf terms, FP64 sums / solve / pose -- the product's
//               semantics, in the product's own summation order (128-leaf tiles, warp
//               Kahan sums, FP64 partials), its Cholesky and its canonical FP64 expmap,
//               so that a run is bit-identical to the GPU's.
//   MODE_FP64   everything in double -- the precision reference.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <future>
#include <type_traits>
#include <vector>

#include "orc_align.hpp"
#include "orc_math.hpp"

namespace orc {

enum { ST_INLIER = 0, ST_OUTLIER = 1, ST_BAD = 2, ST_ERR_NORMAL = 3, ST_ERR_FN = 4 };

template <class T> struct Cache {
  Iso<T> Xm, Xf, Xmf;
};

template <class T> struct LeafRes {
  int match = -1;
  int status = ST_BAD;
  T e = 0, chi2 = 0, gamma = 0;
  T J[18];
};

static inline bool is_leaf(const Node& n) { return n.left < 0 && n.right < 0; }

template <class T> static inline V3<T> nmean(const Node& n) { return v3<T>((T)n.mean[0], (T)n.mean[1], (T)n.mean[2]); }
template <class T> static inline V3<T> ndir(const Node& n) { return v3<T>((T)n.dir[0], (T)n.dir[1], (T)n.dir[2]); }

template <class T> static inline bool which_side(const Node& nd, const V3<T>& q) {
  return dot3(ndir<T>(nd), vsub(q, nmean<T>(nd))) > T(0);
}

template <class T> static int descend(const Tree& F, const V3<T>& q) {
  int idx = 0;
  if (F.nodes.empty()) return -1;
  while (idx >= 0 && !is_leaf(F.nodes[idx])) {
    const Node& a = F.nodes[idx];
    idx = which_side(a, q) ? a.left : a.right;
  }
  return idx;
}

// CTICP_3D_Traits::applyVelocities(v, node) (kd/d3/cticp_impl_.h:75-85)
template <class T> static void warp_leaf(const T* v, T dt, const V3<T>& m, const V3<T>& n, V3<T>& mo, V3<T>& no) {
  V3<T> td = v3<T>(v[0] * dt, v[1] * dt, v[2] * dt);
  V3<T> rd = v3<T>(v[3] * dt, v[4] * dt, v[5] * dt);
  M3<T> R = rodrigues(rd);
  mo = vadd(mat_vec(R, m), td);
  no = mat_vec(R, n);
}

// errorAndJacobianVelocityA (kd/d3/cticp_impl_.h:10-39)
template <class T>
void err_jac_vel_A(T& e, T* J, const Iso<T>& Ta, const V3<T>& pa_l, const V3<T>& na_l, const V3<T>& pb_g,
                   const V3<T>& nb_g, const T* va, T dt) {
  T ma[6];
  for (int i = 0; i < 6; ++i) ma[i] = va[i] * dt;
  V3<T> tm = v3<T>(ma[0], ma[1], ma[2]);
  V3<T> wa = v3<T>(ma[3], ma[4], ma[5]);
  V3<T> pa_m, na_m;
  M3<T> dRp, dRn;
  dRxp(pa_m, dRp, wa, pa_l);
  dRxp(na_m, dRn, wa, na_l);
  pa_m = vadd(pa_m, tm);
  const M3<T>& Ra = Ta.R;
  V3<T> pa_g = vadd(mat_vec(Ra, pa_m), Ta.t);
  V3<T> na_g = mat_vec(Ra, na_m);
  V3<T> n = vadd(na_g, nb_g);
  V3<T> dp = vsub(pa_g, pb_g);
  e = dot3(dp, n);
  M3<T> A = mat_mul(Ra, dRp), B = mat_mul(Ra, dRn);
  for (int c = 0; c < 3; ++c) {
    J[c] = dot3(n, mcol(Ra, c));
    J[3 + c] = dot3(n, mcol(A, c)) + dot3(dp, mcol(B, c));
  }
  for (int i = 0; i < 6; ++i) J[i] = J[i] * dt;
}

// errorAndJacobianVelocityB (kd/d3/cticp_impl_.h:43-73)
template <class T>
void err_jac_vel_B(T& e, T* J, const Iso<T>& Tb, const V3<T>& pa_g, const V3<T>& na_g, const V3<T>& pb_l,
                   const V3<T>& nb_l, const T* vb, T dt) {
  T mb[6];
  for (int i = 0; i < 6; ++i) mb[i] = vb[i] * dt;
  V3<T> tm = v3<T>(mb[0], mb[1], mb[2]);
  V3<T> wb = v3<T>(mb[3], mb[4], mb[5]);
  V3<T> pb_m, nb_m;
  M3<T> dRp, dRn;
  dRxp(pb_m, dRp, wb, pb_l);
  dRxp(nb_m, dRn, wb, nb_l);
  pb_m = vadd(pb_m, tm);
  const M3<T>& Rb = Tb.R;
  V3<T> pb_g = vadd(mat_vec(Rb, pb_m), Tb.t);
  V3<T> nb_g = mat_vec(Rb, nb_m);
  V3<T> n = vadd(na_g, nb_g);
  V3<T> dp = vsub(pa_g, pb_g);
  e = dot3(dp, n);
  M3<T> A = mat_mul(Rb, dRp), B = mat_mul(Rb, dRn);
  V3<T> nn = vneg(n);
  for (int c = 0; c < 3; ++c) {
    J[c] = dot3(nn, mcol(Rb, c));
    J[3 + c] = dot3(nn, mcol(A, c)) + dot3(dp, mcol(B, c));
  }
  for (int i = 0; i < 6; ++i) J[i] = J[i] * dt;
}

// forced_status >= 0 replays a recorded correspondence: the fixed leaf is forced_match,
// the gates are skipped and the leaf contributes iff forced_status is inlier or outlier
// (the robust weight is recomputed in T from the error).
template <class T>
static LeafRes<T> leaf_term(int kind, const Tree& F, const Node& ml, const Cache<T>& C, const T* vel, const T* fvel,
                            const AlignParams& P, bool stats_mode, int forced_match = -1, int forced_status = -1) {
  LeafRes<T> r;
  for (int i = 0; i < 18; ++i) r.J[i] = T(0);
  V3<T> m = nmean<T>(ml), nrm = ndir<T>(ml);
  V3<T> mw = m, nw = nrm;
  T dt = (T)ml.dts_mean;
  if (kind != KIND_ICP) warp_leaf(vel, dt, m, nrm, mw, nw);
  V3<T> p_mif = apply_iso(C.Xmf, mw);
  const bool forced = forced_status >= 0;
  int idx = forced ? forced_match : descend(F, p_mif);
  r.match = idx;
  if (forced && forced_status != ST_INLIER && forced_status != ST_OUTLIER) { r.status = forced_status; return r; }
  if (idx < 0) { r.status = ST_BAD; return r; }
  const Node& fl = F.nodes[idx];
  V3<T> pf = nmean<T>(fl), nf = ndir<T>(fl);
  V3<T> p_moving = apply_iso(C.Xm, mw);
  V3<T> n_moving = apply_rot(C.Xm, nw);
  V3<T> p_fixed = apply_iso(C.Xf, pf);
  V3<T> n_fixed = apply_rot(C.Xf, nf);
  // ICP_3D_Traits::errorAndJacobian
  if (!forced && dot3(n_fixed, n_moving) < (T)P.min_normal_cos) { r.status = ST_ERR_NORMAL; return r; }
  V3<T> ns = vadd(n_moving, n_fixed);
  T e = dot3(vsub(p_moving, p_fixed), ns);
  if (!forced && std::fabs(e) > (T)P.max_error) { r.status = ST_ERR_FN; return r; }
  V3<T> jr = vadd(cross(p_moving, n_fixed), cross(p_fixed, n_moving));
  for (int i = 0; i < 3; ++i) { r.J[i] = ns[i]; r.J[3 + i] = jr[i]; }
  if (kind != KIND_ICP) {
    T e_vel;
    err_jac_vel_A(e_vel, r.J + 6, C.Xm, m, nrm, p_fixed, n_fixed, vel, dt);
  }
  T chi2 = e * e;
  T kt = (T)P.kernel_threshold;
  T gamma;
  if (kind == KIND_CT_DUAL) {
    gamma = stats_mode ? T(0) : T(1);
    if (chi2 > kt) { r.status = ST_OUTLIER; gamma = std::sqrt(kt / chi2); }
    else r.status = ST_INLIER;
    T e_vel_b;
    T dtb = (T)fl.dts_mean;
    err_jac_vel_B(e_vel_b, r.J + 12, C.Xf, p_moving, n_moving, pf, nf, fvel, dtb);
  } else {
    gamma = T(1);
    if (chi2 > kt) { r.status = ST_OUTLIER; gamma = stats_mode ? T(0) : std::sqrt(kt / chi2); }
    else r.status = ST_INLIER;
  }
  r.e = e;
  r.chi2 = chi2;
  r.gamma = gamma;
  return r;
}

static inline int kind_dim(int kind) { return kind == KIND_ICP ? 6 : (kind == KIND_CT ? 12 : 18); }
static inline int packed_dim(int D) { return D * (D + 1) / 2 + D; }

// Packed item: upper triangle (r <= c, row-major) of gamma*J^T J, then gamma*J^T e.
template <class T> static void pack_item(const LeafRes<T>& r, int D, T* out) {
  int k = 0;
  for (int a = 0; a < D; ++a)
    for (int b = a; b < D; ++b) out[k++] = r.J[a] * r.J[b] * r.gamma;
  for (int a = 0; a < D; ++a) out[k++] = r.J[a] * r.e * r.gamma;
}

template <class S> struct StatsAcc {
  int ni = 0, no = 0, nb = 0, nn = 0, nf = 0;
  S chi2 = 0, chi2k = 0;
};

// StableAdder_ over a vector of K scalars (batch 1024, 5 levels).
template <class S> struct StableVec {
  int K;
  std::vector<S> val[5];
  size_t cnt[5];
  StatsAcc<S> sval[5];
  explicit StableVec(int k) : K(k) {
    for (int i = 0; i < 5; ++i) { val[i].assign(K, S(0)); cnt[i] = 0; sval[i] = StatsAcc<S>(); }
  }
  void add(const S* v, const StatsAcc<S>& st) {
    std::vector<S> cur(v, v + K);
    StatsAcc<S> cs = st;
    int i = 0;
    while (i < 5) {
      for (int k = 0; k < K; ++k) val[i][k] = val[i][k] + cur[k];
      sval[i].ni += cs.ni; sval[i].no += cs.no; sval[i].nb += cs.nb; sval[i].nn += cs.nn; sval[i].nf += cs.nf;
      sval[i].chi2 = sval[i].chi2 + cs.chi2;
      sval[i].chi2k = sval[i].chi2k + cs.chi2k;
      ++cnt[i];
      if (cnt[i] < 1024) break;
      cur = val[i];
      cs = sval[i];
      val[i].assign(K, S(0));
      sval[i] = StatsAcc<S>();
      cnt[i] = 0;
      ++i;
    }
  }
  void sum(S* out, StatsAcc<S>& st) const {
    for (int k = 0; k < K; ++k) out[k] = S(0);
    st = StatsAcc<S>();
    for (int i = 0; i < 5; ++i) {
      for (int k = 0; k < K; ++k) out[k] = out[k] + val[i][k];
      st.ni += sval[i].ni; st.no += sval[i].no; st.nb += sval[i].nb; st.nn += sval[i].nn; st.nf += sval[i].nf;
      st.chi2 = st.chi2 + sval[i].chi2;
      st.chi2k = st.chi2k + sval[i].chi2k;
    }
  }
};

template <class T> static void leaf_stats(const LeafRes<T>& r, StatsAcc<T>& s) {
  s = StatsAcc<T>();
  switch (r.status) {
    case ST_INLIER: s.ni = 1; break;
    case ST_OUTLIER: s.no = 1; break;
    case ST_BAD: s.nb = 1; return;
    case ST_ERR_NORMAL: s.nn = 1; return;
    case ST_ERR_FN: s.nf = 1; return;
  }
  s.chi2 = r.chi2;
  s.chi2k = r.chi2 * r.gamma;
}

// ---------------------------------------------------------------------------
// The product's summation order (kd_slam2_b200/csrc/kds_align.cu: tile_body,
// k_linearize, job_tail), restated so that MODE_MIXED's H and b are bit-identical to
// the GPU's.  The moving leaves are cut into tiles of 128 (per fixed entry, in leaf
// order), a tile into 4 warps of 32 lanes (lane = leaf, missing leaves count as zero
// rows).  Per warp and packed entry (r, c): a float Kahan sum over the 32 lanes of
// (J_r * J_c) * gamma (c = D: J_r * e * gamma), then s - comp in double.  The warp
// sums of chi2 and gamma * chi2 (doubles) are the xor-butterfly over offsets 16..1.
// The tile partial is ((((0 + w0) + w1) + w2) + w3); the job's sum runs over its tiles
// in order into 4 interleaved accumulators, combined as (a0 + a1) + (a2 + a3).
constexpr int kTileLeaves = 128;
constexpr int kPartStride = 200;  // doubles per tile partial
constexpr int kPartStats = 192;   // 7 stats values: counts x5, chi2, chi2 kernelized

static void packed_rc(int D, int k, int& r, int& c) {
  int T = D * (D + 1) / 2;
  if (k >= T) { r = k - T; c = D; return; }
  int rr = 0, off = 0;
  while (off + (D - rr) <= k) { off += D - rr; ++rr; }
  r = rr;
  c = rr + (k - off);
}

static double butterfly32(const double* v) {
  double a[32], b[32];
  for (int l = 0; l < 32; ++l) a[l] = v[l];
  for (int off = 16; off > 0; off >>= 1) {
    for (int l = 0; l < 32; ++l) b[l] = a[l] + a[l ^ off];
    for (int l = 0; l < 32; ++l) a[l] = b[l];
  }
  return a[0];
}

// Appends one partial per tile of Mv's leaves against F.
static void gpu_tile_partials(int kind, const Tree& F, const Tree& Mv, const Cache<float>& C, const float* vel,
                              const float* fvel, const AlignParams& P, bool stats_mode, std::vector<double>& parts,
                              int32_t* match_out, int32_t* status_out, int32_t* rec_match, int32_t* rec_status) {
  const int D = kind_dim(kind);
  const int K = packed_dim(D);
  const size_t n = Mv.leaves.size();
  for (size_t b0 = 0; b0 < n; b0 += kTileLeaves) {
    double wp[4][kPartStride];
    for (int w = 0; w < 4; ++w) {
      float rows[32][20];
      double chi2[32], chi2k[32];
      int cnt[5] = {0, 0, 0, 0, 0};
      for (int l = 0; l < 32; ++l) {
        const size_t i = b0 + (size_t)w * 32 + l;
        bool contrib = false;
        LeafRes<float> r;
        if (i < n) {
          const Node& ml = Mv.nodes[Mv.leaves[i]];
          r = leaf_term(kind, F, ml, C, vel, fvel, P, stats_mode);
          if (match_out) { match_out[i] = r.match; status_out[i] = r.status; }
          if (rec_match) { rec_match[i] = r.match; rec_status[i] = r.status; }
          contrib = r.status == ST_INLIER || r.status == ST_OUTLIER;
          cnt[r.status] += 1;
        }
        for (int k = 0; k < D; ++k) rows[l][k] = contrib ? r.J[k] : 0.f;
        rows[l][D] = contrib ? r.e : 0.f;
        rows[l][D + 1] = contrib ? r.gamma : 0.f;
        chi2[l] = contrib ? (double)(r.e * r.e) : 0.0;
        chi2k[l] = contrib ? (double)((r.e * r.e) * r.gamma) : 0.0;
      }
      for (int k = 0; k < K; ++k) {
        int rr, cc;
        packed_rc(D, k, rr, cc);
        float s = 0.f, comp = 0.f;
        for (int l = 0; l < 32; ++l) {
          float val = (rows[l][rr] * rows[l][cc]) * rows[l][D + 1];
          float y = val - comp;
          float t = s + y;
          comp = (t - s) - y;
          s = t;
        }
        wp[w][k] = (double)s - (double)comp;
      }
      for (int q = 0; q < 5; ++q) wp[w][kPartStats + q] = (double)cnt[q];
      wp[w][kPartStats + 5] = butterfly32(chi2);
      wp[w][kPartStats + 6] = butterfly32(chi2k);
    }
    const size_t o = parts.size();
    parts.resize(o + kPartStride, 0.0);
    for (int k = 0; k < kPartStride; ++k) {
      if ((k >= K && k < kPartStats) || k >= kPartStats + 7) continue;
      double acc = 0.0;
      for (int w = 0; w < 4; ++w) acc += wp[w][k];
      parts[o + k] = acc;
    }
  }
}

// The job's sum of its tile partials (job_tail): 4 interleaved accumulators in tile order.
static void gpu_reduce_tiles(const std::vector<double>& parts, double* red) {
  const size_t nt = parts.size() / kPartStride;
  for (int k = 0; k < kPartStride; ++k) {
    double a4[4] = {0.0, 0.0, 0.0, 0.0};
    size_t t = 0;
    for (; t + 4 <= nt; t += 4)
      for (int u = 0; u < 4; ++u) a4[u] += parts[(t + u) * kPartStride + k];
    for (; t < nt; ++t) a4[0] += parts[t * kPartStride + k];
    red[k] = (a4[0] + a4[1]) + (a4[2] + a4[3]);
  }
}

// One linearization over all moving leaves against one fixed tree.
// LeafT: per-leaf arithmetic; SumT: accumulation type.
template <class LeafT, class SumT>
static void linearize(int kind, const Tree& F, const Tree& Mv, const Cache<LeafT>& C, const LeafT* vel,
                      const LeafT* fvel, const AlignParams& P, bool stats_mode, bool stable_adder, int num_threads,
                      SumT* Hb_out /* packed K */, StatsAcc<SumT>& st_out, int32_t* match_out, int32_t* status_out) {
  const int D = kind_dim(kind);
  const int K = packed_dim(D);
  const size_t n = Mv.leaves.size();
  auto chunk = [&](size_t i0, size_t i1, std::vector<SumT>& acc, StatsAcc<SumT>& st) {
    acc.assign(K, SumT(0));
    st = StatsAcc<SumT>();
    std::vector<LeafT> item(K);
    if (stable_adder) {
      StableVec<SumT> sa(K);
      std::vector<SumT> itemS(K);
      for (size_t i = i0; i < i1; ++i) {
        const Node& ml = Mv.nodes[Mv.leaves[i]];
        LeafRes<LeafT> r = leaf_term(kind, F, ml, C, vel, fvel, P, stats_mode);
        if (match_out) { match_out[i] = r.match; status_out[i] = r.status; }
        StatsAcc<LeafT> s;
        leaf_stats(r, s);
        bool contributes = (r.status == ST_INLIER || r.status == ST_OUTLIER);
        for (int k = 0; k < K; ++k) item[k] = LeafT(0);
        if (contributes) pack_item(r, D, item.data());
        for (int k = 0; k < K; ++k) itemS[k] = (SumT)item[k];
        StatsAcc<SumT> sS;
        sS.ni = s.ni; sS.no = s.no; sS.nb = s.nb; sS.nn = s.nn; sS.nf = s.nf;
        sS.chi2 = (SumT)s.chi2; sS.chi2k = (SumT)s.chi2k;
        sa.add(itemS.data(), sS);
      }
      sa.sum(acc.data(), st);
    } else {
      for (size_t i = i0; i < i1; ++i) {
        const Node& ml = Mv.nodes[Mv.leaves[i]];
        LeafRes<LeafT> r = leaf_term(kind, F, ml, C, vel, fvel, P, stats_mode);
        if (match_out) { match_out[i] = r.match; status_out[i] = r.status; }
        StatsAcc<LeafT> s;
        leaf_stats(r, s);
        st.ni += s.ni; st.no += s.no; st.nb += s.nb; st.nn += s.nn; st.nf += s.nf;
        st.chi2 += (SumT)s.chi2;
        st.chi2k += (SumT)s.chi2k;
        if (r.status == ST_INLIER || r.status == ST_OUTLIER) {
          pack_item(r, D, item.data());
          for (int k = 0; k < K; ++k) acc[k] += (SumT)item[k];
        }
      }
    }
  };
  int nt = std::min(num_threads, 8);
  if (nt <= 1 || match_out) {
    std::vector<SumT> acc;
    chunk(0, n, acc, st_out);
    for (int k = 0; k < K; ++k) Hb_out[k] = acc[k];
    return;
  }
  // ICP_CPU_::_buildQuadraticForm chunking: nt contiguous chunks, remainder spread over the first.
  std::vector<std::future<std::pair<std::vector<SumT>, StatsAcc<SumT>>>> fut;
  size_t ch = n / nt, rem = n % nt, start = 0;
  for (int i = 0; i < nt; ++i) {
    size_t end = start + ch + ((size_t)i < rem ? 1 : 0);
    fut.push_back(std::async(std::launch::async, [&, start, end]() {
      std::vector<SumT> acc;
      StatsAcc<SumT> st;
      chunk(start, end, acc, st);
      return std::make_pair(acc, st);
    }));
    start = end;
  }
  for (int k = 0; k < K; ++k) Hb_out[k] = SumT(0);
  st_out = StatsAcc<SumT>();
  for (int i = 0; i < nt; ++i) {
    auto pr = fut[i].get();
    for (int k = 0; k < K; ++k) Hb_out[k] = Hb_out[k] + pr.first[k];
    st_out.ni += pr.second.ni; st_out.no += pr.second.no; st_out.nb += pr.second.nb;
    st_out.nn += pr.second.nn; st_out.nf += pr.second.nf;
    st_out.chi2 = st_out.chi2 + pr.second.chi2;
    st_out.chi2k = st_out.chi2k + pr.second.chi2k;
  }
}

template <class S> static void unpack_Hb(int D, const S* packed, S* H, S* b) {
  int k = 0;
  for (int a = 0; a < D; ++a)
    for (int c = a; c < D; ++c) { H[a * D + c] = packed[k]; H[c * D + a] = packed[k]; ++k; }
  for (int a = 0; a < D; ++a) b[a] = packed[k++];
}

template <class StateT, class LeafT> static Cache<LeafT> make_cache(const Iso<StateT>& X, const Iso<StateT>& Xf) {
  Cache<StateT> c;
  c.Xm = X;
  c.Xf = Xf;
  Iso<StateT> iXf = iso_inverse(Xf);
  c.Xmf = iso_mul(iXf, X);
  Cache<LeafT> o;
  o.Xm = iso_cast<LeafT>(c.Xm);
  o.Xf = iso_cast<LeafT>(c.Xf);
  o.Xmf = iso_cast<LeafT>(c.Xmf);
  return o;
}

template <class T> static T score_of(const OStats& s) {
  // ICPStats_::score (kd/icp/icp_stats_.h:32-35), float arithmetic
  int nl = s.num_inliers + s.num_outliers + s.num_bad + s.num_err_normal + s.num_err_fn;
  float ratio = nl ? (float)s.num_inliers / (float)nl : 0.f;
  return (T)(ratio / (s.chi2_kernelized / (float)s.num_inliers + 1e-6f));
}

// gpu_order (MODE_MIXED): the product's summation order, Cholesky and canonical expmap,
// so that every iteration is bit-identical to the GPU's.  rec (nullable) receives the
// correspondences and status of every iteration (iteration-major, fixed entries in
// order, leaves in order) for the FP64 replay.
struct Record {
  std::vector<int32_t> match, status;
};

template <class StateT, class LeafT, class SumT>
static int run_align(int kind, const std::vector<const Tree*>& fixed, const std::vector<Iso<double>>& fixed_X,
                     const Tree& Mv, const AlignParams& P, const OPrior* prior, double* X12, double* v6,
                     const double* fv6, int stats_mode, bool stable_adder, int num_threads, OResult* out,
                     bool gpu_order = false, Record* rec = nullptr) {
  constexpr bool kMixed = std::is_same<StateT, double>::value && std::is_same<LeafT, float>::value &&
                          std::is_same<SumT, double>::value;
  const int D = (kind == KIND_ICP) ? 6 : 12;
  const int K = packed_dim(D);
  Iso<StateT> X = iso_from12<StateT>(X12);
  StateT v[6];
  for (int i = 0; i < 6; ++i) v[i] = (StateT)(kind == KIND_ICP ? 0.0 : v6[i]);
  LeafT fvl[6];
  for (int i = 0; i < 6; ++i) fvl[i] = (LeafT)(fv6 ? fv6[i] : 0.0);
  int max_iter = stats_mode ? 1 : P.max_iterations;
  double prev_score = 0.0;
  int ret = P.max_iterations;
  bool done = false;
  std::vector<SumT> Hb(K), acc(K);
  out->iterations = 0;
  for (int it = 0; it < max_iter && !done; ++it) {
    LeafT vl[6];
    for (int i = 0; i < 6; ++i) vl[i] = (LeafT)v[i];
    for (int k = 0; k < K; ++k) Hb[k] = SumT(0);
    StatsAcc<SumT> st;
    bool done_sum = false;
    if constexpr (kMixed) {
      if (gpu_order) {
        std::vector<double> parts;
        const size_t nl = Mv.leaves.size();
        size_t r0 = 0;
        if (rec) {
          r0 = rec->match.size();
          rec->match.resize(r0 + nl * fixed.size());
          rec->status.resize(r0 + nl * fixed.size());
        }
        for (size_t f = 0; f < fixed.size(); ++f) {
          Iso<StateT> Xf = iso_cast<StateT>(fixed_X[f]);
          Cache<LeafT> C = make_cache<StateT, LeafT>(X, Xf);
          gpu_tile_partials(kind, *fixed[f], Mv, C, vl, fvl, P, stats_mode != 0, parts, nullptr, nullptr,
                            rec ? rec->match.data() + r0 + f * nl : nullptr,
                            rec ? rec->status.data() + r0 + f * nl : nullptr);
        }
        double red[kPartStride];
        gpu_reduce_tiles(parts, red);
        for (int k = 0; k < K; ++k) Hb[k] = red[k];
        st.ni = (int)red[kPartStats + 0];
        st.no = (int)red[kPartStats + 1];
        st.nb = (int)red[kPartStats + 2];
        st.nn = (int)red[kPartStats + 3];
        st.nf = (int)red[kPartStats + 4];
        st.chi2 = red[kPartStats + 5];
        st.chi2k = red[kPartStats + 6];
        done_sum = true;
      }
    }
    for (size_t f = 0; f < fixed.size() && !done_sum; ++f) {
      Iso<StateT> Xf = iso_cast<StateT>(fixed_X[f]);
      Cache<LeafT> C = make_cache<StateT, LeafT>(X, Xf);
      StatsAcc<SumT> s1;
      linearize<LeafT, SumT>(kind, *fixed[f], Mv, C, vl, fvl, P, stats_mode != 0, stable_adder, num_threads,
                             acc.data(), s1, nullptr, nullptr);
      for (int k = 0; k < K; ++k) Hb[k] = Hb[k] + acc[k];
      st.ni += s1.ni; st.no += s1.no; st.nb += s1.nb; st.nn += s1.nn; st.nf += s1.nf;
      st.chi2 = st.chi2 + s1.chi2;
      st.chi2k = st.chi2k + s1.chi2k;
    }
    StateT H[144], b[12];
    {
      SumT Hs[144], bs[12];
      unpack_Hb(D, Hb.data(), Hs, bs);
      for (int i = 0; i < D * D; ++i) H[i] = (StateT)Hs[i];
      for (int i = 0; i < D; ++i) b[i] = (StateT)bs[i];
    }
    // pose prior (pose block only)
    if (prior && prior->enabled) {
      Iso<StateT> Xr = iso_from12<StateT>(prior->X_ref), Z = iso_from12<StateT>(prior->Z);
      Iso<StateT> ZXi = iso_inverse(iso_mul(Xr, Z));
      StateT e[6], J[6][6];
      pose_to_pose_error(ZXi, X, e);
      dpose_to_pose_error(ZXi, X, J);
      StateT Om[6][6];
      for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Om[i][j] = (StateT)prior->info[i * 6 + j];
      StateT OJ[6][6];
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
          StateT a = 0;
          for (int k = 0; k < 6; ++k) a += Om[i][k] * J[k][j];
          OJ[i][j] = a;
        }
      for (int i = 0; i < 6; ++i) {
        for (int j = 0; j < 6; ++j) {
          StateT a = 0;
          for (int k = 0; k < 6; ++k) a += J[k][i] * OJ[k][j];
          H[i * D + j] += a;
        }
        StateT bb = 0;
        for (int k = 0; k < 6; ++k) {
          StateT oe = 0;
          for (int l = 0; l < 6; ++l) oe += Om[k][l] * e[l];
          bb += J[k][i] * oe;
        }
        b[i] += bb;
      }
    }
    OStats& S = out->log[it < 64 ? it : 63];
    S.num_inliers = st.ni; S.num_outliers = st.no; S.num_bad = st.nb;
    S.num_err_normal = st.nn; S.num_err_fn = st.nf;
    S.chi2 = (float)st.chi2;
    S.chi2_kernelized = (float)st.chi2k;
    S.pert_pose_norm = 0.f;
    S.pert_vel_norm = 0.f;
    for (int i = 0; i < D * D; ++i) out->H[i] = (double)H[i];
    for (int i = 0; i < D; ++i) out->b[i] = (double)b[i];
    out->iterations = it + 1;
    if (st.ni + st.no < P.min_good_measurements) {
      out->stats = S;
      ret = -it;
      done = true;
      break;
    }
    StateT A[144], rhs[12], dx[12];
    for (int i = 0; i < D * D; ++i) A[i] = H[i];
    for (int i = 0; i < D; ++i) {
      A[i * D + i] += (i < 6) ? (StateT)P.damping : (StateT)P.velocity_damping;
      rhs[i] = -b[i];
    }
    bool solved = false;
    if constexpr (kMixed) {
      if (gpu_order) {
        chol_solve_cols(D, A, rhs, dx);
        solved = true;
      }
    }
    if (!solved) ldlt_solve<StateT>(D, A, rhs, dx);
    for (int i = 0; i < D; ++i) out->dx[i] = (double)dx[i];
    StateT pp = 0, pv = 0;
    for (int i = 0; i < 6; ++i) pp += dx[i] * dx[i];
    S.pert_pose_norm = (float)std::sqrt(pp);
    if (D == 12) {
      for (int i = 6; i < 12; ++i) pv += dx[i] * dx[i];
      S.pert_vel_norm = (float)std::sqrt(pv);
    }
    out->stats = S;
    if (!stats_mode) {
      Iso<StateT> dX;
      bool canon = false;
      if constexpr (kMixed) {
        if (gpu_order) {
          dX = expmap_canon(dx);
          canon = true;
        }
      }
      if (!canon) dX = expmap<StateT>(dx);
      X = iso_mul(dX, X);
      if (D == 12)
        for (int i = 0; i < 6; ++i) v[i] += dx[6 + i];
    }
    if (P.term_crit) {
      float sc = score_of<float>(S);
      if (it > 0) {
        bool pert_ok = S.pert_pose_norm < P.d_pert;
        float dsc = sc - (float)prev_score;
        bool score_ok = (dsc > 0) && ((double)dsc / ((double)(float)prev_score + 1e-6) < (double)P.d_score);
        if (pert_ok && score_ok) { ret = it; done = true; }
      }
      prev_score = sc;
    }
  }
  iso_to12(X, X12);
  if (kind != KIND_ICP)
    for (int i = 0; i < 6; ++i) v6[i] = (double)v[i];
  out->ret = ret;
  return ret;
}

int align(int kind, int mode, const std::vector<const Tree*>& fixed, const std::vector<Iso<double>>& fixed_X,
          const Tree& moving, const AlignParams& P, const OPrior* prior, double* X12, double* v6, const double* fv6,
          int stats_mode, int num_threads, OResult* out) {
  std::memset(out, 0, sizeof(OResult));
  if (mode == MODE_REF32)
    return run_align<float, float, float>(kind, fixed, fixed_X, moving, P, prior, X12, v6, fv6, stats_mode, true,
                                          num_threads, out);
  if (mode == MODE_MIXED)
    return run_align<double, float, double>(kind, fixed, fixed_X, moving, P, prior, X12, v6, fv6, stats_mode, false,
                                            1, out, true);
  return run_align<double, double, double>(kind, fixed, fixed_X, moving, P, prior, X12, v6, fv6, stats_mode, false,
                                           1, out);
}

// One linearization at explicit float caches: per-leaf matches and status plus H,b.
void linearize_at(int kind, const Tree& F, const Tree& Mv, const float* caches36, const float* v6, const float* fv6,
                  const AlignParams& P, int stats_mode, int32_t* match_out, int32_t* status_out, double* H_out,
                  double* b_out, OStats* st_out) {
  Cache<float> C;
  C.Xm = iso_from12<float>(caches36);
  C.Xf = iso_from12<float>(caches36 + 12);
  C.Xmf = iso_from12<float>(caches36 + 24);
  const int D = kind_dim(kind);
  float vz[6] = {0, 0, 0, 0, 0, 0};
  std::vector<double> parts;
  gpu_tile_partials(kind, F, Mv, C, v6 ? v6 : vz, fv6 ? fv6 : vz, P, stats_mode != 0, parts, match_out, status_out,
                    nullptr, nullptr);
  double red[kPartStride];
  gpu_reduce_tiles(parts, red);
  StatsAcc<double> st;
  st.ni = (int)red[kPartStats + 0];
  st.no = (int)red[kPartStats + 1];
  st.nb = (int)red[kPartStats + 2];
  st.nn = (int)red[kPartStats + 3];
  st.nf = (int)red[kPartStats + 4];
  st.chi2 = red[kPartStats + 5];
  st.chi2k = red[kPartStats + 6];
  unpack_Hb(D, red, H_out, b_out);
  st_out->num_inliers = st.ni; st_out->num_outliers = st.no; st_out->num_bad = st.nb;
  st_out->num_err_normal = st.nn; st_out->num_err_fn = st.nf;
  st_out->chi2 = (float)st.chi2;
  st_out->chi2_kernelized = (float)st.chi2k;
  st_out->pert_pose_norm = 0.f;
  st_out->pert_vel_norm = 0.f;
}

template void err_jac_vel_A<float>(float&, float*, const Iso<float>&, const V3<float>&, const V3<float>&,
                                   const V3<float>&, const V3<float>&, const float*, float);
template void err_jac_vel_B<float>(float&, float*, const Iso<float>&, const V3<float>&, const V3<float>&,
                                   const V3<float>&, const V3<float>&, const float*, float);
template void err_jac_vel_A<double>(double&, double*, const Iso<double>&, const V3<double>&, const V3<double>&,
                                    const V3<double>&, const V3<double>&, const double*, double);
template void err_jac_vel_B<double>(double&, double*, const Iso<double>&, const V3<double>&, const V3<double>&,
                                    const V3<double>&, const V3<double>&, const double*, double);


// CTICP_::poseHessian (kd/cticp/cticp_.h:169-177): the pose-only information matrix of
// a 12x12 CT-ICP H by the Schur complement over the velocity block,
// H_pp - H_pv (H_vv + 1e-9 I)^-1 H_pv^T, in FP64.  The inverse is Gauss-Jordan
// elimination with partial pivoting (Eigen's .inverse() of a 6x6 is partial-pivoting LU).
// Returns false when the velocity block is singular.
bool pose_hessian(const double* H12, double* out36) {
  double A[6][12];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      A[i][j] = H12[(6 + i) * 12 + 6 + j] + (i == j ? 1e-9 : 0.0);
      A[i][6 + j] = (i == j) ? 1.0 : 0.0;
    }
  for (int c = 0; c < 6; ++c) {
    int p = c;
    for (int r = c + 1; r < 6; ++r)
      if (std::fabs(A[r][c]) > std::fabs(A[p][c])) p = r;
    if (A[p][c] == 0.0) return false;
    if (p != c)
      for (int k = 0; k < 12; ++k) std::swap(A[p][k], A[c][k]);
    const double d = A[c][c];
    for (int k = 0; k < 12; ++k) A[c][k] = A[c][k] / d;
    for (int r = 0; r < 6; ++r) {
      if (r == c) continue;
      const double f = A[r][c];
      for (int k = 0; k < 12; ++k) A[r][k] = A[r][k] - f * A[c][k];
    }
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      double acc = 0.0;  // (H_pv Hvv^-1 H_pv^T)_ij
      for (int k = 0; k < 6; ++k) {
        double t = 0.0;
        for (int l = 0; l < 6; ++l) t += A[k][6 + l] * H12[j * 12 + 6 + l];
        acc += H12[i * 12 + 6 + k] * t;
      }
      out36[i * 6 + j] = H12[i * 12 + j] - acc;
    }
  return true;
}

// The float caches (Xm, Xf, Xmf) the product derives from FP64 poses at the start of
// every iteration, with its operation order (make_cache).
void product_caches(const double* X12, const double* Xf12, float* out36) {
  Cache<float> c = make_cache<double, float>(iso_from12<double>(X12), iso_from12<double>(Xf12));
  iso_to12(c.Xm, out36);
  iso_to12(c.Xf, out36 + 12);
  iso_to12(c.Xmf, out36 + 24);
}

// MODE_MIXED run that also returns every iteration's correspondences and status.
int align_recorded(int kind, const std::vector<const Tree*>& fixed, const std::vector<Iso<double>>& fixed_X,
                   const Tree& moving, const AlignParams& P, double* X12, double* v6, const double* fv6,
                   OResult* out, std::vector<int32_t>& match, std::vector<int32_t>& status) {
  std::memset(out, 0, sizeof(OResult));
  Record rec;
  int ret = run_align<double, float, double>(kind, fixed, fixed_X, moving, P, nullptr, X12, v6, fv6, 0, false, 1, out,
                                             true, &rec);
  match.swap(rec.match);
  status.swap(rec.status);
  return ret;
}

// FP64 replay of a recorded run: `iterations` Gauss-Newton steps in all-FP64 arithmetic
// (per-leaf terms, sums, LDL^T solve, expmap with libm sine/cosine), where iteration it
// uses the recorded fixed leaf of every moving leaf and lets exactly the recorded
// inliers and outliers contribute (the robust weight is recomputed in FP64 from the
// FP64 error).  The distance of its pose from the recorded run's is the arithmetic
// error of the FP32 per-leaf terms alone, with every branch held fixed.
void align_replay64(int kind, const std::vector<const Tree*>& fixed, const std::vector<Iso<double>>& fixed_X,
                    const Tree& Mv, const AlignParams& P, double* X12, double* v6, const double* fv6, int iterations,
                    const int32_t* match, const int32_t* status) {
  const int D = (kind == KIND_ICP) ? 6 : 12;
  const int K = packed_dim(D);
  Iso<double> X = iso_from12<double>(X12);
  double v[6], fv[6];
  for (int i = 0; i < 6; ++i) {
    v[i] = kind == KIND_ICP ? 0.0 : v6[i];
    fv[i] = fv6 ? fv6[i] : 0.0;
  }
  const size_t nl = Mv.leaves.size();
  std::vector<double> Hb(K), item(K);
  for (int it = 0; it < iterations; ++it) {
    for (int k = 0; k < K; ++k) Hb[k] = 0.0;
    for (size_t f = 0; f < fixed.size(); ++f) {
      Cache<double> C = make_cache<double, double>(X, fixed_X[f]);
      const size_t base = ((size_t)it * fixed.size() + f) * nl;
      for (size_t i = 0; i < nl; ++i) {
        const Node& ml = Mv.nodes[Mv.leaves[i]];
        LeafRes<double> r = leaf_term(kind, *fixed[f], ml, C, v, fv, P, false, match[base + i], status[base + i]);
        if (r.status != ST_INLIER && r.status != ST_OUTLIER) continue;
        const double kt = (double)P.kernel_threshold;
        r.gamma = r.chi2 > kt ? std::sqrt(kt / r.chi2) : 1.0;
        pack_item(r, D, item.data());
        for (int k = 0; k < K; ++k) Hb[k] += item[k];
      }
    }
    double H[144], b[12], A[144], rhs[12], dx[12];
    unpack_Hb(D, Hb.data(), H, b);
    for (int i = 0; i < D * D; ++i) A[i] = H[i];
    for (int i = 0; i < D; ++i) {
      A[i * D + i] += (i < 6) ? (double)P.damping : (double)P.velocity_damping;
      rhs[i] = -b[i];
    }
    ldlt_solve<double>(D, A, rhs, dx);
    X = iso_mul(expmap<double>(dx), X);
    if (D == 12)
      for (int i = 0; i < 6; ++i) v[i] += dx[6 + i];
  }
  iso_to12(X, X12);
  if (kind != KIND_ICP)
    for (int i = 0; i < 6; ++i) v6[i] = v[i];
}

}  // namespace orc
