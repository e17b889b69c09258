// CPU oracle: canonical surfel KD-tree build -- TEST INFRASTRUCTURE ONLY.
//
// Restates TreeGenerator_::makeTree (kd/tree/tree_generator_impl_.h:7-19):
//   recursive build with FlatLeafPolicy_  (kd/tree/flat_leaf_policy_.h:52-108,
//   kd/tree/count_leaf_policy_.h:27-43, kd/tree/label_policy_base_impl_.h:12-97),
//   split by Node_::whichSide            (kd/tree/node_.h:53-56),
//   prune by IsGoodLeafPredicate_        (kd/tree/tree_predicates_.h:7-30,
//                                          kd/tree/tree_cpu_.h:172-232),
//   breadth-first relabel                (kd/tree/tree_cpu_impl_.h:48-74,136-158).
//
// Canonical arithmetic (parity unpinned against the reference, pinned between this
// oracle and the CUDA build):
//  * Moment sums [xx,xy,xz,yy,yz,zz,x,y,z,dt,dt^2] are accumulated as 128-bit
//    fixed point with 2^-64 resolution.  Each float product is exact in double and is
//    floored onto the grid, so the sums are independent of summation order (the
//    reference sums in float with StableAdder_, kd/utils/stable_adder_.h:21-74).
//  * Mean, covariance and eigen decomposition are FP64; the eigensolver is cyclic
//    Jacobi (Golub & Van Loan, sec. 8.5) with a fixed sweep count, which uses only
//    IEEE-exact + - * / sqrt; a rotation is skipped (off-diagonal set to zero) when
//    |a_pq| <= 1e-18 (|a_pp| + |a_qq|), and the sweeps stop once all off-diagonals are
//    zero.  The reference uses Eigen's computeDirect in float.
//  * Partitions are stable (left points keep their order, then right points); the
//    reference swaps with the range end (kd/tree/node_impl_.h:12-26).  Leaf membership
//    does not depend on this order because the sums are order independent.
//  * Nodes are created level by level, left child before right, which is the BFS
//    order that prune()+breadthFirstPermutation() produce.
//  * A node at level max_level-1 is not split further (the reference recurses
//    without bound and overflows the stack on a degenerate split).
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <future>
#include <limits>
#include <vector>

#include "orc_math.hpp"
#include "orc_tree.hpp"

namespace orc {

typedef __int128 i128;

// floor(v * 2^64) exactly, from the integer mantissa and exponent of v (|v| < 2^62).
// Splitting v into floor(v) and a fraction in double is not exact for small negative
// v (1 - |v| can need more than 53 bits), so the floor is formed with integer shifts.
static inline i128 fx_of(double v) {
  if (v == 0.0) return 0;
  int ex = 0;
  const double fr = std::frexp(std::fabs(v), &ex);   // |v| = fr * 2^ex, fr in [0.5, 1)
  const uint64_t m = (uint64_t)std::ldexp(fr, 53);   // exact 53-bit integer
  const int sh = ex - 53 + 64;                       // |v| * 2^64 = m * 2^sh
  i128 mag = 0;
  bool rem = false;
  if (sh >= 0) {
    mag = (i128)m << sh;
  } else if (sh > -64) {
    mag = (i128)(m >> (-sh));
    rem = (m & ((1ull << (-sh)) - 1ull)) != 0ull;
  } else {
    rem = true;
  }
  if (v < 0.0) return -mag - (rem ? 1 : 0);
  return mag;
}
void fx_floor_parts(double v, int64_t* hi, uint64_t* lo) {
  const i128 q = fx_of(v);
  *hi = (int64_t)(q >> 64);
  *lo = (uint64_t)q;
}

static inline double fx_to_d(i128 q) {
  int64_t hi = (int64_t)(q >> 64);
  uint64_t lo = (uint64_t)q;
  return ((double)hi * 0x1p64 + (double)lo) * 0x1p-64;
}

struct Moments {
  i128 s[11];
};

static void moments_of(const float* xyz, const double* st, const int64_t* order, int64_t b, int64_t e,
                       double ts_start, Moments& M) {
  for (int k = 0; k < 11; ++k) M.s[k] = 0;
  for (int64_t i = b; i < e; ++i) {
    int64_t p = order[i];
    double x = xyz[3 * p], y = xyz[3 * p + 1], z = xyz[3 * p + 2];
    M.s[0] += fx_of(x * x);
    M.s[1] += fx_of(x * y);
    M.s[2] += fx_of(x * z);
    M.s[3] += fx_of(y * y);
    M.s[4] += fx_of(y * z);
    M.s[5] += fx_of(z * z);
    M.s[6] += fx_of(x);
    M.s[7] += fx_of(y);
    M.s[8] += fx_of(z);
    double dt = st ? (st[p] - ts_start) : 0.0;
    M.s[9] += fx_of(dt);
    M.s[10] += fx_of(dt * dt);
  }
}

// Cyclic Jacobi for a symmetric 3x3; eigenvalues ascending, eigenvectors as columns.
void jacobi3(const double Ain[3][3], double ev[3], double V[3][3]) {
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) { a[i][j] = Ain[i][j]; V[i][j] = (i == j) ? 1.0 : 0.0; }
  for (int sweep = 0; sweep < 8; ++sweep) {
    if (a[0][1] == 0.0 && a[0][2] == 0.0 && a[1][2] == 0.0) break;
    for (int pq = 0; pq < 3; ++pq) {
      int p = (pq == 2) ? 1 : 0;
      int q = (pq == 0) ? 1 : 2;
      int r = 3 - p - q;
      double apq = a[p][q];
      // negligible off-diagonal: set to zero and skip the rotation
      if (std::fabs(apq) <= 1e-18 * (std::fabs(a[p][p]) + std::fabs(a[q][q]))) {
        a[p][q] = 0.0;
        a[q][p] = 0.0;
        continue;
      }
      double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
      double t = 1.0 / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
      if (theta < 0.0) t = -t;
      double c = 1.0 / std::sqrt(t * t + 1.0);
      double s = t * c;
      double arp = a[r][p], arq = a[r][q];
      a[p][p] = a[p][p] - t * apq;
      a[q][q] = a[q][q] + t * apq;
      a[p][q] = 0.0;
      a[q][p] = 0.0;
      double nrp = c * arp - s * arq;
      double nrq = s * arp + c * arq;
      a[r][p] = nrp; a[p][r] = nrp;
      a[r][q] = nrq; a[q][r] = nrq;
      for (int k = 0; k < 3; ++k) {
        double vkp = V[k][p], vkq = V[k][q];
        V[k][p] = c * vkp - s * vkq;
        V[k][q] = s * vkp + c * vkq;
      }
    }
  }
  double d[3] = {a[0][0], a[1][1], a[2][2]};
  int idx[3] = {0, 1, 2};
  // stable insertion sort, ascending
  for (int i = 1; i < 3; ++i) {
    int k = idx[i];
    int j = i - 1;
    while (j >= 0 && d[k] < d[idx[j]]) { idx[j + 1] = idx[j]; --j; }
    idx[j + 1] = k;
  }
  double Vs[3][3];
  for (int c2 = 0; c2 < 3; ++c2) {
    ev[c2] = d[idx[c2]];
    for (int r2 = 0; r2 < 3; ++r2) Vs[r2][c2] = V[r2][idx[c2]];
  }
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) V[i][j] = Vs[i][j];
}

static inline double ddot3(const double* a, const double* b) {
  double p0 = a[0] * b[0], p1 = a[1] * b[1], p2 = a[2] * b[2];
  return p0 + (p1 + p2);
}

struct Meta {
  bool is_node = false, is_leaf = false, is_bad = true, is_flat = false, has_prop = false;
  double prop[3] = {0, 0, 0};
};

// fillMetadata of FlatLeafPolicy_ (with CountLeafPolicy_ and LabelPolicyBase_ below it).
// root (nullable): the root's frame, [0..2] eigenvalues, [3..11] eigenvectors column-major
// (fillMetadata's reorientation of columns 0 and 2, label_policy_base_impl_.h:89-95, then
// column 0 negated for a negative determinant, tree_cpu_.h:79-82), [12..14] mean.
static void fill_metadata(const Moments& M, int64_t n, bool has_parent, bool parent_has_prop,
                          const double* parent_prop, int level, const TreeParams& P, Node& node,
                          Meta& meta, double* root) {
  meta = Meta();
  for (int i = 0; i < 3; ++i) { node.mean[i] = 0.f; node.dir[i] = 0.f; }
  node.dts_mean = 0.0;
  node.dts_cov = 0.0;
  double mean_d[3] = {0, 0, 0};
  double e0[3] = {0, 0, 0}, e2[3] = {0, 0, 0};
  double lam[3] = {0, 0, 0};
  bool is_bad = true;
  if (n > 0) {
    double dn = (double)n;
    double Sd[11];
    for (int k = 0; k < 11; ++k) Sd[k] = fx_to_d(M.s[k]);
    node.dts_mean = Sd[9] / dn;
    node.dts_cov = Sd[10] / dn - node.dts_mean * node.dts_mean;
    for (int i = 0; i < 3; ++i) mean_d[i] = Sd[6 + i] / dn;
    for (int i = 0; i < 3; ++i) node.mean[i] = (float)mean_d[i];
    if (n >= 3) {
      double C[3][3];
      C[0][0] = Sd[0] / dn - mean_d[0] * mean_d[0];
      C[0][1] = Sd[1] / dn - mean_d[0] * mean_d[1];
      C[0][2] = Sd[2] / dn - mean_d[0] * mean_d[2];
      C[1][1] = Sd[3] / dn - mean_d[1] * mean_d[1];
      C[1][2] = Sd[4] / dn - mean_d[1] * mean_d[2];
      C[2][2] = Sd[5] / dn - mean_d[2] * mean_d[2];
      C[1][0] = C[0][1];
      C[2][0] = C[0][2];
      C[2][1] = C[1][2];
      double V[3][3];
      jacobi3(C, lam, V);
      for (int i = 0; i < 3; ++i) { e0[i] = V[i][0]; e2[i] = V[i][2]; }
      if (ddot3(mean_d, e0) > 0.0) for (int i = 0; i < 3; ++i) e0[i] = -e0[i];
      if (ddot3(mean_d, e2) > 0.0) for (int i = 0; i < 3; ++i) e2[i] = -e2[i];
      is_bad = false;
      if (root) {
        const double e1[3] = {V[0][1], V[1][1], V[2][1]};
        const double cx = e1[1] * e2[2] - e1[2] * e2[1];
        const double cy = e1[2] * e2[0] - e1[0] * e2[2];
        const double cz = e1[0] * e2[1] - e1[1] * e2[0];
        const double det = e0[0] * cx + (e0[1] * cy + e0[2] * cz);
        const double sg = det < 0.0 ? -1.0 : 1.0;
        for (int i = 0; i < 3; ++i) {
          root[i] = lam[i];
          root[3 + i] = sg * e0[i];
          root[6 + i] = e1[i];
          root[9 + i] = e2[i];
        }
      }
    }
  }
  if (root) {
    if (is_bad)
      for (int i = 0; i < 12; ++i) root[i] = 0.0;
    for (int i = 0; i < 3; ++i) root[12 + i] = mean_d[i];
  }
  // CountLeafPolicy_
  bool is_node = false, is_leaf = false;
  if (is_bad) {
    is_leaf = true;
  } else if ((float)n > (float)P.leaf_max_points) {
    is_node = true;
    for (int i = 0; i < 3; ++i) node.dir[i] = (float)e2[i];
  } else {
    is_leaf = true;
    for (int i = 0; i < 3; ++i) node.dir[i] = (float)e0[i];
  }
  // FlatLeafPolicy_
  bool has_prop = false;
  double prop[3] = {0, 0, 0};
  if (has_parent && P.propagate_normal) {
    has_prop = parent_has_prop;
    for (int i = 0; i < 3; ++i) prop[i] = parent_prop[i];
  }
  auto propagate = [&]() -> bool {
    is_leaf = true;
    if (has_prop) {
      double d[3] = {prop[0], prop[1], prop[2]};
      if (ddot3(mean_d, d) > 0.0) for (int i = 0; i < 3; ++i) d[i] = -d[i];
      for (int i = 0; i < 3; ++i) node.dir[i] = (float)d[i];
      return true;
    }
    return false;
  };
  bool is_flat = false;
  if (is_bad || (float)n < (float)P.leaf_min_points) {
    is_bad = !propagate();
  } else {
    double eigenratio = lam[0] / lam[2];
    is_flat = eigenratio < (double)P.leaf_normal_eigenratio &&
              std::fabs(ddot3(mean_d, e0)) > (double)P.leaf_min_normal_incidence;
    if (is_flat) {
      has_prop = true;
      for (int i = 0; i < 3; ++i) prop[i] = e0[i];
    }
    if (!is_node) {
      double volume = lam[1] * lam[2];
      double density = (double)n / volume;
      if (density < (double)P.leaf_density) {
        is_leaf = false;
        is_node = true;
        is_bad = false;
        for (int i = 0; i < 3; ++i) node.dir[i] = (float)e2[i];
      } else if (is_leaf && is_flat) {
        for (int i = 0; i < 3; ++i) node.dir[i] = (float)e0[i];
      } else {
        is_bad = !propagate();
      }
    }
  }
  // Depth cap: a node that would split at the last level becomes a leaf.
  if (is_node && level >= P.max_level - 1) {
    is_node = false;
    is_leaf = true;
    if (is_flat) {
      for (int i = 0; i < 3; ++i) node.dir[i] = (float)e0[i];
    } else if (!propagate()) {
      for (int i = 0; i < 3; ++i) node.dir[i] = (float)e0[i];
    }
  }
  meta.is_node = is_node;
  meta.is_leaf = is_leaf;
  meta.is_bad = is_bad;
  meta.is_flat = is_flat;
  meta.has_prop = has_prop;
  for (int i = 0; i < 3; ++i) meta.prop[i] = prop[i];
}

// Node_::whichSide (kd/tree/node_.h:53-56) in float: dir . (q - mean) > 0
static inline bool which_side(const float* mean, const float* dir, const float* q) {
  float d0 = q[0] - mean[0], d1 = q[1] - mean[1], d2 = q[2] - mean[2];
  float p0 = dir[0] * d0, p1 = dir[1] * d1, p2 = dir[2] * d2;
  return (p0 + (p1 + p2)) > 0.0f;
}

// IsGoodLeafPredicate_ (kd/tree/tree_predicates_.h:18-29) in float.
static inline bool good_leaf(const Node& n, float incidence) {
  if (!(n.left < 0 && n.right < 0)) return false;
  float q0 = n.dir[0] * n.dir[0], q1 = n.dir[1] * n.dir[1], q2 = n.dir[2] * n.dir[2];
  if (!((q0 + (q1 + q2)) > 0.0f)) return false;
  float m0 = n.mean[0] * n.dir[0], m1 = n.mean[1] * n.dir[1], m2 = n.mean[2] * n.dir[2];
  float inc = m0 + (m1 + m2);
  return std::fabs(inc) > incidence;
}

Tree build_tree(const float* xyz, const double* st, int64_t n, const TreeParams& P) {
  Tree T;
  T.num_points = n;
  T.perm.resize(n);
  for (int64_t i = 0; i < n; ++i) T.perm[i] = i;
  T.ts_start = 0.0;
  if (st && n > 0) {
    double m = std::numeric_limits<double>::max();
    for (int64_t i = 0; i < n; ++i) m = std::min(m, st[i]);
    T.ts_start = m;
  }
  T.accepted = false;
  if (n < (int64_t)P.leaf_min_points || n == 0) return T;

  std::vector<Node> nodes;
  std::vector<int> levels;
  std::vector<char> par_has;
  std::vector<double> par_prop;  // 3 per node: propagated normal handed down by the parent
  std::vector<char> has_parent;
  nodes.reserve(2 * n + 2);
  Node root;
  root.start = 0;
  root.end = n;
  root.left = root.right = -1;
  nodes.push_back(root);
  levels.push_back(0);
  par_has.push_back(0);
  has_parent.push_back(0);
  par_prop.insert(par_prop.end(), {0.0, 0.0, 0.0});

  std::vector<int64_t> tmp(n);
  size_t lb = 0, le = 1;
  while (lb < le) {
    for (size_t i = lb; i < le; ++i) {
      Moments M;
      int64_t s = nodes[i].start, e = nodes[i].end;
      moments_of(xyz, st, T.perm.data(), s, e, T.ts_start, M);
      Meta meta;
      Node nd = nodes[i];
      double root[15];
      fill_metadata(M, e - s, has_parent[i], par_has[i], &par_prop[3 * i], levels[i], P, nd, meta,
                    i == 0 ? root : nullptr);
      if (i == 0) {
        for (int k = 0; k < 3; ++k) {
          T.root_eigenvalues[k] = (float)root[k];
          T.root_mean[k] = (float)root[12 + k];
        }
        for (int k = 0; k < 9; ++k) T.root_eigenvectors[k] = (float)root[3 + k];
      }
      nd.left = nd.right = -1;
      if (meta.is_node) {
        // stable partition of perm[s..e)
        int64_t nl = 0;
        for (int64_t k = s; k < e; ++k) {
          int64_t p = T.perm[k];
          if (which_side(nd.mean, nd.dir, xyz + 3 * p)) tmp[s + nl++] = p;
        }
        int64_t nr = 0;
        for (int64_t k = s; k < e; ++k) {
          int64_t p = T.perm[k];
          if (!which_side(nd.mean, nd.dir, xyz + 3 * p)) tmp[s + nl + nr++] = p;
        }
        for (int64_t k = s; k < e; ++k) T.perm[k] = tmp[k];
        int64_t mid = s + nl;
        int li = (int)nodes.size();
        nd.left = li;
        nd.right = li + 1;
        Node c;
        c.left = c.right = -1;
        c.start = s; c.end = mid;
        nodes.push_back(c);
        c.start = mid; c.end = e;
        nodes.push_back(c);
        for (int k = 0; k < 2; ++k) {
          levels.push_back(levels[i] + 1);
          par_has.push_back(meta.has_prop ? 1 : 0);
          has_parent.push_back(1);
          par_prop.insert(par_prop.end(), {meta.prop[0], meta.prop[1], meta.prop[2]});
        }
      }
      nodes[i] = nd;
    }
    lb = le;
    le = nodes.size();
  }

  // prune: bottom-up survival; children always have larger indices than parents.
  size_t nn = nodes.size();
  std::vector<char> alive(nn, 0);
  for (size_t ii = nn; ii-- > 0;) {
    const Node& nd = nodes[ii];
    if (nd.left < 0 && nd.right < 0) {
      alive[ii] = good_leaf(nd, P.prune_min_normal_incidence) ? 1 : 0;
    } else {
      bool a = (nd.left >= 0 && alive[nd.left]) || (nd.right >= 0 && alive[nd.right]);
      alive[ii] = a ? 1 : 0;
    }
  }
  std::vector<int> newidx(nn, -1);
  int cnt = 0;
  for (size_t ii = 0; ii < nn; ++ii)
    if (alive[ii]) newidx[ii] = cnt++;
  T.nodes.resize(cnt);
  T.levels.resize(cnt);
  for (size_t ii = 0; ii < nn; ++ii) {
    if (!alive[ii]) continue;
    Node nd = nodes[ii];
    nd.left = (nd.left >= 0 && alive[nd.left]) ? newidx[nd.left] : -1;
    nd.right = (nd.right >= 0 && alive[nd.right]) ? newidx[nd.right] : -1;
    T.nodes[newidx[ii]] = nd;
    T.levels[newidx[ii]] = levels[ii];
  }
  for (int i = 0; i < cnt; ++i)
    if (T.nodes[i].left < 0 && T.nodes[i].right < 0) T.leaves.push_back(i);
  T.num_unpruned = (int64_t)nn;
  T.accepted = (int64_t)T.leaves.size() >= (int64_t)P.tree_min_good_leaves;
  return T;
}

// ---------------------------------------------------------------------------
// The reference's own CPU build arithmetic, for the timed CPU baseline (not a parity
// definition: its float sums make it differ from the canonical build above in the last
// bits, which moves a split or a leaf decision now and then).  It restates:
//   Node_ constructor and splitRange       kd/tree/node_impl_.h:12-70 (swap partition,
//                                          std::async for both children while the
//                                          node's level < parallel_level >= 0)
//   LabelPolicyBase_::fillMetadata         kd/tree/label_policy_base_impl_.h:12-97
//                                          (float StableAdder_ over the packed
//                                          [xx..zz, x, y, z], double StableAdder_ over
//                                          (dt, dt^2), mean/cov in float)
//   SelfAdjointEigenSolver::computeDirect  a closed-form symmetric 3x3 eigen solve in
//                                          float: the trigonometric roots of the
//                                          characteristic polynomial (Smith 1961) and
//                                          eigenvectors as the longest cross product of
//                                          two rows of A - lambda I
//   CountLeafPolicy_ / FlatLeafPolicy_     as fill_metadata above, on the float values
// then the same prune and breadth-first relabel.
namespace {

struct RefPoint {
  float x, y, z;
  double t;
  int64_t id;
};

template <class T, int K> struct RefAdder {  // StableAdder_<T[K], 1024, 5>
  T acc[5][K];
  int cnt[5];
  RefAdder() {
    for (int l = 0; l < 5; ++l) {
      cnt[l] = 0;
      for (int k = 0; k < K; ++k) acc[l][k] = T(0);
    }
  }
  void add(const T* v) {
    T cur[K];
    for (int k = 0; k < K; ++k) cur[k] = v[k];
    for (int l = 0; l < 5; ++l) {
      for (int k = 0; k < K; ++k) acc[l][k] += cur[k];
      if (++cnt[l] < 1024) break;
      for (int k = 0; k < K; ++k) { cur[k] = acc[l][k]; acc[l][k] = T(0); }
      cnt[l] = 0;
    }
  }
  void sum(T* out) const {
    for (int k = 0; k < K; ++k) out[k] = T(0);
    for (int l = 0; l < 5; ++l)
      for (int k = 0; k < K; ++k) out[k] += acc[l][k];
  }
};

// eigenvalues ascending, eigenvectors as columns of V
void eig3_direct(const float A[3][3], float ev[3], float V[3][3]) {
  const float m = (A[0][0] + A[1][1] + A[2][2]) / 3.0f;
  float K[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) K[i][j] = A[i][j] - (i == j ? m : 0.0f);
  float p = 0.0f;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) p += K[i][j] * K[i][j];
  p = p / 6.0f;
  if (!(p > 1e-30f)) {
    for (int i = 0; i < 3; ++i) {
      ev[i] = m;
      for (int j = 0; j < 3; ++j) V[i][j] = i == j ? 1.0f : 0.0f;
    }
    return;
  }
  const float detK = K[0][0] * (K[1][1] * K[2][2] - K[1][2] * K[2][1]) -
                     K[0][1] * (K[1][0] * K[2][2] - K[1][2] * K[2][0]) +
                     K[0][2] * (K[1][0] * K[2][1] - K[1][1] * K[2][0]);
  const float sp = std::sqrt(p);
  float r = detK / (2.0f * p * sp);
  r = std::max(-1.0f, std::min(1.0f, r));
  const float phi = std::acos(r) / 3.0f;
  float l3 = m + 2.0f * sp * std::cos(phi);
  float l1 = m + 2.0f * sp * std::cos(phi + 2.0943951f);
  float l2 = 3.0f * m - l1 - l3;
  float lam[3] = {l1, l2, l3};
  std::sort(lam, lam + 3);
  for (int c = 0; c < 3; ++c) {
    float B[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) B[i][j] = A[i][j] - (i == j ? lam[c] : 0.0f);
    float best[3] = {0, 0, 0}, bn = -1.0f;
    for (int a = 0; a < 3; ++a) {
      const int b = (a + 1) % 3;
      const float cx = B[a][1] * B[b][2] - B[a][2] * B[b][1];
      const float cy = B[a][2] * B[b][0] - B[a][0] * B[b][2];
      const float cz = B[a][0] * B[b][1] - B[a][1] * B[b][0];
      const float nn = cx * cx + cy * cy + cz * cz;
      if (nn > bn) { bn = nn; best[0] = cx; best[1] = cy; best[2] = cz; }
    }
    const float inv = bn > 0.0f ? 1.0f / std::sqrt(bn) : 0.0f;
    for (int i = 0; i < 3; ++i) V[i][c] = bn > 0.0f ? best[i] * inv : (i == c ? 1.0f : 0.0f);
    ev[c] = lam[c];
  }
}

struct RefMeta {
  bool is_node = false, has_prop = false;
  float prop[3] = {0, 0, 0};
  int level = 0;
  double ts_start = 0.0;
};

struct RefBuild {
  RefPoint* pts;
  Node* nodes;
  int* levels;
  std::atomic<int>* idx;
  int cap;
  const TreeParams* P;
  int parallel_level;

  // fillMetadata + the leaf policies on the node's points; returns the node's metadata
  RefMeta fill(Node& node, const RefMeta* parent) const {
    RefMeta meta;
    meta.level = parent ? parent->level + 1 : 0;
    meta.ts_start = parent ? parent->ts_start : 0.0;
    const int64_t n = node.end - node.start;
    for (int i = 0; i < 3; ++i) { node.mean[i] = 0.f; node.dir[i] = 0.f; }
    node.dts_mean = node.dts_cov = 0.0;
    bool is_bad = n == 0;
    float mean[3] = {0, 0, 0}, lam[3] = {0, 0, 0}, e0[3] = {0, 0, 0}, e2[3] = {0, 0, 0};
    if (n > 0) {
      if (!parent) {
        double t0 = std::numeric_limits<double>::max();
        for (int64_t i = node.start; i < node.end; ++i) t0 = std::min(t0, pts[i].t);
        meta.ts_start = t0;
      }
      const float isize = 1.0f / (float)n;
      RefAdder<double, 2> ta;
      RefAdder<float, 9> acc;
      for (int64_t i = node.start; i < node.end; ++i) {
        const double dt = pts[i].t - meta.ts_start;
        const double tv[2] = {dt, dt * dt};
        ta.add(tv);
        const float v[3] = {pts[i].x, pts[i].y, pts[i].z};
        float packed[9];
        int k = 0;
        for (int r = 0; r < 3; ++r)
          for (int c = r; c < 3; ++c) packed[k++] = v[r] * v[c];
        for (int r = 0; r < 3; ++r) packed[k++] = v[r];
        acc.add(packed);
      }
      double ts2[2];
      ta.sum(ts2);
      node.dts_mean = ts2[0] * isize;
      node.dts_cov = ts2[1] * isize - node.dts_mean * node.dts_mean;
      float sums[9];
      acc.sum(sums);
      float C[3][3];
      int k = 0;
      for (int r = 0; r < 3; ++r)
        for (int c = r; c < 3; ++c, ++k) C[r][c] = C[c][r] = sums[k] * isize;
      for (int r = 0; r < 3; ++r, ++k) mean[r] = sums[k] * isize;
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) C[r][c] -= mean[r] * mean[c];
      for (int i = 0; i < 3; ++i) node.mean[i] = mean[i];
      if (n < 3) {
        is_bad = true;
      } else {
        float V[3][3];
        eig3_direct(C, lam, V);
        for (int i = 0; i < 3; ++i) { e0[i] = V[i][0]; e2[i] = V[i][2]; }
        if (mean[0] * e0[0] + mean[1] * e0[1] + mean[2] * e0[2] > 0.f) for (int i = 0; i < 3; ++i) e0[i] = -e0[i];
        if (mean[0] * e2[0] + mean[1] * e2[1] + mean[2] * e2[2] > 0.f) for (int i = 0; i < 3; ++i) e2[i] = -e2[i];
      }
    }
    bool is_node = false;
    if (is_bad) {
    } else if ((float)n > (float)P->leaf_max_points) {
      is_node = true;
      for (int i = 0; i < 3; ++i) node.dir[i] = e2[i];
    } else {
      for (int i = 0; i < 3; ++i) node.dir[i] = e0[i];
    }
    bool has_prop = false;
    float prop[3] = {0, 0, 0};
    if (parent && P->propagate_normal) {
      has_prop = parent->has_prop;
      for (int i = 0; i < 3; ++i) prop[i] = parent->prop[i];
    }
    auto propagate = [&]() {
      if (has_prop) {
        float d[3] = {prop[0], prop[1], prop[2]};
        if (mean[0] * d[0] + mean[1] * d[1] + mean[2] * d[2] > 0.f) for (int i = 0; i < 3; ++i) d[i] = -d[i];
        for (int i = 0; i < 3; ++i) node.dir[i] = d[i];
      }
    };
    bool is_flat = false;
    if (is_bad || (float)n < (float)P->leaf_min_points) {
      propagate();
    } else {
      const float ratio = lam[0] / lam[2];
      is_flat = ratio < P->leaf_normal_eigenratio &&
                std::fabs(mean[0] * e0[0] + mean[1] * e0[1] + mean[2] * e0[2]) > P->leaf_min_normal_incidence;
      if (is_flat) {
        has_prop = true;
        for (int i = 0; i < 3; ++i) prop[i] = e0[i];
      }
      if (!is_node) {
        const float density = (float)n / (lam[1] * lam[2]);
        if (density < P->leaf_density) {
          is_node = true;
          for (int i = 0; i < 3; ++i) node.dir[i] = e2[i];
        } else if (is_flat) {
          for (int i = 0; i < 3; ++i) node.dir[i] = e0[i];
        } else {
          propagate();
        }
      }
    }
    if (is_node && meta.level >= P->max_level - 1) {
      is_node = false;
      for (int i = 0; i < 3; ++i) node.dir[i] = e0[i];
    }
    meta.is_node = is_node;
    meta.has_prop = has_prop;
    for (int i = 0; i < 3; ++i) meta.prop[i] = prop[i];
    return meta;
  }

  int make(int64_t s, int64_t e, const RefMeta* parent) const {
    const int my = idx->fetch_add(1);
    if (my >= cap) return -1;
    Node node;
    node.start = s;
    node.end = e;
    node.left = node.right = -1;
    const RefMeta meta = fill(node, parent);
    levels[my] = meta.level;
    if (meta.is_node) {
      int64_t a = s, b = e - 1;  // splitRange: swap with the range end
      while (a <= b) {
        const RefPoint& p = pts[a];
        const float d0 = p.x - node.mean[0], d1 = p.y - node.mean[1], d2 = p.z - node.mean[2];
        if (node.dir[0] * d0 + (node.dir[1] * d1 + node.dir[2] * d2) > 0.0f) {
          ++a;
        } else {
          std::swap(pts[a], pts[b]);
          --b;
        }
      }
      const int64_t mid = a;
      if (parallel_level < 0 || meta.level >= parallel_level) {
        node.left = make(s, mid, &meta);
        node.right = make(mid, e, &meta);
      } else {
        auto hl = std::async(std::launch::async, [&]() { return make(s, mid, &meta); });
        auto hr = std::async(std::launch::async, [&]() { return make(mid, e, &meta); });
        node.left = hl.get();
        node.right = hr.get();
      }
    }
    nodes[my] = node;
    return my;
  }
};

}  // namespace

Tree build_tree_ref32(const float* xyz, const double* st, int64_t n, const TreeParams& P, int parallel_level) {
  Tree T;
  T.num_points = n;
  T.accepted = false;
  if (n < (int64_t)P.leaf_min_points || n == 0) return T;
  std::vector<RefPoint> pts(n);
  for (int64_t i = 0; i < n; ++i) pts[i] = RefPoint{xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], st ? st[i] : 0.0, i};
  const int cap = (int)std::min<int64_t>(4 * n + 64, INT32_MAX / 2);
  std::vector<Node> nodes(cap);
  std::vector<int> levels(cap, 0);
  std::atomic<int> idx(0);
  RefBuild B{pts.data(), nodes.data(), levels.data(), &idx, cap, &P, parallel_level};
  B.make(0, n, nullptr);
  const int nn = std::min(idx.load(), cap);
  T.perm.resize(n);
  for (int64_t i = 0; i < n; ++i) T.perm[i] = pts[i].id;
  // prune (TreeCPU_::prune, kd/tree/tree_cpu_.h:172-196): a node lives if it is a good
  // leaf or has a living child; then breadth-first relabel from the root
  std::vector<char> alive(nn, 0);
  std::vector<int> order;
  order.reserve(nn);
  order.push_back(0);
  for (size_t h = 0; h < order.size(); ++h) {
    const Node& nd = nodes[order[h]];
    if (nd.left >= 0) order.push_back(nd.left);
    if (nd.right >= 0) order.push_back(nd.right);
  }
  for (size_t h = order.size(); h-- > 0;) {
    const int i = order[h];
    const Node& nd = nodes[i];
    if (nd.left < 0 && nd.right < 0) alive[i] = good_leaf(nd, P.prune_min_normal_incidence) ? 1 : 0;
    else alive[i] = ((nd.left >= 0 && alive[nd.left]) || (nd.right >= 0 && alive[nd.right])) ? 1 : 0;
  }
  std::vector<int> newidx(nn, -1);
  int cnt = 0;
  for (int i : order)
    if (alive[i]) newidx[i] = cnt++;
  T.nodes.resize(cnt);
  T.levels.resize(cnt);
  for (int i : order) {
    if (!alive[i]) continue;
    Node nd = nodes[i];
    nd.left = (nd.left >= 0 && alive[nd.left]) ? newidx[nd.left] : -1;
    nd.right = (nd.right >= 0 && alive[nd.right]) ? newidx[nd.right] : -1;
    T.nodes[newidx[i]] = nd;
    T.levels[newidx[i]] = levels[i];
  }
  for (int i = 0; i < cnt; ++i)
    if (T.nodes[i].left < 0 && T.nodes[i].right < 0) T.leaves.push_back(i);
  T.num_unpruned = nn;
  T.accepted = (int64_t)T.leaves.size() >= (int64_t)P.tree_min_good_leaves;
  return T;
}

}  // namespace orc
