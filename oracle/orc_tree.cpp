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
#include <cstdint>
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

}  // namespace orc
