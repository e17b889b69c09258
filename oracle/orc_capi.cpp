// C entry points of the CPU oracle for ctypes -- TEST INFRASTRUCTURE ONLY.
// Used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg.
#include <cstring>
#include <vector>

#include "orc_align.hpp"
#include "orc_math.hpp"
#include "orc_tree.hpp"

using namespace orc;

extern "C" {

void* orc_tree_build(const float* xyz, const double* stamps, int64_t n, const TreeParams* P) {
  Tree* t = new Tree(build_tree(xyz, stamps, n, *P));
  return t;
}

void* orc_tree_build_ref32(const float* xyz, const double* stamps, int64_t n, const TreeParams* P,
                           int32_t parallel_level) {
  return new Tree(build_tree_ref32(xyz, stamps, n, *P, parallel_level));
}

// Tree from a node array (Node_ fields): used to run the oracle aligner on trees
// produced elsewhere.  Leaves are the nodes with no children, in array order.
void* orc_tree_from_nodes(const float* mean, const float* dir, const double* dts_mean, const int32_t* left,
                          const int32_t* right, int64_t num_nodes) {
  Tree* t = new Tree();
  t->nodes.resize(num_nodes);
  t->levels.assign(num_nodes, 0);
  for (int64_t i = 0; i < num_nodes; ++i) {
    Node& n = t->nodes[i];
    for (int k = 0; k < 3; ++k) { n.mean[k] = mean[3 * i + k]; n.dir[k] = dir[3 * i + k]; }
    n.dts_mean = dts_mean ? dts_mean[i] : 0.0;
    n.dts_cov = 0.0;
    n.start = n.end = 0;
    n.left = left[i];
    n.right = right[i];
    if (n.left < 0 && n.right < 0) t->leaves.push_back(i);
  }
  t->accepted = true;
  return t;
}

int64_t orc_tree_num_nodes(void* h) { return (int64_t)((Tree*)h)->nodes.size(); }
int64_t orc_tree_num_leaves(void* h) { return (int64_t)((Tree*)h)->leaves.size(); }
int64_t orc_tree_num_points(void* h) { return ((Tree*)h)->num_points; }
int64_t orc_tree_num_unpruned(void* h) { return ((Tree*)h)->num_unpruned; }
int32_t orc_tree_accepted(void* h) { return ((Tree*)h)->accepted ? 1 : 0; }
double orc_tree_ts_start(void* h) { return ((Tree*)h)->ts_start; }

void orc_tree_export(void* h, float* mean, float* dir, double* dts_mean, double* dts_cov, int64_t* start,
                     int64_t* end, int32_t* left, int32_t* right, int32_t* level, int64_t* leaves, int64_t* perm) {
  Tree* t = (Tree*)h;
  for (size_t i = 0; i < t->nodes.size(); ++i) {
    const Node& n = t->nodes[i];
    for (int k = 0; k < 3; ++k) { mean[3 * i + k] = n.mean[k]; dir[3 * i + k] = n.dir[k]; }
    dts_mean[i] = n.dts_mean;
    dts_cov[i] = n.dts_cov;
    start[i] = n.start;
    end[i] = n.end;
    left[i] = n.left;
    right[i] = n.right;
    level[i] = t->levels[i];
  }
  for (size_t i = 0; i < t->leaves.size(); ++i) leaves[i] = t->leaves[i];
  if (perm)
    for (size_t i = 0; i < t->perm.size(); ++i) perm[i] = t->perm[i];
}

void orc_tree_root(void* h, float* mean, float* eigenvalues, float* eigenvectors) {
  const Tree* t = (const Tree*)h;
  std::memcpy(mean, t->root_mean, sizeof(t->root_mean));
  std::memcpy(eigenvalues, t->root_eigenvalues, sizeof(t->root_eigenvalues));
  std::memcpy(eigenvectors, t->root_eigenvectors, sizeof(t->root_eigenvectors));
}

void orc_tree_free(void* h) { delete (Tree*)h; }

int32_t orc_align(int32_t kind, int32_t mode, void* const* fixed, const double* fixed_X, int32_t num_fixed,
                  void* moving, const AlignParams* P, const OPrior* prior, double* X12, double* v6, const double* fv6,
                  int32_t stats_mode, int32_t num_threads, OResult* out) {
  std::vector<const Tree*> F;
  std::vector<Iso<double>> FX;
  for (int i = 0; i < num_fixed; ++i) {
    F.push_back((const Tree*)fixed[i]);
    FX.push_back(iso_from12<double>(fixed_X + 12 * i));
  }
  return align(kind, mode, F, FX, *(const Tree*)moving, *P, prior, X12, v6, fv6, stats_mode, num_threads, out);
}

// MODE_MIXED compute() that also writes every iteration's correspondences and status:
// match/status hold max_iterations x num_fixed x moving leaves entries.
int32_t orc_align_recorded(int32_t kind, void* const* fixed, const double* fixed_X, int32_t num_fixed, void* moving,
                           const AlignParams* P, double* X12, double* v6, const double* fv6, OResult* out,
                           int32_t* match, int32_t* status) {
  std::vector<const Tree*> F;
  std::vector<Iso<double>> FX;
  for (int i = 0; i < num_fixed; ++i) {
    F.push_back((const Tree*)fixed[i]);
    FX.push_back(iso_from12<double>(fixed_X + 12 * i));
  }
  std::vector<int32_t> m, s;
  int32_t ret = align_recorded(kind, F, FX, *(const Tree*)moving, *P, X12, v6, fv6, out, m, s);
  std::memcpy(match, m.data(), m.size() * sizeof(int32_t));
  std::memcpy(status, s.data(), s.size() * sizeof(int32_t));
  return ret;
}

void orc_align_replay64(int32_t kind, void* const* fixed, const double* fixed_X, int32_t num_fixed, void* moving,
                        const AlignParams* P, double* X12, double* v6, const double* fv6, int32_t iterations,
                        const int32_t* match, const int32_t* status) {
  std::vector<const Tree*> F;
  std::vector<Iso<double>> FX;
  for (int i = 0; i < num_fixed; ++i) {
    F.push_back((const Tree*)fixed[i]);
    FX.push_back(iso_from12<double>(fixed_X + 12 * i));
  }
  align_replay64(kind, F, FX, *(const Tree*)moving, *P, X12, v6, fv6, iterations, match, status);
}

void orc_sincos_canon_d(double x, double* s, double* c) { sincos_canon_d(x, s, c); }

int32_t orc_pose_hessian(const double* H144, double* out36) { return pose_hessian(H144, out36) ? 1 : 0; }

void orc_product_caches(const double* X12, const double* Xf12, float* out36) { product_caches(X12, Xf12, out36); }

void orc_linearize(int32_t kind, void* fixed, void* moving, const float* caches36, const float* v6, const float* fv6,
                   const AlignParams* P, int32_t stats_mode, int32_t* match, int32_t* status, double* H, double* b,
                   OStats* st) {
  linearize_at(kind, *(const Tree*)fixed, *(const Tree*)moving, caches36, v6, fv6, *P, stats_mode, match, status, H,
               b, st);
}

// ---- math pins --------------------------------------------------------------
void orc_sincosf(float x, float* s, float* c) { sincos_canon(x, s, c); }

void orc_err_jac_vel_A(int32_t dbl, void* e, void* J6, const void* Ta12, const void* pa_l, const void* na_l,
                       const void* pb_g, const void* nb_g, const void* va6, double dt) {
  if (dbl) {
    const double* p = (const double*)pa_l; const double* n = (const double*)na_l;
    const double* pb = (const double*)pb_g; const double* nb = (const double*)nb_g;
    err_jac_vel_A<double>(*(double*)e, (double*)J6, iso_from12<double>((const double*)Ta12), v3(p[0], p[1], p[2]),
                          v3(n[0], n[1], n[2]), v3(pb[0], pb[1], pb[2]), v3(nb[0], nb[1], nb[2]),
                          (const double*)va6, dt);
  } else {
    const float* p = (const float*)pa_l; const float* n = (const float*)na_l;
    const float* pb = (const float*)pb_g; const float* nb = (const float*)nb_g;
    err_jac_vel_A<float>(*(float*)e, (float*)J6, iso_from12<float>((const float*)Ta12), v3(p[0], p[1], p[2]),
                         v3(n[0], n[1], n[2]), v3(pb[0], pb[1], pb[2]), v3(nb[0], nb[1], nb[2]), (const float*)va6,
                         (float)dt);
  }
}

void orc_err_jac_vel_B(int32_t dbl, void* e, void* J6, const void* Tb12, const void* pa_g, const void* na_g,
                       const void* pb_l, const void* nb_l, const void* vb6, double dt) {
  if (dbl) {
    const double* p = (const double*)pa_g; const double* n = (const double*)na_g;
    const double* pb = (const double*)pb_l; const double* nb = (const double*)nb_l;
    err_jac_vel_B<double>(*(double*)e, (double*)J6, iso_from12<double>((const double*)Tb12), v3(p[0], p[1], p[2]),
                          v3(n[0], n[1], n[2]), v3(pb[0], pb[1], pb[2]), v3(nb[0], nb[1], nb[2]),
                          (const double*)vb6, dt);
  } else {
    const float* p = (const float*)pa_g; const float* n = (const float*)na_g;
    const float* pb = (const float*)pb_l; const float* nb = (const float*)nb_l;
    err_jac_vel_B<float>(*(float*)e, (float*)J6, iso_from12<float>((const float*)Tb12), v3(p[0], p[1], p[2]),
                         v3(n[0], n[1], n[2]), v3(pb[0], pb[1], pb[2]), v3(nb[0], nb[1], nb[2]), (const float*)vb6,
                         (float)dt);
  }
}

void orc_pose_to_pose_error(int32_t dbl, const void* ZXi12, const void* Xm12, void* e6) {
  if (dbl) pose_to_pose_error(iso_from12<double>((const double*)ZXi12), iso_from12<double>((const double*)Xm12), (double*)e6);
  else pose_to_pose_error(iso_from12<float>((const float*)ZXi12), iso_from12<float>((const float*)Xm12), (float*)e6);
}

void orc_dpose_to_pose_error(int32_t dbl, const void* ZXi12, const void* Xm12, void* J36) {
  if (dbl) {
    double J[6][6];
    dpose_to_pose_error(iso_from12<double>((const double*)ZXi12), iso_from12<double>((const double*)Xm12), J);
    std::memcpy(J36, J, sizeof(J));
  } else {
    float J[6][6];
    dpose_to_pose_error(iso_from12<float>((const float*)ZXi12), iso_from12<float>((const float*)Xm12), J);
    std::memcpy(J36, J, sizeof(J));
  }
}

void orc_expmap(int32_t dbl, const void* v6, void* X12) {
  if (dbl) iso_to12(expmap<double>((const double*)v6), (double*)X12);
  else iso_to12(expmap<float>((const float*)v6), (float*)X12);
}

void orc_iso_mul(const double* A12, const double* B12, double* C12) {
  iso_to12(iso_mul(iso_from12<double>(A12), iso_from12<double>(B12)), C12);
}

// CTICP_3D_Traits::applyVelocities on one (mean, dir) with float dt (kd/d3/cticp_impl_.h:75-85)
void orc_warp_leaf(const float* v6, float dt, const float* m, const float* n, float* mo, float* no) {
  M3<float> R = rodrigues(v3<float>(v6[3] * dt, v6[4] * dt, v6[5] * dt));
  V3<float> a = vadd(mat_vec(R, v3<float>(m[0], m[1], m[2])), v3<float>(v6[0] * dt, v6[1] * dt, v6[2] * dt));
  V3<float> b = mat_vec(R, v3<float>(n[0], n[1], n[2]));
  for (int i = 0; i < 3; ++i) { mo[i] = a[i]; no[i] = b[i]; }
}

// Tree_::applyVelocitiesInPlace over every node (kd/tree/tree_cuda_impl_.h:132-150):
// the per-node warp of orc_warp_leaf at dt = (float)dts_mean.
void orc_tree_apply_velocities(void* h, const float* v6) {
  Tree* t = (Tree*)h;
  for (Node& n : t->nodes) {
    float mo[3], no[3];
    orc_warp_leaf(v6, (float)n.dts_mean, n.mean, n.dir, mo, no);
    for (int i = 0; i < 3; ++i) { n.mean[i] = mo[i]; n.dir[i] = no[i]; }
  }
}

// Tree_::applyIsometryInPlace (kd/tree/tree_cuda_impl_.h:152-173) with applyIsometry_'s
// row loop ((t + R0 p0) + R1 p1) + R2 p2 (kd/utils/geometry_.h:11-25); directions are
// rotated by the same loop from 0.  X: 3x4 row-major floats.
void orc_tree_apply_isometry(void* h, const float* X) {
  Tree* t = (Tree*)h;
  for (Node& n : t->nodes) {
    float m[3], d[3];
    for (int r = 0; r < 3; ++r) {
      const float* R = X + 4 * r;
      m[r] = ((R[3] + R[0] * n.mean[0]) + R[1] * n.mean[1]) + R[2] * n.mean[2];
      d[r] = ((0.0f + R[0] * n.dir[0]) + R[1] * n.dir[1]) + R[2] * n.dir[2];
    }
    for (int i = 0; i < 3; ++i) { n.mean[i] = m[i]; n.dir[i] = d[i]; }
  }
}

// Deep copy (a keyframe kept while the caller's tree moves on).
void* orc_tree_clone(void* h) { return new Tree(*(Tree*)h); }

void orc_jacobi3(const double* A9, double* ev3, double* V9) {
  double A[3][3], V[3][3];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) A[i][j] = A9[i * 3 + j];
  jacobi3(A, ev3, V);
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) V9[i * 3 + j] = V[i][j];
}

void orc_fx_floor(double v, int64_t* hi, uint64_t* lo) { orc::fx_floor_parts(v, hi, lo); }

}  // extern "C"
