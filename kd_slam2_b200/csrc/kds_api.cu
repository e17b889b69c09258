// C ABI of libkds (declared in include/kds.h).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <vector>

#include "kds_align.cuh"
#include "kds_internal.cuh"

namespace kds {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

int cuda_status(cudaError_t e, const char* what, const char* file, int line) {
  set_error("%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  if (e == cudaErrorMemoryAllocation) return KDS_ERR_OOM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return KDS_ERR_NO_DEVICE;
  return KDS_ERR_CUDA;
}

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

static std::once_flag g_once;
static int g_init_status = KDS_OK;

int ensure_init() {
  std::call_once(g_once, []() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
      cudaGetLastError();
      set_error("no CUDA device available");
      g_init_status = KDS_ERR_NO_DEVICE;
      return;
    }
    // keep memory freed with cudaFreeAsync in the device's pool for reuse
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
  });
  if (g_init_status != KDS_OK) set_error("no CUDA device available");
  return g_init_status;
}

}  // namespace kds

using namespace kds;

#define KDS_INIT()                   \
  do {                               \
    int _rc = ::kds::ensure_init();  \
    if (_rc) return _rc;             \
  } while (0)

struct kds_aligner {
  int32_t type;
  kds_aligner_params P;
  const kds_tree* fixed = nullptr;
  const kds_tree* moving = nullptr;
  double X[12];
  double Xf[12];
  double v[6];
  double fv[6];
  int32_t prior_enabled = 0;
  double prior_Xref[12], prior_Z[12], prior_info[36];
  struct Entry {
    const kds_tree* tree;
    double X[12];
  };
  std::vector<Entry> forest;
  cudaStream_t stream = nullptr;
  Runner runner;
  JobOut out;
  std::vector<kds_stats> log;
  int32_t log_n = 0;
  int32_t D() const { return type == KDS_ICP ? 6 : 12; }
};

struct kds_batch {
  Runner runner;
};

static void iso_identity(double* X) {
  for (int i = 0; i < 12; ++i) X[i] = 0.0;
  X[0] = X[5] = X[10] = 1.0;
}

extern "C" {

const char* kds_last_error(void) { return g_last_error.c_str(); }

int64_t kds_launch_count(void) { return g_launches.load(); }

int kds_init(int32_t device, int32_t blocking_sync) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    set_error("no CUDA device available");
    return KDS_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n) { set_error("kds_init: device %d out of range", device); return KDS_ERR_INVALID_ARG; }
  KDS_CK(cudaSetDevice(device));
  if (blocking_sync) {
    e = cudaSetDeviceFlags(cudaDeviceScheduleBlockingSync);
    if (e != cudaSuccess && e != cudaErrorSetOnActiveProcess) return cuda_status(e, "cudaSetDeviceFlags", __FILE__, __LINE__);
    cudaGetLastError();
  }
  return ensure_init();
}

// ---------------------------------------------------------------------------- tree
void kds_tree_params_default(kds_tree_params* p) {
  p->propagate_normal = 0;
  p->tree_min_good_leaves = 10;
  p->leaf_min_points = 5;
  p->leaf_max_points = 30;
  p->leaf_density = 100.f;
  p->leaf_min_normal_incidence = 0.1f;
  p->leaf_eigenvalue_threshold = 1e-3f;
  p->leaf_normal_eigenratio = 0.1f;
  p->prune_min_normal_incidence = 0.1f;
  p->max_level = 48;
}

int kds_tree_build(const float* xyz, const double* stamps, int64_t n, int32_t mem, const kds_tree_params* p,
                   void* stream, kds_tree** out) {
  if (!out) { set_error("kds_tree_build: out is NULL"); return KDS_ERR_INVALID_ARG; }
  *out = nullptr;
  KDS_INIT();
  if ((!xyz && n > 0) || (mem != KDS_MEM_HOST && mem != KDS_MEM_DEVICE)) {
    set_error("kds_tree_build: bad arguments");
    return KDS_ERR_INVALID_ARG;
  }
  kds_tree_params def;
  if (!p) { kds_tree_params_default(&def); p = &def; }
  return tree_build(xyz, stamps, n, mem, p, as_stream(stream), out);
}

int kds_tree_build_batch(const float* xyz, const double* stamps, const int64_t* offsets, int32_t num_trees,
                         int32_t mem, const kds_tree_params* p, void* stream, kds_tree** out, int32_t* status) {
  if (!out || !status || !offsets || num_trees <= 0 || (mem != KDS_MEM_HOST && mem != KDS_MEM_DEVICE)) {
    set_error("kds_tree_build_batch: bad arguments");
    return KDS_ERR_INVALID_ARG;
  }
  for (int r = 0; r < num_trees; ++r) out[r] = nullptr;
  KDS_INIT();
  kds_tree_params def;
  if (!p) { kds_tree_params_default(&def); p = &def; }
  return tree_build_forest(xyz, stamps, offsets, num_trees, mem, p, as_stream(stream), out, status);
}

int kds_tree_build_batch_gather(const float* const* xyz, const double* const* stamps, const int64_t* counts,
                                int32_t num_trees, const kds_tree_params* p, void* stream, kds_tree** out,
                                int32_t* status) {
  if (!out || !status || !xyz || !counts || num_trees <= 0) {
    set_error("kds_tree_build_batch_gather: bad arguments");
    return KDS_ERR_INVALID_ARG;
  }
  for (int r = 0; r < num_trees; ++r) out[r] = nullptr;
  std::vector<int64_t> off((size_t)num_trees + 1, 0);
  bool any_st = false;
  for (int r = 0; r < num_trees; ++r) {
    if (counts[r] < 0 || (counts[r] > 0 && !xyz[r]) || counts[r] > ((int64_t)1 << 30)) {
      set_error("kds_tree_build_batch_gather: cloud %d has a bad count or a NULL point array", r);
      return KDS_ERR_INVALID_ARG;
    }
    off[r + 1] = off[r] + counts[r];
    any_st = any_st || (stamps && stamps[r]);
  }
  if (off[num_trees] > ((int64_t)1 << 30)) { set_error("kds_tree_build_batch_gather: too many points"); return KDS_ERR_INVALID_ARG; }
  KDS_INIT();
  kds_tree_params def;
  if (!p) { kds_tree_params_default(&def); p = &def; }
  cudaStream_t s = as_stream(stream);
  const int64_t N = off[num_trees];
  float* d_xyz = nullptr;
  double* d_st = nullptr;
  cudaError_t e = cudaMallocAsync(&d_xyz, sizeof(float) * 3 * std::max<int64_t>(N, 1), s);
  if (e == cudaSuccess && any_st) e = cudaMallocAsync(&d_st, sizeof(double) * std::max<int64_t>(N, 1), s);
  // each cloud straight into its place: no host-side concatenation
  for (int r = 0; r < num_trees && e == cudaSuccess; ++r) {
    if (counts[r] == 0) continue;
    e = cudaMemcpyAsync(d_xyz + 3 * off[r], xyz[r], sizeof(float) * 3 * counts[r], cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && d_st)
      e = stamps[r] ? cudaMemcpyAsync(d_st + off[r], stamps[r], sizeof(double) * counts[r], cudaMemcpyHostToDevice, s)
                    : cudaMemsetAsync(d_st + off[r], 0, sizeof(double) * counts[r], s);
  }
  int rc = e == cudaSuccess ? tree_build_forest(d_xyz, d_st, off.data(), num_trees, KDS_MEM_DEVICE, p, s, out, status)
                            : cuda_status(e, "kds_tree_build_batch_gather copies", __FILE__, __LINE__);
  if (d_xyz) cudaFreeAsync(d_xyz, s);
  if (d_st) cudaFreeAsync(d_st, s);
  return rc;
}

int kds_tree_import(const float* mean, const float* dir, const double* dts_mean, const double* dts_cov,
                    const int64_t* idx_start, const int64_t* idx_end, const int32_t* left, const int32_t* right,
                    int64_t num_nodes, double ts_start, kds_tree** out) {
  if (!out) { set_error("kds_tree_import: out is NULL"); return KDS_ERR_INVALID_ARG; }
  *out = nullptr;
  KDS_INIT();
  return tree_import(mean, dir, dts_mean, dts_cov, idx_start, idx_end, left, right, num_nodes, ts_start, out);
}

int kds_tree_get_info(const kds_tree* t, kds_tree_info* info) {
  if (!t || !info) { set_error("kds_tree_get_info: NULL argument"); return KDS_ERR_INVALID_ARG; }
  info->num_nodes = t->d.num_nodes;
  info->num_leaves = t->d.num_leaves;
  info->num_points = t->d.num_points;
  info->num_unpruned = t->d.num_unpruned;
  info->ts_start = t->d.ts_start;
  info->accepted = t->d.accepted;
  info->depth = t->d.depth;
  info->global_levels = t->d.global_levels;
  info->pad_ = 0;
  return KDS_OK;
}

void kds_voxel_params_default(kds_voxel_params* p) {
  if (!p) return;
  p->range_min = 0.f;
  p->range_max = 100.f;
  p->space_res = 0.f;
  p->time_res = 0.f;
  p->use_boundary = 0;
}

int kds_points_voxelize(const float* xyz, const double* stamps, int64_t n, int32_t mem, double msg_t,
                        double scan_duration, const kds_voxel_params* p, void* stream, float* out_xyz,
                        double* out_stamps, int64_t* out_n) {
  KDS_INIT();
  return points_voxelize(xyz, stamps, n, mem, msg_t, scan_duration, p, as_stream(stream), out_xyz, out_stamps,
                         out_n);
}

int kds_tree_get_root(const kds_tree* t, float mean[3], float eigenvalues[3], float eigenvectors[9]) {
  if (!t) { set_error("kds_tree_get_root: NULL tree"); return KDS_ERR_INVALID_ARG; }
  if (mean) memcpy(mean, t->root_mean, sizeof(t->root_mean));
  if (eigenvalues) memcpy(eigenvalues, t->root_eigenvalues, sizeof(t->root_eigenvalues));
  if (eigenvectors) memcpy(eigenvectors, t->root_eigenvectors, sizeof(t->root_eigenvectors));
  return KDS_OK;
}

int kds_tree_from_msg(const kds_kdtree3f* msg, kds_tree** out) {
  if (!out || !msg) { set_error("kds_tree_from_msg: NULL argument"); return KDS_ERR_INVALID_ARG; }
  *out = nullptr;
  KDS_INIT();
  return tree_from_msg(msg, out);
}

int kds_tree_to_msg(const kds_tree* t, kds_kdtree3f* msg) {
  if (!t || !msg || msg->num_nodes < 0) { set_error("kds_tree_to_msg: bad argument"); return KDS_ERR_INVALID_ARG; }
  const int64_t n = t->d.num_nodes, cap = msg->num_nodes;
  msg->ts_start = t->d.ts_start;
  memcpy(msg->root_mean, t->root_mean, sizeof(t->root_mean));
  memcpy(msg->root_eigenvalues, t->root_eigenvalues, sizeof(t->root_eigenvalues));
  memcpy(msg->root_eigenvectors, t->root_eigenvectors, sizeof(t->root_eigenvectors));
  msg->num_nodes = n;
  if (cap < n || (n > 0 && !msg->nodes)) {
    if (cap == 0 && !msg->nodes) return KDS_OK;  // count query
    set_error("kds_tree_to_msg: %lld node records do not fit in %lld", (long long)n, (long long)cap);
    return KDS_ERR_CAPACITY;
  }
  if (n == 0) return KDS_OK;
  std::vector<float> mean(3 * n), dir(3 * n);
  std::vector<double> dm(n), dc(n);
  std::vector<int64_t> s0(n), e0(n);
  std::vector<int32_t> l(n), r(n);
  int rc = tree_export(t, mean.data(), dir.data(), dm.data(), dc.data(), s0.data(), e0.data(), l.data(), r.data(),
                       nullptr, nullptr, nullptr);
  if (rc) return rc;
  for (int64_t i = 0; i < n; ++i) {
    kds_kdnode3f& k = msg->nodes[i];
    for (int d = 0; d < 3; ++d) {
      k.mean[d] = mean[3 * i + d];
      k.direction[d] = dir[3 * i + d];
    }
    k.idx_start = (uint32_t)s0[i];
    k.idx_end = (uint32_t)e0[i];
    k.idx_left = l[i];
    k.idx_right = r[i];
    k.dts_mean = dm[i];
    k.dts_covariance = dc[i];
  }
  return KDS_OK;
}

int kds_tree_export(const kds_tree* t, float* mean, float* dir, double* dts_mean, double* dts_cov, int64_t* idx_start,
                    int64_t* idx_end, int32_t* left, int32_t* right, int32_t* level, int64_t* leaves, int64_t* perm) {
  if (!t) { set_error("kds_tree_export: NULL tree"); return KDS_ERR_INVALID_ARG; }
  return tree_export(t, mean, dir, dts_mean, dts_cov, idx_start, idx_end, left, right, level, leaves, perm);
}

int kds_tree_apply_velocities(kds_tree* t, const float v[6], int32_t skip_leaves, void* stream) {
  if (!t || !v) { set_error("kds_tree_apply_velocities: NULL argument"); return KDS_ERR_INVALID_ARG; }
  return tree_apply_velocities(t, v, skip_leaves, as_stream(stream));
}

int kds_tree_apply_isometry(kds_tree* t, const float X[12], void* stream) {
  if (!t || !X) { set_error("kds_tree_apply_isometry: NULL argument"); return KDS_ERR_INVALID_ARG; }
  return tree_apply_isometry(t, X, as_stream(stream));
}

int kds_tree_extract_compressed_leaves(const kds_tree* t, const float* v6, float* out, void* stream) {
  if (!t || !out) { set_error("kds_tree_extract_compressed_leaves: NULL argument"); return KDS_ERR_INVALID_ARG; }
  return tree_extract_leaves(t, v6, out, nullptr, as_stream(stream));
}

int kds_tree_extract_compressed_leaves_device(const kds_tree* t, const float* v6, float* out_device, void* stream) {
  if (!t || !out_device) {
    set_error("kds_tree_extract_compressed_leaves_device: NULL argument");
    return KDS_ERR_INVALID_ARG;
  }
  return tree_extract_leaves(t, v6, nullptr, out_device, as_stream(stream));
}

void kds_tree_free(kds_tree* t) {
  if (!t) return;
  tree_release(t->d);
  delete t;
}

// ---------------------------------------------------------------------------- aligner
void kds_aligner_params_default(kds_aligner_params* p) {
  p->kernel_threshold = 0.1f;
  p->damping = 1.0f;
  p->max_error = 1.0f;
  p->min_normal_cos = (float)std::cos(25.0 / 180.0 * M_PI);
  p->min_good_measurements = 10;
  p->max_iterations = 20;
  p->velocity_damping = 100.f;
  p->term_crit = 0;
  p->d_pert = 1e-3f;
  p->d_score = 1e-3f;
}

int kds_aligner_create(int32_t type, const kds_aligner_params* p, kds_aligner** out) {
  if (!out || (type != KDS_ICP && type != KDS_CTICP)) { set_error("kds_aligner_create: bad arguments"); return KDS_ERR_INVALID_ARG; }
  KDS_INIT();
  kds_aligner* a = new kds_aligner();
  a->type = type;
  if (p) a->P = *p;
  else kds_aligner_params_default(&a->P);
  iso_identity(a->X);
  iso_identity(a->Xf);
  for (int i = 0; i < 6; ++i) { a->v[i] = 0.0; a->fv[i] = 0.0; }
  memset(&a->out, 0, sizeof(a->out));
  *out = a;
  return KDS_OK;
}

#define CHECK_A(a)                                                    \
  do {                                                                \
    if (!(a)) { set_error("NULL aligner"); return KDS_ERR_INVALID_ARG; } \
  } while (0)

int kds_aligner_set_params(kds_aligner* a, const kds_aligner_params* p) { CHECK_A(a); if (!p) return KDS_ERR_INVALID_ARG; a->P = *p; return KDS_OK; }
int kds_aligner_set_stream(kds_aligner* a, void* s) { CHECK_A(a); a->stream = (cudaStream_t)s; return KDS_OK; }
int kds_aligner_set_fixed(kds_aligner* a, const kds_tree* t) { CHECK_A(a); a->fixed = t; return KDS_OK; }
int kds_aligner_set_moving(kds_aligner* a, const kds_tree* t) { CHECK_A(a); a->moving = t; return KDS_OK; }
int kds_aligner_set_x(kds_aligner* a, const double X[12]) { CHECK_A(a); memcpy(a->X, X, sizeof(a->X)); return KDS_OK; }
int kds_aligner_get_x(const kds_aligner* a, double X[12]) { CHECK_A(a); memcpy(X, a->X, sizeof(a->X)); return KDS_OK; }
int kds_aligner_set_fixed_x(kds_aligner* a, const double X[12]) {
  CHECK_A(a);
  memcpy(a->Xf, X, sizeof(a->Xf));
  if (a->type == KDS_CTICP)  // CTICP_::setFixedX zeroes the fixed velocities (kd/cticp/cticp_.h:222-225)
    for (int i = 0; i < 6; ++i) a->fv[i] = 0.0;
  return KDS_OK;
}
int kds_aligner_set_velocities(kds_aligner* a, const double v[6]) {
  CHECK_A(a);
  if (a->type == KDS_ICP) return KDS_OK;  // TreeAlignerBase_::setVelocities is a no-op for ICP
  memcpy(a->v, v, sizeof(a->v));
  return KDS_OK;
}
int kds_aligner_get_velocities(const kds_aligner* a, double v[6]) {
  CHECK_A(a);
  if (a->type == KDS_ICP) { for (int i = 0; i < 6; ++i) v[i] = 0.0; return KDS_OK; }
  memcpy(v, a->v, sizeof(a->v));
  return KDS_OK;
}
int kds_aligner_set_fixed_velocities(kds_aligner* a, const double v[6]) { CHECK_A(a); memcpy(a->fv, v, sizeof(a->fv)); return KDS_OK; }
int kds_aligner_reset_moving_state(kds_aligner* a) {
  CHECK_A(a);
  if (a->type == KDS_CTICP) for (int i = 0; i < 6; ++i) a->v[i] = 0.0;
  return KDS_OK;
}
int kds_aligner_set_pose_prior(kds_aligner* a, const double X_ref[12], const double Z[12], const double info[36]) {
  CHECK_A(a);
  bool nz = false;
  for (int i = 0; i < 36; ++i) nz |= info[i] != 0.0;
  a->prior_enabled = nz ? 1 : 0;
  memcpy(a->prior_Xref, X_ref, sizeof(a->prior_Xref));
  memcpy(a->prior_Z, Z, sizeof(a->prior_Z));
  memcpy(a->prior_info, info, sizeof(a->prior_info));
  return KDS_OK;
}
int kds_aligner_add_fixed_entry(kds_aligner* a, const kds_tree* t, const double X[12]) {
  CHECK_A(a);
  if (!t) return KDS_ERR_INVALID_ARG;
  kds_aligner::Entry e;
  e.tree = t;
  memcpy(e.X, X, sizeof(e.X));
  a->forest.push_back(e);
  return KDS_OK;
}
int kds_aligner_clear_fixed_forest(kds_aligner* a) { CHECK_A(a); a->forest.clear(); return KDS_OK; }

static ParamsF to_paramsf(const kds_aligner_params& p) {
  ParamsF f;
  f.kernel_threshold = p.kernel_threshold;
  f.damping = p.damping;
  f.max_error = p.max_error;
  f.min_normal_cos = p.min_normal_cos;
  f.min_good_measurements = p.min_good_measurements;
  f.max_iterations = p.max_iterations;
  f.velocity_damping = p.velocity_damping;
  f.term_crit = p.term_crit;
  f.d_pert = p.d_pert;
  f.d_score = p.d_score;
  return f;
}

static void mul12(const double* A, const double* B, double* C) {
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) C[i * 4 + j] = A[i * 4] * B[j] + A[i * 4 + 1] * B[4 + j] + A[i * 4 + 2] * B[8 + j];
    C[i * 4 + 3] = A[i * 4] * B[3] + A[i * 4 + 1] * B[7] + A[i * 4 + 2] * B[11] + A[i * 4 + 3];
  }
}
static void inv12(const double* A, double* B) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) B[i * 4 + j] = A[j * 4 + i];
  for (int i = 0; i < 3; ++i) B[i * 4 + 3] = -(B[i * 4] * A[3] + B[i * 4 + 1] * A[7] + B[i * 4 + 2] * A[11]);
}

// Fills one job (+ its fixed entries) from an aligner.
static int make_job(kds_aligner* a, int kind, int mode, int stats_mode, int max_iter_override, JobIn& J,
                    std::vector<LinDev>& lins) {
  if (!a->moving) { set_error("aligner has no moving tree"); return KDS_ERR_STATE; }
  if (a->forest.empty() && !a->fixed) { set_error("aligner has no fixed tree"); return KDS_ERR_STATE; }
  memset(&J, 0, sizeof(J));
  J.m_md = a->moving->d.leaf_md;
  J.m_nrm = a->moving->d.leaf_nrm;
  J.m_num_leaves = (int32_t)a->moving->d.num_leaves;
  J.kind = kind;
  J.mode = mode;
  J.stats_mode = stats_mode;
  J.P = to_paramsf(a->P);
  if (max_iter_override > 0) {
    J.P.max_iterations = max_iter_override;
    J.P.term_crit = 0;
  }
  J.prior_enabled = a->prior_enabled;
  if (a->prior_enabled) {
    double XZ[12];
    mul12(a->prior_Xref, a->prior_Z, XZ);
    inv12(XZ, J.prior_ZXi);
    memcpy(J.prior_info, a->prior_info, sizeof(J.prior_info));
  }
  memcpy(J.X0, a->X, sizeof(J.X0));
  memcpy(J.v0, a->v, sizeof(J.v0));
  J.lin_begin = (int32_t)lins.size();
  auto add_lin = [&](const kds_tree* t, const double* Xf) {
    LinDev L;
    memset(&L, 0, sizeof(L));
    L.fnodes = t->d.nodes;
    L.fdts = t->d.dts_f;
    L.f_num_nodes = (int32_t)t->d.num_nodes;
    L.job = 0;
    memcpy(L.Xf, Xf, sizeof(L.Xf));
    memcpy(L.fv, a->fv, sizeof(L.fv));
    lins.push_back(L);
  };
  if (a->forest.empty()) add_lin(a->fixed, a->Xf);
  else
    for (auto& e : a->forest) add_lin(e.tree, e.X);
  J.lin_count = (int32_t)lins.size() - J.lin_begin;
  return KDS_OK;
}

static int run_single(kds_aligner* a, int kind, int mode, int stats_mode, int max_iter_override, bool use_graph,
                      int32_t* dbg_match, int32_t* dbg_status, const float* caches, bool update_state) {
  std::vector<JobIn> jobs(1);
  std::vector<LinDev> lins;
  int rc = make_job(a, kind, mode, stats_mode, max_iter_override, jobs[0], lins);
  if (rc) return rc;
  if (caches) {
    jobs[0].keep_cache = 1;
    for (auto& L : lins) {
      memcpy(L.cache.Xm, caches, 12 * sizeof(float));
      memcpy(L.cache.Xf, caches + 12, 12 * sizeof(float));
      memcpy(L.cache.Xmf, caches + 24, 12 * sizeof(float));
    }
  }
  cudaStream_t s = a->stream ? a->stream : cudaStreamPerThread;
  rc = a->runner.setup(jobs, lins, s);
  if (rc) return rc;
  rc = a->runner.run(s, use_graph, dbg_match, dbg_status);
  if (rc) return rc;
  std::vector<JobOut> outs;
  rc = a->runner.fetch(s, outs, mode == KDS_JOB_COMPUTE ? &a->log : nullptr);
  if (rc && rc != KDS_ERR_TIMEOUT) return rc;  // a timeout still delivers valid outputs
  a->out = outs[0];
  if (mode == KDS_JOB_COMPUTE) {
    a->log_n = std::min(outs[0].iterations, (int32_t)kMaxLog);
    if (update_state) {
      memcpy(a->X, outs[0].X, sizeof(a->X));
      if (a->type == KDS_CTICP) memcpy(a->v, outs[0].v, sizeof(a->v));
    }
  }
  return rc;
}

int kds_aligner_compute(kds_aligner* a, int32_t stats_mode, int32_t* result) {
  CHECK_A(a);
  int rc = run_single(a, a->type == KDS_ICP ? 0 : 1, KDS_JOB_COMPUTE, stats_mode, 0, true, nullptr, nullptr, nullptr,
                      true);
  if (rc) return rc;
  if (result) *result = a->out.result;
  return KDS_OK;
}

int kds_aligner_one_round(kds_aligner* a, int32_t stats_mode, int32_t* ok) {
  CHECK_A(a);
  int rc = run_single(a, a->type == KDS_ICP ? 0 : 1, KDS_JOB_COMPUTE, stats_mode, 1, false, nullptr, nullptr, nullptr,
                      true);
  if (rc) return rc;
  if (ok) *ok = (a->out.result == 1) ? 1 : 0;
  return KDS_OK;
}

int kds_aligner_build_quadratic_form(kds_aligner* a, int32_t stats_mode) {
  CHECK_A(a);
  return run_single(a, a->type == KDS_ICP ? 0 : 1, KDS_JOB_LINEARIZE, stats_mode, 0, false, nullptr, nullptr, nullptr,
                    false);
}

int kds_aligner_build_quadratic_form_dual(kds_aligner* a, int32_t stats_mode) {
  CHECK_A(a);
  if (a->type != KDS_CTICP) {
    // ICP_::buildQuadraticFormDual: J_B = -J_A, so no extra accumulation is needed
    return kds_aligner_build_quadratic_form(a, stats_mode);
  }
  return run_single(a, 2, KDS_JOB_LINEARIZE_DUAL, stats_mode, 0, false, nullptr, nullptr, nullptr, false);
}

int kds_aligner_get_hb(const kds_aligner* a, double* H, double* b, double* dx) {
  CHECK_A(a);
  int D = a->D();
  if (H) memcpy(H, a->out.H, sizeof(double) * D * D);
  if (b) memcpy(b, a->out.b, sizeof(double) * D);
  if (dx) memcpy(dx, a->out.dx, sizeof(double) * D);
  return KDS_OK;
}

int kds_aligner_get_dual(const kds_aligner* a, double H_vel_B[36], double b_vel_B[6], double H_cross_pose_vel_B[36],
                         double H_cross_vel_AB[36]) {
  CHECK_A(a);
  if (H_vel_B) memcpy(H_vel_B, a->out.H_vel_B, sizeof(double) * 36);
  if (b_vel_B) memcpy(b_vel_B, a->out.b_vel_B, sizeof(double) * 6);
  if (H_cross_pose_vel_B) memcpy(H_cross_pose_vel_B, a->out.H_cross_pose_vel_B, sizeof(double) * 36);
  if (H_cross_vel_AB) memcpy(H_cross_vel_AB, a->out.H_cross_vel_AB, sizeof(double) * 36);
  return KDS_OK;
}

// 6x6 inverse by Gauss-Jordan with partial pivoting (host, FP64)
static bool inv6(const double* A, double* Ai) {
  double M[6][12];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 12; ++j) M[i][j] = j < 6 ? A[i * 6 + j] : (j - 6 == i ? 1.0 : 0.0);
  for (int c = 0; c < 6; ++c) {
    int p = c;
    for (int r = c + 1; r < 6; ++r)
      if (std::fabs(M[r][c]) > std::fabs(M[p][c])) p = r;
    if (M[p][c] == 0.0) return false;
    for (int j = 0; j < 12; ++j) std::swap(M[c][j], M[p][j]);
    double d = M[c][c];
    for (int j = 0; j < 12; ++j) M[c][j] /= d;
    for (int r = 0; r < 6; ++r) {
      if (r == c) continue;
      double f = M[r][c];
      for (int j = 0; j < 12; ++j) M[r][j] -= f * M[c][j];
    }
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) Ai[i * 6 + j] = M[i][6 + j];
  return true;
}

int kds_aligner_get_pose_hessian(const kds_aligner* a, double H6[36]) {
  CHECK_A(a);
  if (a->type == KDS_ICP) { memcpy(H6, a->out.H, sizeof(double) * 36); return KDS_OK; }
  // CTICP_::poseHessian (kd/cticp/cticp_.h:169-177): H_pp - H_pv (H_vv + 1e-9 I)^-1 H_pv^T
  const double* H = a->out.H;
  double Hvv[36], Hvvi[36];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) Hvv[i * 6 + j] = H[(6 + i) * 12 + 6 + j] + (i == j ? 1e-9 : 0.0);
  if (!inv6(Hvv, Hvvi)) { set_error("velocity block is singular"); return KDS_ERR_STATE; }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      double acc = H[i * 12 + j];
      for (int k = 0; k < 6; ++k)
        for (int l = 0; l < 6; ++l) acc -= H[i * 12 + 6 + k] * Hvvi[k * 6 + l] * H[j * 12 + 6 + l];
      H6[i * 6 + j] = acc;
    }
  return KDS_OK;
}

int kds_aligner_get_stats(const kds_aligner* a, kds_stats* s) { CHECK_A(a); *s = a->out.stats; return KDS_OK; }

int kds_aligner_get_stats_log(const kds_aligner* a, kds_stats* log, int32_t cap, int32_t* n) {
  CHECK_A(a);
  int m = std::min(cap, a->log_n);
  for (int i = 0; i < m; ++i) log[i] = a->log[i];
  if (n) *n = a->log_n;
  return KDS_OK;
}

int kds_aligner_linearize_debug(kds_aligner* a, const float caches[36], const float v[6], const float fixed_v[6],
                                int32_t kind, int32_t stats_mode, int32_t* match, int32_t* status, double* H,
                                double* b, kds_stats* stats) {
  CHECK_A(a);
  if (!a->moving || !a->fixed || !caches || kind < 0 || kind > 2) { set_error("linearize_debug: bad arguments"); return KDS_ERR_INVALID_ARG; }
  double vs[6], fvs[6];
  memcpy(vs, a->v, sizeof(vs));
  memcpy(fvs, a->fv, sizeof(fvs));
  for (int i = 0; i < 6; ++i) { a->v[i] = v ? v[i] : 0.0; a->fv[i] = fixed_v ? fixed_v[i] : 0.0; }
  std::vector<kds_aligner::Entry> forest;
  forest.swap(a->forest);
  int64_t n = a->moving->d.num_leaves;
  int32_t *dm = nullptr, *ds = nullptr;
  int rc = KDS_OK;
  cudaError_t e1 = cudaMalloc(&dm, sizeof(int32_t) * std::max<int64_t>(n, 1));
  cudaError_t e2 = cudaMalloc(&ds, sizeof(int32_t) * std::max<int64_t>(n, 1));
  if (e1 != cudaSuccess || e2 != cudaSuccess) rc = KDS_ERR_OOM;
  if (!rc) {
    // exact float velocities: the caches carry them
    float cc[36];
    memcpy(cc, caches, sizeof(cc));
    std::vector<JobIn> jobs(1);
    std::vector<LinDev> lins;
    rc = make_job(a, kind, kind == 2 ? KDS_JOB_LINEARIZE_DUAL : KDS_JOB_LINEARIZE, stats_mode, 0, jobs[0], lins);
    if (!rc) {
      jobs[0].keep_cache = 1;
      for (auto& L : lins) {
        memcpy(L.cache.Xm, cc, 12 * sizeof(float));
        memcpy(L.cache.Xf, cc + 12, 12 * sizeof(float));
        memcpy(L.cache.Xmf, cc + 24, 12 * sizeof(float));
        for (int i = 0; i < 6; ++i) { L.cache.v[i] = v ? v[i] : 0.f; L.cache.fv[i] = fixed_v ? fixed_v[i] : 0.f; }
      }
      cudaStream_t s = a->stream ? a->stream : cudaStreamPerThread;
      rc = a->runner.setup(jobs, lins, s);
      if (!rc) rc = a->runner.run(s, false, dm, ds);
      std::vector<JobOut> outs;
      if (!rc) rc = a->runner.fetch(s, outs, nullptr);
      if (!rc) {
        a->out = outs[0];
        int D = kind == 0 ? 6 : 12;
        if (H) memcpy(H, outs[0].H, sizeof(double) * D * D);
        if (b) memcpy(b, outs[0].b, sizeof(double) * D);
        if (stats) *stats = outs[0].stats;
        if (match && n) { cudaError_t e = cudaMemcpy(match, dm, sizeof(int32_t) * n, cudaMemcpyDeviceToHost); if (e) rc = cuda_status(e, "copy", __FILE__, __LINE__); }
        if (status && n) { cudaError_t e = cudaMemcpy(status, ds, sizeof(int32_t) * n, cudaMemcpyDeviceToHost); if (e) rc = cuda_status(e, "copy", __FILE__, __LINE__); }
      }
    }
  }
  if (dm) cudaFree(dm);
  if (ds) cudaFree(ds);
  forest.swap(a->forest);
  memcpy(a->v, vs, sizeof(vs));
  memcpy(a->fv, fvs, sizeof(fvs));
  return rc;
}

int kds_aligner_set_profiling(kds_aligner* a, int32_t on) {
  CHECK_A(a);
  a->runner.profiling = on != 0;
  return phase_stamps(on != 0 ? 1 : 0, nullptr);
}

int kds_set_tma_wait_limit(int32_t polls) { return set_wait_spins(polls); }

int kds_phase_stamps(uint64_t* out16) {
  if (!out16) return KDS_ERR_INVALID_ARG;
  return phase_stamps(-1, reinterpret_cast<unsigned long long*>(out16));
}

int kds_linearize_static(const kds_tree* fixed, const kds_tree* moving, int32_t type,
                         const kds_aligner_params* params, const double X[12], const double fixed_X[12],
                         const double v[6], const double fixed_v[6], int32_t stats_mode, void* stream, double* H,
                         double* b, kds_stats* stats) {
  KDS_INIT();
  if (!fixed || !moving || !params || !X || !fixed_X || (type != KDS_ICP && type != KDS_CTICP)) {
    set_error("kds_linearize_static: fixed, moving, params, X and fixed_X are required; type is KDS_ICP or KDS_CTICP");
    return KDS_ERR_INVALID_ARG;
  }
  return linearize_static(fixed->d, moving->d, type, *params, X, fixed_X, v, fixed_v, stats_mode, as_stream(stream),
                          H, b, stats);
}

int kds_aligner_get_profile(const kds_aligner* a, double* mean_ms, int32_t* launches) {
  CHECK_A(a);
  int n = 0;
  double m = a->runner.profile_mean_ms(&n);
  if (mean_ms) *mean_ms = m;
  if (launches) *launches = n;
  return KDS_OK;
}

int kds_aligner_count_touched_nodes(kds_aligner* a, int64_t* count) {
  CHECK_A(a);
  if (!count) return KDS_ERR_INVALID_ARG;
  std::vector<JobIn> jobs(1);
  std::vector<LinDev> lins;
  int kind = a->type == KDS_ICP ? 0 : 1;
  int rc = make_job(a, kind, KDS_JOB_LINEARIZE, 0, 0, jobs[0], lins);
  if (rc) return rc;
  cudaStream_t s = a->stream ? a->stream : cudaStreamPerThread;
  rc = a->runner.setup(jobs, lins, s);
  if (rc) return rc;
  const kds_tree* f = a->forest.empty() ? a->fixed : a->forest[0].tree;
  return count_touched(a->runner, kind, f->d.num_nodes, count, s);
}

void kds_aligner_free(kds_aligner* a) { delete a; }

// ---------------------------------------------------------------------------- batch
int kds_batch_create(kds_batch** out) {
  if (!out) return KDS_ERR_INVALID_ARG;
  KDS_INIT();
  *out = new kds_batch();
  return KDS_OK;
}

static int batch_inputs(kds_job* jobs, int32_t num_jobs, std::vector<JobIn>& J, std::vector<LinDev>& lins) {
  J.assign(num_jobs, JobIn());
  lins.clear();
  for (int j = 0; j < num_jobs; ++j) {
    kds_job& q = jobs[j];
    if (!q.fixed || !q.moving || (q.type != KDS_ICP && q.type != KDS_CTICP)) {
      set_error("kds_batch_run: job %d is incomplete", j);
      return KDS_ERR_INVALID_ARG;
    }
    JobIn& Jn = J[j];
    memset(&Jn, 0, sizeof(Jn));
    Jn.m_md = q.moving->d.leaf_md;
    Jn.m_nrm = q.moving->d.leaf_nrm;
    Jn.m_num_leaves = (int32_t)q.moving->d.num_leaves;
    int kind = q.type == KDS_ICP ? 0 : 1;
    if (q.mode == KDS_JOB_LINEARIZE_DUAL && q.type == KDS_CTICP) kind = 2;
    Jn.kind = kind;
    Jn.mode = q.mode;
    Jn.stats_mode = q.stats_mode;
    Jn.P = to_paramsf(q.params);
    memcpy(Jn.X0, q.X, sizeof(Jn.X0));
    for (int i = 0; i < 6; ++i) Jn.v0[i] = q.type == KDS_ICP ? 0.0 : q.v[i];
    Jn.lin_begin = (int32_t)lins.size();
    Jn.lin_count = 1;
    LinDev L;
    memset(&L, 0, sizeof(L));
    L.fnodes = q.fixed->d.nodes;
    L.fdts = q.fixed->d.dts_f;
    L.f_num_nodes = (int32_t)q.fixed->d.num_nodes;
    L.job = j;
    memcpy(L.Xf, q.fixed_X, sizeof(L.Xf));
    memcpy(L.fv, q.fixed_v, sizeof(L.fv));
    lins.push_back(L);
  }
  return KDS_OK;
}

// Candidate launch configurations of the autotuner: (tree-top nodes staged per block,
// tiles of larger jobs first).
static const int kTuneStage[3] = {0, 1023, 2047};
// config = stage index + 3 * order_by_size + 6 * form; form 0: one launch per iteration
// and kind, one tile per block; 1: persistent; 2: one launch per iteration and kind, two
// tiles per block
static const int kTuneConfigs = 18;
static void apply_config(Runner& R, int c) {
  R.stage_nodes = kTuneStage[c % 3];
  R.order_by_size = (c / 3) % 2;
  R.persistent = (c / 6) == 1 ? 1 : 0;
  R.pair_tiles = (c / 6) == 2 ? 1 : 0;
}

int kds_batch_autotune(kds_batch* B, kds_job* jobs, int32_t num_jobs, void* stream, int32_t* chosen,
                       double* ms_out) {
  if (!B || num_jobs <= 0 || !jobs) { set_error("kds_batch_autotune: bad arguments"); return KDS_ERR_INVALID_ARG; }
  std::vector<JobIn> J;
  std::vector<LinDev> lins;
  int rc = batch_inputs(jobs, num_jobs, J, lins);
  if (rc) return rc;
  cudaStream_t s = as_stream(stream);
  cudaEvent_t e0, e1;
  KDS_CK(cudaEventCreate(&e0));
  KDS_CK(cudaEventCreate(&e1));
  int best = -1;
  double best_ms = 1e300;
  for (int c = 0; c < kTuneConfigs && rc == KDS_OK; ++c) {
    apply_config(B->runner, c);
    double sum = 0.0;
    for (int rep = 0; rep < 5 && rc == KDS_OK; ++rep) {  // two warm-ups (direct, graph capture), three timed
      rc = B->runner.setup(J, lins, s);
      if (rc) break;
      if (cudaEventRecord(e0, s) != cudaSuccess) { rc = cuda_status(cudaGetLastError(), "autotune", __FILE__, __LINE__); break; }
      rc = B->runner.run(s, true, nullptr, nullptr);
      if (rc) break;
      cudaEventRecord(e1, s);
      cudaError_t e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) { rc = cuda_status(e, "autotune", __FILE__, __LINE__); break; }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 1) sum += ms;
    }
    if (rc) break;
    const double mean = sum / 3.0;
    if (ms_out) ms_out[c] = mean;
    if (mean < best_ms) { best_ms = mean; best = c; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  apply_config(B->runner, best);
  if (chosen) *chosen = best;
  return KDS_OK;
}

int kds_batch_configure(kds_batch* B, int32_t config) {
  if (!B || config < 0 || config >= kTuneConfigs) {
    set_error("kds_batch_configure: config must be in [0, %d)", kTuneConfigs);
    return KDS_ERR_INVALID_ARG;
  }
  apply_config(B->runner, config);
  return KDS_OK;
}

int kds_batch_assemble(kds_batch* B, const kds_factor* factors, int32_t num_factors, int32_t num_vars,
                       float disable_inlier_ratio, void* stream, int32_t* num_blocks, int32_t* block_rc,
                       double* H_blocks, double* b_vec, int32_t* enabled) {
  if (!B) { set_error("kds_batch_assemble: NULL batch"); return KDS_ERR_INVALID_ARG; }
  return batch_assemble(B->runner, factors, num_factors, num_vars, disable_inlier_ratio, as_stream(stream),
                        num_blocks, block_rc, H_blocks, b_vec, enabled);
}

int kds_batch_run(kds_batch* B, kds_job* jobs, int32_t num_jobs, int32_t use_graph, void* stream) {
  if (!B || (num_jobs > 0 && !jobs) || num_jobs < 0) { set_error("kds_batch_run: bad arguments"); return KDS_ERR_INVALID_ARG; }
  std::vector<JobIn> J;
  std::vector<LinDev> lins;
  {
    int rc0 = batch_inputs(jobs, num_jobs, J, lins);
    if (rc0) return rc0;
  }
  cudaStream_t s = as_stream(stream);
  int rc = B->runner.setup(J, lins, s);
  if (rc) return rc;
  rc = B->runner.run(s, use_graph != 0, nullptr, nullptr);
  if (rc) return rc;
  std::vector<JobOut> outs;
  rc = B->runner.fetch(s, outs, nullptr);
  if (rc && rc != KDS_ERR_TIMEOUT) return rc;  // a timeout still delivers valid outputs
  for (int j = 0; j < num_jobs; ++j) {
    kds_job& q = jobs[j];
    const JobOut& o = outs[j];
    int D = q.type == KDS_ICP ? 6 : 12;
    memcpy(q.X, o.X, sizeof(q.X));
    if (q.type == KDS_CTICP) memcpy(q.v, o.v, sizeof(q.v));
    q.result = o.result;
    q.iterations = o.iterations;
    q.stats = o.stats;
    memcpy(q.H, o.H, sizeof(double) * D * D);
    memcpy(q.b, o.b, sizeof(double) * D);
    memcpy(q.H_vel_B, o.H_vel_B, sizeof(q.H_vel_B));
    memcpy(q.b_vel_B, o.b_vel_B, sizeof(q.b_vel_B));
    memcpy(q.H_cross_pose_vel_B, o.H_cross_pose_vel_B, sizeof(q.H_cross_pose_vel_B));
    memcpy(q.H_cross_vel_AB, o.H_cross_vel_AB, sizeof(q.H_cross_vel_AB));
  }
  return rc;
}

void kds_batch_free(kds_batch* B) { delete B; }

}  // extern "C"
