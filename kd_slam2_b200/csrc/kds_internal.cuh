// Internal definitions shared by the libkds CUDA translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/kds.h"

namespace kds {

// ---------------------------------------------------------------------------
// Error reporting: every entry point returns a status; the text goes to a
// thread-local slot read by kds_last_error().
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what, const char* file, int line);

#define KDS_CK(call)                                                      \
  do {                                                                    \
    cudaError_t _e = (call);                                              \
    if (_e != cudaSuccess) return ::kds::cuda_status(_e, #call, __FILE__, __LINE__); \
  } while (0)

// Number of kernels this library has launched (process-wide), for launch accounting.
void count_launch();

inline cudaStream_t as_stream(void* s) { return s ? (cudaStream_t)s : cudaStreamPerThread; }
int ensure_init();

// ---------------------------------------------------------------------------
// Device tree layout.
//   DNode (32 B, one sector): a = (mean.x, mean.y, mean.z, dir.x)
//                             b = (dir.y, dir.z, bits(left), bits(right))
// One descent step reads exactly one node record.
struct __align__(16) DNode {
  float4 a;
  float4 b;
};

struct TreeDev {
  int64_t num_nodes = 0;
  int64_t num_leaves = 0;
  int64_t num_points = 0;
  int64_t num_unpruned = 0;
  double ts_start = 0.0;
  int32_t depth = 0;
  int32_t accepted = 1;
  int32_t global_levels = 0;  // levels built level by level (the rest in shared-memory subtrees)
  DNode* nodes = nullptr;         // [num_nodes]
  float* dts_f = nullptr;         // [num_nodes] (float)dts_mean
  double* dts_mean = nullptr;     // [num_nodes]
  double* dts_cov = nullptr;      // [num_nodes]
  int64_t* range = nullptr;       // [2*num_nodes] idx_start, idx_end
  int32_t* level = nullptr;       // [num_nodes]
  int32_t* leaf_idx = nullptr;    // [num_leaves]
  float4* leaf_md = nullptr;      // [num_leaves] mean.xyz, (float)dts_mean
  float4* leaf_nrm = nullptr;     // [num_leaves] normal.xyz, 0
  int32_t* perm = nullptr;        // [num_points] input index at each final position
  void* block = nullptr;          // single allocation backing the arrays above
  cudaStream_t stream = nullptr;  // stream the block was allocated on (stream-ordered pool)
};

int tree_alloc(TreeDev& t, int64_t nodes, int64_t leaves, int64_t points, cudaStream_t s);
void tree_release(TreeDev& t);

// Gathers leaf_md / leaf_nrm from the node arrays (after build, import or morph).
int tree_gather_leaves(TreeDev& t, cudaStream_t s);

}  // namespace kds

struct kds_tree {
  kds::TreeDev d;
  // Tree_::root_mean / root_eigenvalues / root_eigenvectors (column-major), host copies:
  // from the build's root decision, or carried by a tree message
  float root_mean[3] = {0.f, 0.f, 0.f};
  float root_eigenvalues[3] = {0.f, 0.f, 0.f};
  float root_eigenvectors[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
};

// ---------------------------------------------------------------------------
// Exact-order single precision helpers.  Each call rounds once and is never fused,
// reproducing the CPU oracle compiled with -ffp-contract=off.
namespace kds {

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }

struct F3 {
  float x, y, z;
};
__device__ __forceinline__ F3 f3(float x, float y, float z) { F3 r; r.x = x; r.y = y; r.z = z; return r; }
// Eigen's order for a fixed-size-3 reduction: x0 + (x1 + x2)
__device__ __forceinline__ float dot3x(F3 a, F3 b) { return fa(fm(a.x, b.x), fa(fm(a.y, b.y), fm(a.z, b.z))); }
__device__ __forceinline__ F3 add3x(F3 a, F3 b) { return f3(fa(a.x, b.x), fa(a.y, b.y), fa(a.z, b.z)); }
__device__ __forceinline__ F3 sub3x(F3 a, F3 b) { return f3(fs(a.x, b.x), fs(a.y, b.y), fs(a.z, b.z)); }

// 3x4 row-major isometry in float, and a 6-vector, passed by value to kernels
struct Iso12 {
  float m[12];
};
struct Vel6 {
  float v[6];
};
// applyIsometry_ row loop: ((t + R0 p0) + R1 p1) + R2 p2 (kd/utils/geometry_.h:11-25)
__device__ __forceinline__ F3 apply_iso_x(const float* X, F3 p) {
  F3 r;
  r.x = fa(fa(fa(X[3], fm(X[0], p.x)), fm(X[1], p.y)), fm(X[2], p.z));
  r.y = fa(fa(fa(X[7], fm(X[4], p.x)), fm(X[5], p.y)), fm(X[6], p.z));
  r.z = fa(fa(fa(X[11], fm(X[8], p.x)), fm(X[9], p.y)), fm(X[10], p.z));
  return r;
}
__device__ __forceinline__ F3 apply_rot_x(const float* X, F3 p) {
  F3 r;
  r.x = fa(fa(fa(0.0f, fm(X[0], p.x)), fm(X[1], p.y)), fm(X[2], p.z));
  r.y = fa(fa(fa(0.0f, fm(X[4], p.x)), fm(X[5], p.y)), fm(X[6], p.z));
  r.z = fa(fa(fa(0.0f, fm(X[8], p.x)), fm(X[9], p.y)), fm(X[10], p.z));
  return r;
}

// Canonical sine/cosine: Cody-Waite reduction by pi/2 (three-part constant) and
// Taylor polynomials on [-pi/4, pi/4], all in explicit single roundings.
__device__ __forceinline__ void sincos_canon(float x, float* s_out, float* c_out) {
  const float two_over_pi = 0.636619772367581343f;
  float q = rintf(fm(x, two_over_pi));
  int j = (int)q;
  float r = fs(x, fm(q, 1.5703125f));
  r = fs(r, fm(q, 4.837512969970703125e-4f));
  r = fs(r, fm(q, 7.54978995489188216e-8f));
  float r2 = fm(r, r);
  float t = fm(r2, 2.75573192e-6f);
  t = fa(-1.98412698e-4f, t);
  t = fm(r2, t);
  t = fa(8.33333333e-3f, t);
  t = fm(r2, t);
  t = fa(-1.66666667e-1f, t);
  t = fm(r2, t);
  float sn = fa(r, fm(r, t));
  float u = fm(r2, -2.75573192e-7f);
  u = fa(2.48015873e-5f, u);
  u = fm(r2, u);
  u = fa(-1.38888889e-3f, u);
  u = fm(r2, u);
  u = fa(4.16666667e-2f, u);
  u = fm(r2, u);
  u = fa(-0.5f, u);
  u = fm(r2, u);
  float cs = fa(1.0f, u);
  switch (j & 3) {
    case 0: *s_out = sn; *c_out = cs; break;
    case 1: *s_out = cs; *c_out = -sn; break;
    case 2: *s_out = -sn; *c_out = -cs; break;
    default: *s_out = -cs; *c_out = sn; break;
  }
}

__device__ __forceinline__ F3 node_mean(const DNode& n) { return f3(n.a.x, n.a.y, n.a.z); }
__device__ __forceinline__ F3 node_dir(const DNode& n) { return f3(n.a.w, n.b.x, n.b.y); }
__device__ __forceinline__ int node_left(const DNode& n) { return __float_as_int(n.b.z); }
__device__ __forceinline__ int node_right(const DNode& n) { return __float_as_int(n.b.w); }
__device__ __forceinline__ DNode load_node(const DNode* p) {
  DNode n;
  const float4* q = reinterpret_cast<const float4*>(p);
  n.a = __ldg(q);
  n.b = __ldg(q + 1);
  return n;
}

}  // namespace kds

namespace kds {
// rodrigues(w) (kd/utils/geometry_3d_impl_.h:37-46) with exact single roundings and
// the canonical sine/cosine; R row-major.
__device__ __forceinline__ void rodrigues_x(F3 w, float* R) {
  float angle = __fsqrt_rn(dot3x(w, w));
  if (angle < 1e-9f) {
#pragma unroll
    for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1.0f : 0.0f;
    return;
  }
  float inv = __fdiv_rn(1.0f, angle);
  F3 n = f3(fm(w.x, inv), fm(w.y, inv), fm(w.z, inv));
  float S[9] = {0.0f, -n.z, n.y, n.z, 0.0f, -n.x, -n.y, n.x, 0.0f};
  float S2[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      S2[i * 3 + j] = dot3x(f3(S[i * 3], S[i * 3 + 1], S[i * 3 + 2]), f3(S[j], S[3 + j], S[6 + j]));
  float s, c;
  sincos_canon(angle, &s, &c);
  float omc = fs(1.0f, c);
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    float id = (i % 4 == 0) ? 1.0f : 0.0f;
    R[i] = fa(fa(id, fm(s, S[i])), fm(omc, S2[i]));
  }
}
__device__ __forceinline__ F3 mat_vec_x(const float* R, F3 p) {
  return f3(dot3x(f3(R[0], R[1], R[2]), p), dot3x(f3(R[3], R[4], R[5]), p), dot3x(f3(R[6], R[7], R[8]), p));
}
// CTICP_3D_Traits::applyVelocities (kd/d3/cticp_impl_.h:75-85): m' = R(w dt) m + v dt, n' = R n
__device__ __forceinline__ void warp_x(const float* v, float dt, F3 m, F3 n, F3& mo, F3& no) {
  F3 td = f3(fm(v[0], dt), fm(v[1], dt), fm(v[2], dt));
  F3 rd = f3(fm(v[3], dt), fm(v[4], dt), fm(v[5], dt));
  float R[9];
  rodrigues_x(rd, R);
  mo = add3x(mat_vec_x(R, m), td);
  no = mat_vec_x(R, n);
}
}  // namespace kds

namespace kds {
// Exclusive scan of n int32 (kds_tree.cu); tile_sums needs n / 4096 + 2 entries.
int scan_exclusive(const int32_t* in, int32_t* out, int32_t n, int32_t* tile_sums, int32_t* total, cudaStream_t s);
// Tree build (kds_build.cu)
int tree_build_forest(const float* xyz, const double* stamps, const int64_t* offsets, int32_t R, int32_t mem,
                      const kds_tree_params* prm, cudaStream_t s, kds_tree** out, int32_t* status);
// Tree operations (kds_tree.cu / kds_build.cu)
int tree_build(const float* xyz, const double* stamps, int64_t n, int32_t mem, const kds_tree_params* p,
               cudaStream_t s, kds_tree** out);
int tree_import(const float* mean, const float* dir, const double* dts_mean, const double* dts_cov,
                const int64_t* s0, const int64_t* e0, const int32_t* left, const int32_t* right, int64_t num_nodes,
                double ts_start, kds_tree** out);
int tree_apply_velocities(kds_tree* t, const float* v, int skip_leaves, cudaStream_t s);
int tree_apply_isometry(kds_tree* t, const float* X, cudaStream_t s);
int tree_extract_leaves(const kds_tree* t, const float* v6, float* out_host, float* out_device, cudaStream_t s);
int tree_from_msg(const kds_kdtree3f* msg, kds_tree** out);
int tree_clone(const kds_tree* src, cudaStream_t s, kds_tree** out);
int points_voxelize(const float* xyz, const double* stamps, int64_t n, int32_t mem, double msg_t,
                    double scan_duration, const kds_voxel_params* prm, cudaStream_t s, float* out_xyz,
                    double* out_stamps, int64_t* out_n);
int tree_export(const kds_tree* t, float* mean, float* dir, double* dts_mean, double* dts_cov, int64_t* s0,
                int64_t* e0, int32_t* left, int32_t* right, int32_t* level, int64_t* leaves, int64_t* perm);
}  // namespace kds
