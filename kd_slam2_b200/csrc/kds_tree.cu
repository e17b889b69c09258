// GPU surfel KD-tree: build, import/export, morph.  Compiled with -fmad=false so that
// every double/float expression rounds each multiply and add separately, as the CPU
// oracle does; the build is then bit-identical to it.
//
// Build (replaces TreeGenerator_::makeTree, kd/tree/tree_generator_impl_.h:7-19, which
// the reference runs on the CPU only): level-synchronous over the tree.
//   * Per node moments [xx,xy,xz,yy,yz,zz,x,y,z,dt,dt^2] are exact-order-free 128-bit
//     fixed-point sums (each double product floored onto a 2^-64 grid), so warps,
//     blocks and atomics may add them in any order.
//   * FP64 covariance, cyclic Jacobi eigensolver, FlatLeafPolicy_ decision
//     (kd/tree/flat_leaf_policy_.h:52-108) in FP64.
//   * Stable partition by Node_::whichSide in float (kd/tree/node_.h:53-56).
//   * Children are numbered by an exclusive scan over the level's split flags, so the
//     node array is in BFS order; prune keeps BFS order (kd/tree/tree_cpu_.h:172-207).
// Small nodes (<= kBig points) are handled by one warp each; large nodes by chunks of
// kChunk points per block with 128-bit atomics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "kds_internal.cuh"

namespace kds {

namespace {

constexpr int kBig = 2048;
constexpr int kChunk = 2048;
constexpr int kBuildThreads = 256;

// ---------------------------------------------------------------------------
// 128-bit fixed point as two 64-bit words (two's complement).
struct U128 {
  unsigned long long lo, hi;
};
__host__ __device__ __forceinline__ U128 u128_zero() { U128 r; r.lo = 0ull; r.hi = 0ull; return r; }
__host__ __device__ __forceinline__ U128 u128_add(U128 a, U128 b) {
  U128 r;
  r.lo = a.lo + b.lo;
  r.hi = a.hi + b.hi + (r.lo < a.lo ? 1ull : 0ull);
  return r;
}
// floor(v * 2^64) split into signed high word and unsigned low word
__device__ __forceinline__ U128 fx_of(double v) {
  double hi = floor(v);
  double lo = (v - hi) * 0x1p64;
  U128 r;
  r.hi = (unsigned long long)__double2ll_rz(hi);
  r.lo = __double2ull_rz(lo);
  return r;
}
__host__ __device__ __forceinline__ double fx_to_d(U128 q) {
  long long hi = (long long)q.hi;
  return ((double)hi * 0x1p64 + (double)q.lo) * 0x1p-64;
}
__device__ __forceinline__ U128 shfl_xor_u128(U128 v, int m) {
  U128 r;
  r.lo = __shfl_xor_sync(0xffffffffu, v.lo, m);
  r.hi = __shfl_xor_sync(0xffffffffu, v.hi, m);
  return r;
}
__device__ __forceinline__ void atomic_add_u128(U128* dst, U128 v) {
  unsigned long long old = atomicAdd(&dst->lo, v.lo);
  unsigned long long carry = (old + v.lo < old) ? 1ull : 0ull;
  atomicAdd(&dst->hi, v.hi + carry);
}

struct Moments {
  U128 s[11];
};

__device__ __forceinline__ void moments_add_point(Moments& M, float4 p, double st, double ts_start) {
  double x = p.x, y = p.y, z = p.z;
  M.s[0] = u128_add(M.s[0], fx_of(x * x));
  M.s[1] = u128_add(M.s[1], fx_of(x * y));
  M.s[2] = u128_add(M.s[2], fx_of(x * z));
  M.s[3] = u128_add(M.s[3], fx_of(y * y));
  M.s[4] = u128_add(M.s[4], fx_of(y * z));
  M.s[5] = u128_add(M.s[5], fx_of(z * z));
  M.s[6] = u128_add(M.s[6], fx_of(x));
  M.s[7] = u128_add(M.s[7], fx_of(y));
  M.s[8] = u128_add(M.s[8], fx_of(z));
  double dt = st - ts_start;
  M.s[9] = u128_add(M.s[9], fx_of(dt));
  M.s[10] = u128_add(M.s[10], fx_of(dt * dt));
}

// ---------------------------------------------------------------------------
// Build-time node record.
struct BNode {
  int32_t start, end;
  int32_t level;
  int32_t split;      // 1: inner node
  int32_t mid;
  int32_t left, right;
  int32_t has_parent;
  int32_t par_has;    // propagated normal received from the parent
  int32_t has_prop;   // propagated normal handed to the children
  float mean[3], dir[3];
  double dts_mean, dts_cov;
  double prop[3];
  double par_prop[3];
};

struct BuildParams {
  int32_t propagate_normal;
  int32_t leaf_min_points;
  int32_t leaf_max_points;
  float leaf_density;
  float leaf_min_normal_incidence;
  float leaf_normal_eigenratio;
  float prune_incidence;
  int32_t max_level;
};

__device__ __forceinline__ double ddot3(const double* a, const double* b) {
  double p0 = a[0] * b[0], p1 = a[1] * b[1], p2 = a[2] * b[2];
  return p0 + (p1 + p2);
}

// Cyclic Jacobi eigensolver for a symmetric 3x3 (Golub & Van Loan, sec. 8.5), fixed
// 8 sweeps; eigenvalues ascending, eigenvectors as columns of V.
__device__ void jacobi3(const double Ain[3][3], double ev[3], double V[3][3]) {
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) { a[i][j] = Ain[i][j]; V[i][j] = (i == j) ? 1.0 : 0.0; }
  for (int sweep = 0; sweep < 8; ++sweep) {
    for (int pq = 0; pq < 3; ++pq) {
      int p = (pq == 2) ? 1 : 0;
      int q = (pq == 0) ? 1 : 2;
      int r = 3 - p - q;
      double apq = a[p][q];
      if (apq == 0.0) continue;
      double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
      double t = 1.0 / (fabs(theta) + sqrt(theta * theta + 1.0));
      if (theta < 0.0) t = -t;
      double c = 1.0 / sqrt(t * t + 1.0);
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
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) V[i][j] = Vs[i][j];
}

// FlatLeafPolicy_::fillMetadata over CountLeafPolicy_ and LabelPolicyBase_
// (kd/tree/flat_leaf_policy_.h:52-108, count_leaf_policy_.h:27-43,
// label_policy_base_impl_.h:12-97), FP64 statistics.
__device__ void decide(const Moments& M, int64_t n, BNode& nd, const BuildParams& P) {
  for (int i = 0; i < 3; ++i) { nd.mean[i] = 0.f; nd.dir[i] = 0.f; }
  nd.dts_mean = 0.0;
  nd.dts_cov = 0.0;
  double mean_d[3] = {0, 0, 0};
  double e0[3] = {0, 0, 0}, e2[3] = {0, 0, 0};
  double lam[3] = {0, 0, 0};
  bool is_bad = true;
  if (n > 0) {
    double dn = (double)n;
    double Sd[11];
    for (int k = 0; k < 11; ++k) Sd[k] = fx_to_d(M.s[k]);
    nd.dts_mean = Sd[9] / dn;
    nd.dts_cov = Sd[10] / dn - nd.dts_mean * nd.dts_mean;
    for (int i = 0; i < 3; ++i) mean_d[i] = Sd[6 + i] / dn;
    for (int i = 0; i < 3; ++i) nd.mean[i] = (float)mean_d[i];
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
    }
  }
  bool is_node = false, is_leaf = false;
  if (is_bad) {
    is_leaf = true;
  } else if ((float)n > (float)P.leaf_max_points) {
    is_node = true;
    for (int i = 0; i < 3; ++i) nd.dir[i] = (float)e2[i];
  } else {
    is_leaf = true;
    for (int i = 0; i < 3; ++i) nd.dir[i] = (float)e0[i];
  }
  bool has_prop = false;
  double prop[3] = {0, 0, 0};
  if (nd.has_parent && P.propagate_normal) {
    has_prop = nd.par_has != 0;
    for (int i = 0; i < 3; ++i) prop[i] = nd.par_prop[i];
  }
  bool is_flat = false;
  bool do_prop = false;
  if (is_bad || (float)n < (float)P.leaf_min_points) {
    do_prop = true;
  } else {
    double eigenratio = lam[0] / lam[2];
    is_flat = eigenratio < (double)P.leaf_normal_eigenratio &&
              fabs(ddot3(mean_d, e0)) > (double)P.leaf_min_normal_incidence;
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
        for (int i = 0; i < 3; ++i) nd.dir[i] = (float)e2[i];
      } else if (is_leaf && is_flat) {
        for (int i = 0; i < 3; ++i) nd.dir[i] = (float)e0[i];
      } else {
        do_prop = true;
      }
    }
  }
  if (do_prop) {
    is_leaf = true;
    if (has_prop) {
      double d[3] = {prop[0], prop[1], prop[2]};
      if (ddot3(mean_d, d) > 0.0) for (int i = 0; i < 3; ++i) d[i] = -d[i];
      for (int i = 0; i < 3; ++i) nd.dir[i] = (float)d[i];
    }
  }
  if (is_node && nd.level >= P.max_level - 1) {
    is_node = false;
    if (is_flat) {
      for (int i = 0; i < 3; ++i) nd.dir[i] = (float)e0[i];
    } else if (has_prop) {
      double d[3] = {prop[0], prop[1], prop[2]};
      if (ddot3(mean_d, d) > 0.0) for (int i = 0; i < 3; ++i) d[i] = -d[i];
      for (int i = 0; i < 3; ++i) nd.dir[i] = (float)d[i];
    } else {
      for (int i = 0; i < 3; ++i) nd.dir[i] = (float)e0[i];
    }
  }
  nd.split = is_node ? 1 : 0;
  nd.has_prop = has_prop ? 1 : 0;
  for (int i = 0; i < 3; ++i) nd.prop[i] = prop[i];
}

__device__ __forceinline__ bool which_side_f(const float* mean, const float* dir, float4 q) {
  F3 d = sub3x(f3(q.x, q.y, q.z), f3(mean[0], mean[1], mean[2]));
  return dot3x(f3(dir[0], dir[1], dir[2]), d) > 0.0f;
}

struct LevelStatus {
  int32_t next_count;   // nodes at the next level
  int32_t max_size;     // largest node at the next level
  int32_t error;        // 1: node capacity exceeded, 2: input out of range
  int32_t pad;
};

// ---------------------------------------------------------------------------
// Kernels

// Input conversion + validation: float xyz (3 per point) -> float4, stamps, ids.
__global__ void k_ingest(const float* xyz, const double* st, int64_t n, float4* pts, double* sts, int32_t* ids,
                         LevelStatus* status) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    double s = st ? st[i] : 0.0;
    bool ok = fabsf(x) < 32768.f && fabsf(y) < 32768.f && fabsf(z) < 32768.f && isfinite(s);
    if (!ok) status->error = 2;
    pts[i] = make_float4(x, y, z, 0.f);
    sts[i] = s;
    ids[i] = (int32_t)i;
  }
}

// Minimum timestamp (root ts_start, label_policy_base_impl_.h:28-35); one block.
__global__ void k_ts_min(const double* sts, int64_t n, double* out, LevelStatus* status) {
  __shared__ double sm[1024];
  double m = 1.0e308;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) m = fmin(m, sts[i]);
  sm[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sm[threadIdx.x] = fmin(sm[threadIdx.x], sm[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = (n > 0) ? sm[0] : 0.0;
}

__global__ void k_dt_check(const double* sts, int64_t n, const double* ts0, LevelStatus* status) {
  double t0 = *ts0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double dt = sts[i] - t0;
    if (!(dt < 65536.0)) status->error = 2;
  }
}

// One warp per small node of the level: moments, decision, stable partition.
__global__ void k_small_nodes(BNode* nodes, int32_t lb, int32_t le, const float4* pts_in, const double* st_in,
                              const int32_t* id_in, float4* pts_out, double* st_out, int32_t* id_out,
                              int32_t* perm_final, const double* ts0p, BuildParams P) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  int ni = lb + warp;
  if (ni >= le) return;
  BNode nd = nodes[ni];
  int s = nd.start, e = nd.end;
  int n = e - s;
  if (n > kBig) return;
  double ts0 = *ts0p;
  Moments M;
  for (int k = 0; k < 11; ++k) M.s[k] = u128_zero();
  for (int i = s + lane; i < e; i += 32) moments_add_point(M, pts_in[i], st_in[i], ts0);
  for (int off = 16; off > 0; off >>= 1)
    for (int k = 0; k < 11; ++k) M.s[k] = u128_add(M.s[k], shfl_xor_u128(M.s[k], off));
  decide(M, n, nd, P);
  if (nd.split) {
    int nl = 0;
    for (int base = s; base < e; base += 32) {
      int i = base + lane;
      bool left = false;
      if (i < e) left = which_side_f(nd.mean, nd.dir, pts_in[i]);
      nl += __popc(__ballot_sync(0xffffffffu, left));
    }
    int cl = 0, cr = 0;
    unsigned lt = (1u << lane) - 1u;
    for (int base = s; base < e; base += 32) {
      int i = base + lane;
      bool valid = i < e;
      bool left = false;
      float4 p;
      if (valid) { p = pts_in[i]; left = which_side_f(nd.mean, nd.dir, p); }
      unsigned bl = __ballot_sync(0xffffffffu, valid && left);
      unsigned br = __ballot_sync(0xffffffffu, valid && !left);
      if (valid) {
        int dst = left ? (s + cl + __popc(bl & lt)) : (s + nl + cr + __popc(br & lt));
        pts_out[dst] = p;
        st_out[dst] = st_in[i];
        id_out[dst] = id_in[i];
      }
      cl += __popc(bl);
      cr += __popc(br);
    }
    nd.mid = s + nl;
  } else {
    for (int i = s + lane; i < e; i += 32) perm_final[i] = id_in[i];
    nd.mid = e;
  }
  if (lane == 0) nodes[ni] = nd;
}

// ---- large nodes --------------------------------------------------------------
struct Chunk {
  int32_t node;
  int32_t begin;
  int32_t end;
  int32_t big;  // ordinal of the node among the level's large nodes
};

// One block: lists the level's large nodes and their chunks.
__global__ void k_big_plan(const BNode* nodes, int32_t lb, int32_t le, Chunk* chunks, int32_t chunk_cap,
                           int32_t* num_chunks, int32_t* big_list, int32_t* num_big, int32_t* node_chunk0,
                           U128* acc) {
  if (threadIdx.x != 0) return;
  int nc = 0, nb = 0;
  for (int i = lb; i < le; ++i) {
    int s = nodes[i].start, e = nodes[i].end;
    if (e - s <= kBig) continue;
    big_list[nb] = i;
    node_chunk0[nb] = nc;
    for (int b = s; b < e; b += kChunk) {
      if (nc < chunk_cap) {
        chunks[nc].node = i;
        chunks[nc].begin = b;
        chunks[nc].end = min(b + kChunk, e);
        chunks[nc].big = nb;
      }
      ++nc;
    }
    for (int k2 = 0; k2 < 11; ++k2) acc[(size_t)nb * 11 + k2] = u128_zero();
    ++nb;
  }
  *num_chunks = nc;
  *num_big = nb;
}

__global__ void k_big_moments(const Chunk* chunks, const int32_t* num_chunks, int32_t lb, const float4* pts,
                              const double* st, const double* ts0p, U128* acc) {
  if (blockIdx.x >= *num_chunks) return;
  Chunk c = chunks[blockIdx.x];
  double ts0 = *ts0p;
  Moments M;
  for (int k = 0; k < 11; ++k) M.s[k] = u128_zero();
  for (int i = c.begin + threadIdx.x; i < c.end; i += blockDim.x) moments_add_point(M, pts[i], st[i], ts0);
  for (int off = 16; off > 0; off >>= 1)
    for (int k = 0; k < 11; ++k) M.s[k] = u128_add(M.s[k], shfl_xor_u128(M.s[k], off));
  __shared__ U128 sm[kBuildThreads / 32][11];
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int k = 0; k < 11; ++k) sm[w][k] = M.s[k];
  __syncthreads();
  if (threadIdx.x < 11) {
    U128 t = u128_zero();
    for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) t = u128_add(t, sm[ww][threadIdx.x]);
    atomic_add_u128(&acc[(size_t)c.big * 11 + threadIdx.x], t);
  }
}

__global__ void k_big_decide(BNode* nodes, int32_t lb, const int32_t* big_list, const int32_t* num_big,
                             const U128* acc, BuildParams P) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= *num_big) return;
  int i = big_list[t];
  BNode nd = nodes[i];
  Moments M;
  for (int k = 0; k < 11; ++k) M.s[k] = acc[(size_t)t * 11 + k];
  decide(M, nd.end - nd.start, nd, P);
  nodes[i] = nd;
}

// per chunk: number of points going left
__global__ void k_big_count(const Chunk* chunks, const int32_t* num_chunks, const BNode* nodes, const float4* pts,
                            int32_t* chunk_nl) {
  if (blockIdx.x >= *num_chunks) return;
  Chunk c = chunks[blockIdx.x];
  const BNode& nd = nodes[c.node];
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int local = 0;
  if (nd.split)
    for (int i = c.begin + threadIdx.x; i < c.end; i += blockDim.x) local += which_side_f(nd.mean, nd.dir, pts[i]) ? 1 : 0;
  atomicAdd(&cnt, local);
  __syncthreads();
  if (threadIdx.x == 0) chunk_nl[blockIdx.x] = cnt;
}

// one block: per large node, chunk offsets and split position
__global__ void k_big_offsets(const Chunk* chunks, const int32_t* num_chunks, BNode* nodes, const int32_t* big_list,
                              const int32_t* num_big, const int32_t* node_chunk0, const int32_t* chunk_nl,
                              int32_t* chunk_loff) {
  for (int b = threadIdx.x; b < *num_big; b += blockDim.x) {
    int i = big_list[b];
    int c0 = node_chunk0[b];
    int c1 = (b + 1 < *num_big) ? node_chunk0[b + 1] : *num_chunks;
    int acc = 0;
    for (int c = c0; c < c1; ++c) { chunk_loff[c] = acc; acc += chunk_nl[c]; }
    BNode& nd = nodes[i];
    nd.mid = nd.split ? nd.start + acc : nd.end;
  }
}

// stable scatter of one chunk: each thread owns a contiguous run of points
__global__ void k_big_scatter(const Chunk* chunks, const int32_t* num_chunks, const BNode* nodes, const float4* pts_in,
                              const double* st_in, const int32_t* id_in, float4* pts_out, double* st_out,
                              int32_t* id_out, int32_t* perm_final, const int32_t* chunk_loff) {
  if (blockIdx.x >= *num_chunks) return;
  Chunk c = chunks[blockIdx.x];
  const BNode& nd = nodes[c.node];
  int len = c.end - c.begin;
  if (!nd.split) {
    for (int i = c.begin + threadIdx.x; i < c.end; i += blockDim.x) perm_final[i] = id_in[i];
    return;
  }
  int per = (len + blockDim.x - 1) / blockDim.x;
  int b0 = c.begin + threadIdx.x * per;
  int b1 = min(b0 + per, c.end);
  int mine = 0;
  for (int i = b0; i < b1; ++i) mine += which_side_f(nd.mean, nd.dir, pts_in[i]) ? 1 : 0;
  __shared__ int sc[kBuildThreads];
  sc[threadIdx.x] = mine;
  __syncthreads();
  // inclusive Hillis-Steele scan
  for (int off = 1; off < (int)blockDim.x; off <<= 1) {
    int v = (threadIdx.x >= (unsigned)off) ? sc[threadIdx.x - off] : 0;
    __syncthreads();
    sc[threadIdx.x] += v;
    __syncthreads();
  }
  int lbefore = sc[threadIdx.x] - mine;
  int loff = chunk_loff[blockIdx.x] + lbefore;                      // lefts before my run within the node
  int pbefore = (c.begin - nd.start) + (b0 - c.begin);              // points before my run within the node
  int roff = pbefore - loff;                                        // rights before my run within the node
  int nl_total = nd.mid - nd.start;
  for (int i = b0; i < b1; ++i) {
    float4 p = pts_in[i];
    int dst;
    if (which_side_f(nd.mean, nd.dir, p)) dst = nd.start + loff++;
    else dst = nd.start + nl_total + roff++;
    pts_out[dst] = p;
    st_out[dst] = st_in[i];
    id_out[dst] = id_in[i];
  }
}

// ---- level bookkeeping ----------------------------------------------------------
// Exclusive scan over int32 with a fixed two-level structure (deterministic).
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;  // per thread
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int block_excl_scan(int v, int* sm, int* total) {
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
  for (int off = 1; off < 32; off <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) sm[w] = x;
  __syncthreads();
  if (w == 0) {
    int nw = blockDim.x >> 5;
    int y = (lane < nw) ? sm[lane] : 0;
    for (int off = 1; off < 32; off <<= 1) {
      int z = __shfl_up_sync(0xffffffffu, y, off);
      if (lane >= off) y += z;
    }
    if (lane < nw) sm[lane] = y;
  }
  __syncthreads();
  int wprefix = (w > 0) ? sm[w - 1] : 0;
  *total = sm[(blockDim.x >> 5) - 1];
  __syncthreads();
  return wprefix + x - v;
}

// flag for scan: split nodes of the level (op 0) / alive nodes (op 1) / alive leaves (op 2)
__global__ void k_scan_tiles(const int32_t* in, int32_t n, int32_t* tile_sums) {
  __shared__ int sm[32];
  int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v = 0;
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) v += in[base + k];
  int total;
  block_excl_scan(v, sm, &total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}
__global__ void k_scan_top(int32_t* tile_sums, int32_t ntiles, int32_t* total_out) {
  __shared__ int sm[32];
  // sequential over chunks of blockDim.x
  int carry = 0;
  for (int b = 0; b < ntiles; b += blockDim.x) {
    int i = b + threadIdx.x;
    int v = (i < ntiles) ? tile_sums[i] : 0;
    int tot;
    int ex = block_excl_scan(v, sm, &tot);
    if (i < ntiles) tile_sums[i] = carry + ex;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total_out = carry;
}
__global__ void k_scan_apply(const int32_t* in, int32_t n, const int32_t* tile_sums, int32_t* out) {
  __shared__ int sm[32];
  int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int vals[kScanItems];
  int v = 0;
  for (int k = 0; k < kScanItems; ++k) {
    vals[k] = (base + k < n) ? in[base + k] : 0;
    v += vals[k];
  }
  int total;
  int ex = block_excl_scan(v, sm, &total) + tile_sums[blockIdx.x];
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = ex;
    ex += vals[k];
  }
}

__global__ void k_split_flags(const BNode* nodes, int32_t lb, int32_t le, int32_t* flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (lb + i < le) flags[i] = nodes[lb + i].split ? 1 : 0;
}

__global__ void k_make_children(BNode* nodes, int32_t lb, int32_t le, const int32_t* rank, int32_t cap,
                                LevelStatus* status) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (lb + i >= le) return;
  BNode& nd = nodes[lb + i];
  if (!nd.split) {
    nd.left = -1;
    nd.right = -1;
    return;
  }
  int li = le + 2 * rank[i];
  if (li + 1 >= cap) {
    status->error = 1;
    nd.split = 0;
    nd.left = nd.right = -1;
    return;
  }
  nd.left = li;
  nd.right = li + 1;
  for (int k = 0; k < 2; ++k) {
    BNode c;
    memset(&c, 0, sizeof(c));
    c.start = k == 0 ? nd.start : nd.mid;
    c.end = k == 0 ? nd.mid : nd.end;
    c.level = nd.level + 1;
    c.left = c.right = -1;
    c.has_parent = 1;
    c.par_has = nd.has_prop;
    for (int j = 0; j < 3; ++j) c.par_prop[j] = nd.prop[j];
    nodes[li + k] = c;
    atomicMax(&status->max_size, c.end - c.start);
  }
}

// ---- prune and compaction -----------------------------------------------------------
__global__ void k_alive(const BNode* nodes, int32_t lb, int32_t le, int32_t* alive, float incidence) {
  int i = lb + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= le) return;
  const BNode& nd = nodes[i];
  int a;
  if (nd.left < 0 && nd.right < 0) {
    // IsGoodLeafPredicate_ in float (kd/tree/tree_predicates_.h:18-29)
    F3 d = f3(nd.dir[0], nd.dir[1], nd.dir[2]);
    F3 m = f3(nd.mean[0], nd.mean[1], nd.mean[2]);
    bool ok = dot3x(d, d) > 0.0f && fabsf(dot3x(m, d)) > incidence;
    a = ok ? 1 : 0;
  } else {
    a = ((nd.left >= 0 && alive[nd.left]) || (nd.right >= 0 && alive[nd.right])) ? 1 : 0;
  }
  alive[i] = a;
}

__global__ void k_leaf_flags(const BNode* nodes, int32_t n, const int32_t* alive, int32_t* leaf_flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  leaf_flag[i] = (alive[i] && nodes[i].left < 0 && nodes[i].right < 0) ? 1 : 0;
}

__global__ void k_compact(const BNode* nodes, int32_t n, const int32_t* alive, const int32_t* newidx,
                          const int32_t* leaf_flag, const int32_t* leaf_rank, TreeDev t) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !alive[i]) return;
  const BNode& nd = nodes[i];
  int o = newidx[i];
  int l = (nd.left >= 0 && alive[nd.left]) ? newidx[nd.left] : -1;
  int r = (nd.right >= 0 && alive[nd.right]) ? newidx[nd.right] : -1;
  DNode d;
  d.a = make_float4(nd.mean[0], nd.mean[1], nd.mean[2], nd.dir[0]);
  d.b = make_float4(nd.dir[1], nd.dir[2], __int_as_float(l), __int_as_float(r));
  t.nodes[o] = d;
  t.dts_f[o] = (float)nd.dts_mean;
  t.dts_mean[o] = nd.dts_mean;
  t.dts_cov[o] = nd.dts_cov;
  t.range[2 * o] = nd.start;
  t.range[2 * o + 1] = nd.end;
  t.level[o] = nd.level;
  if (leaf_flag[i]) t.leaf_idx[leaf_rank[i]] = o;
}

__global__ void k_gather_leaves(TreeDev t) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= t.num_leaves) return;
  int o = t.leaf_idx[i];
  DNode d = t.nodes[o];
  t.leaf_md[i] = make_float4(d.a.x, d.a.y, d.a.z, t.dts_f[o]);
  t.leaf_nrm[i] = make_float4(d.a.w, d.b.x, d.b.y, 0.f);
}

__global__ void k_copy_perm(const int32_t* src, int32_t* dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

// ---- morph / transform --------------------------------------------------------------
__global__ void k_apply_velocities(TreeDev t, Vel6 v, int skip_leaves) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= t.num_nodes) return;
  DNode d = t.nodes[i];
  bool leaf = node_left(d) < 0 && node_right(d) < 0;
  if (leaf && skip_leaves) return;
  F3 mo, no;
  warp_x(v.v, t.dts_f[i], node_mean(d), node_dir(d), mo, no);
  d.a = make_float4(mo.x, mo.y, mo.z, no.x);
  d.b.x = no.y;
  d.b.y = no.z;
  t.nodes[i] = d;
}

__global__ void k_apply_isometry(TreeDev t, Iso12 X) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= t.num_nodes) return;
  DNode d = t.nodes[i];
  F3 mo = apply_iso_x(X.m, node_mean(d));
  F3 no = apply_rot_x(X.m, node_dir(d));
  d.a = make_float4(mo.x, mo.y, mo.z, no.x);
  d.b.x = no.y;
  d.b.y = no.z;
  t.nodes[i] = d;
}

__global__ void k_extract_leaves(TreeDev t, Vel6 v, int use_v, float* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= t.num_leaves) return;
  int o = t.leaf_idx[i];
  DNode d = t.nodes[o];
  F3 m = node_mean(d), n = node_dir(d);
  if (use_v) warp_x(v.v, t.dts_f[o], m, n, m, n);
  out[6 * i + 0] = m.x; out[6 * i + 1] = m.y; out[6 * i + 2] = m.z;
  out[6 * i + 3] = n.x; out[6 * i + 4] = n.y; out[6 * i + 5] = n.z;
}

__global__ void k_import(TreeDev t, const float* mean, const float* dir, const double* dts_mean, const double* dts_cov,
                         const int64_t* s0, const int64_t* e0, const int32_t* left, const int32_t* right,
                         int32_t* bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= t.num_nodes) return;
  int l = left[i], r = right[i];
  if (l >= t.num_nodes || r >= t.num_nodes || (l >= 0 && l <= i) || (r >= 0 && r <= i)) *bad = 1;
  DNode d;
  d.a = make_float4(mean[3 * i], mean[3 * i + 1], mean[3 * i + 2], dir[3 * i]);
  d.b = make_float4(dir[3 * i + 1], dir[3 * i + 2], __int_as_float(l), __int_as_float(r));
  t.nodes[i] = d;
  double dm = dts_mean ? dts_mean[i] : 0.0;
  t.dts_mean[i] = dm;
  t.dts_f[i] = (float)dm;
  t.dts_cov[i] = dts_cov ? dts_cov[i] : 0.0;
  t.range[2 * i] = s0 ? s0[i] : 0;
  t.range[2 * i + 1] = e0 ? e0[i] : 0;
  t.level[i] = 0;
}

__global__ void k_leaf_flags_plain(const DNode* nodes, int32_t n, int32_t* flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  DNode d = nodes[i];
  flag[i] = (node_left(d) < 0 && node_right(d) < 0) ? 1 : 0;
}
__global__ void k_leaf_scatter_plain(const int32_t* flag, const int32_t* rank, int32_t n, int32_t* leaf_idx) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (flag[i]) leaf_idx[rank[i]] = i;
}

inline int nblk(int64_t n, int t) { return (int)std::max<int64_t>(1, (n + t - 1) / t); }

// Exclusive scan of n int32 into out; *total receives the sum (device).
int scan_exclusive(const int32_t* in, int32_t* out, int32_t n, int32_t* tile_sums, int32_t* total,
                   cudaStream_t s) {
  int nt = nblk(n, kScanTile);
  k_scan_tiles<<<nt, kScanThreads, 0, s>>>(in, n, tile_sums);
  k_scan_top<<<1, kScanThreads, 0, s>>>(tile_sums, nt, total);
  k_scan_apply<<<nt, kScanThreads, 0, s>>>(in, n, tile_sums, out);
  KDS_CK(cudaGetLastError());
  return KDS_OK;
}

template <class T> T* carve(char*& p, size_t count) {
  size_t bytes = (count * sizeof(T) + 255) & ~(size_t)255;
  T* r = reinterpret_cast<T*>(p);
  p += bytes;
  return r;
}
template <class T> size_t carve_size(size_t count) { return (count * sizeof(T) + 255) & ~(size_t)255; }

}  // namespace

// ---------------------------------------------------------------------------
int tree_alloc(TreeDev& t, int64_t nodes, int64_t leaves, int64_t points) {
  size_t bytes = carve_size<DNode>(nodes) + carve_size<float>(nodes) + 2 * carve_size<double>(nodes) +
                 carve_size<int64_t>(2 * nodes) + carve_size<int32_t>(nodes) + carve_size<int32_t>(leaves) +
                 2 * carve_size<float4>(leaves) + carve_size<int32_t>(points) + 256;
  void* blk = nullptr;
  cudaError_t e = cudaMalloc(&blk, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("cudaMalloc of %zu bytes for a tree failed: %s", bytes, cudaGetErrorString(e));
    return KDS_ERR_OOM;
  }
  char* p = (char*)blk;
  t.block = blk;
  t.nodes = carve<DNode>(p, nodes);
  t.dts_f = carve<float>(p, nodes);
  t.dts_mean = carve<double>(p, nodes);
  t.dts_cov = carve<double>(p, nodes);
  t.range = carve<int64_t>(p, 2 * nodes);
  t.level = carve<int32_t>(p, nodes);
  t.leaf_idx = carve<int32_t>(p, leaves);
  t.leaf_md = carve<float4>(p, leaves);
  t.leaf_nrm = carve<float4>(p, leaves);
  t.perm = points > 0 ? carve<int32_t>(p, points) : nullptr;
  t.num_nodes = nodes;
  t.num_leaves = leaves;
  t.num_points = points;
  return KDS_OK;
}

void tree_release(TreeDev& t) {
  if (t.block) cudaFree(t.block);
  t = TreeDev();
}

int tree_gather_leaves(TreeDev& t, cudaStream_t s) {
  if (t.num_leaves == 0) return KDS_OK;
  k_gather_leaves<<<nblk(t.num_leaves, 256), 256, 0, s>>>(t);
  KDS_CK(cudaGetLastError());
  return KDS_OK;
}

// ---------------------------------------------------------------------------
// Build workspace (per call; sized from the point count).
namespace {
struct BuildWs {
  void* block = nullptr;
  float4 *pa, *pb;
  double *sa, *sb;
  int32_t *ia, *ib;
  int32_t* perm_final;
  BNode* nodes;
  int32_t* flags;
  int32_t* rank;
  int32_t* tile_sums;
  int32_t* alive;
  int32_t* leaf_flag;
  int32_t* leaf_rank;
  Chunk* chunks;
  int32_t* chunk_nl;
  int32_t* chunk_loff;
  int32_t* big_list;
  int32_t* node_chunk0;
  U128* acc;
  double* ts0;
  int32_t* counters;  // [0] num_chunks, [1] num_big, [2] total (scan), [3] total2
  LevelStatus* status;
  int64_t cap_nodes;
  int32_t chunk_cap;
};

int ws_alloc(BuildWs& w, int64_t n) {
  w.cap_nodes = 2 * n + 4096;
  w.chunk_cap = (int32_t)(n / kChunk + n / kBig + 16);
  int64_t cn = w.cap_nodes;
  int64_t ntiles = cn / kScanTile + 2;
  size_t bytes = 2 * carve_size<float4>(n) + 2 * carve_size<double>(n) + 3 * carve_size<int32_t>(n) +
                 carve_size<BNode>(cn) + 5 * carve_size<int32_t>(cn) + carve_size<int32_t>(ntiles) +
                 carve_size<Chunk>(w.chunk_cap) + 4 * carve_size<int32_t>(w.chunk_cap) +
                 carve_size<U128>((size_t)11 * (n / kBig + 2)) + carve_size<double>(1) + carve_size<int32_t>(8) +
                 carve_size<LevelStatus>(1) + 256;
  cudaError_t e = cudaMalloc(&w.block, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("cudaMalloc of %zu bytes for the tree build workspace failed: %s", bytes, cudaGetErrorString(e));
    return KDS_ERR_OOM;
  }
  char* p = (char*)w.block;
  w.pa = carve<float4>(p, n);
  w.pb = carve<float4>(p, n);
  w.sa = carve<double>(p, n);
  w.sb = carve<double>(p, n);
  w.ia = carve<int32_t>(p, n);
  w.ib = carve<int32_t>(p, n);
  w.perm_final = carve<int32_t>(p, n);
  w.nodes = carve<BNode>(p, cn);
  w.flags = carve<int32_t>(p, cn);
  w.rank = carve<int32_t>(p, cn);
  w.alive = carve<int32_t>(p, cn);
  w.leaf_flag = carve<int32_t>(p, cn);
  w.leaf_rank = carve<int32_t>(p, cn);
  w.tile_sums = carve<int32_t>(p, ntiles);
  w.chunks = carve<Chunk>(p, w.chunk_cap);
  w.chunk_nl = carve<int32_t>(p, w.chunk_cap);
  w.chunk_loff = carve<int32_t>(p, w.chunk_cap);
  w.big_list = carve<int32_t>(p, w.chunk_cap);
  w.node_chunk0 = carve<int32_t>(p, w.chunk_cap);
  w.acc = carve<U128>(p, (size_t)11 * (n / kBig + 2));
  w.ts0 = carve<double>(p, 1);
  w.counters = carve<int32_t>(p, 8);
  w.status = carve<LevelStatus>(p, 1);
  return KDS_OK;
}
}  // namespace

int tree_build(const float* xyz, const double* stamps, int64_t n, int32_t mem, const kds_tree_params* prm,
               cudaStream_t s, kds_tree** out) {
  *out = nullptr;
  if (n < 0 || n > (int64_t)1 << 30) { set_error("kds_tree_build: bad point count %lld", (long long)n); return KDS_ERR_INVALID_ARG; }
  if (n < prm->leaf_min_points || n == 0) {
    set_error("kds_tree_build: %lld points < leaf_min_points", (long long)n);
    return KDS_ERR_TREE_REJECTED;
  }
  BuildParams P;
  P.propagate_normal = prm->propagate_normal;
  P.leaf_min_points = prm->leaf_min_points;
  P.leaf_max_points = prm->leaf_max_points;
  P.leaf_density = prm->leaf_density;
  P.leaf_min_normal_incidence = prm->leaf_min_normal_incidence;
  P.leaf_normal_eigenratio = prm->leaf_normal_eigenratio;
  P.prune_incidence = prm->prune_min_normal_incidence;
  P.max_level = prm->max_level > 0 ? std::min(prm->max_level, 64) : 48;

  BuildWs w;
  int rc = ws_alloc(w, n);
  if (rc) return rc;
  struct Guard {
    BuildWs* w;
    void* h_xyz = nullptr;
    void* h_st = nullptr;
    ~Guard() {
      if (w->block) cudaFree(w->block);
      if (h_xyz) cudaFree(h_xyz);
      if (h_st) cudaFree(h_st);
    }
  } guard{&w};

  const float* d_xyz = xyz;
  const double* d_st = stamps;
  if (mem == KDS_MEM_HOST) {
    KDS_CK(cudaMalloc(&guard.h_xyz, sizeof(float) * 3 * n));
    KDS_CK(cudaMemcpyAsync(guard.h_xyz, xyz, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s));
    d_xyz = (const float*)guard.h_xyz;
    if (stamps) {
      KDS_CK(cudaMalloc(&guard.h_st, sizeof(double) * n));
      KDS_CK(cudaMemcpyAsync(guard.h_st, stamps, sizeof(double) * n, cudaMemcpyHostToDevice, s));
      d_st = (const double*)guard.h_st;
    }
  }
  KDS_CK(cudaMemsetAsync(w.status, 0, sizeof(LevelStatus), s));
  k_ingest<<<nblk(n, 256), 256, 0, s>>>(d_xyz, d_st, n, w.pa, w.sa, w.ia, w.status);
  k_ts_min<<<1, 1024, 0, s>>>(w.sa, n, w.ts0, w.status);
  k_dt_check<<<nblk(n, 256), 256, 0, s>>>(w.sa, n, w.ts0, w.status);
  {
    BNode root;
    memset(&root, 0, sizeof(root));
    root.start = 0;
    root.end = (int32_t)n;
    root.left = root.right = -1;
    KDS_CK(cudaMemcpyAsync(w.nodes, &root, sizeof(BNode), cudaMemcpyHostToDevice, s));
  }
  KDS_CK(cudaGetLastError());

  std::vector<int32_t> level_begin;
  int32_t lb = 0, le = 1;
  int32_t max_size = (int32_t)n;
  int cur = 0;  // which point buffer holds the current level
  LevelStatus hst;
  int depth = 0;
  while (lb < le) {
    level_begin.push_back(lb);
    ++depth;
    int32_t nl = le - lb;
    float4* pin = cur ? w.pb : w.pa;
    float4* pout = cur ? w.pa : w.pb;
    double* sin_ = cur ? w.sb : w.sa;
    double* sout = cur ? w.sa : w.sb;
    int32_t* iin = cur ? w.ib : w.ia;
    int32_t* iout = cur ? w.ia : w.ib;
    k_small_nodes<<<nblk((int64_t)nl * 32, 256), 256, 0, s>>>(w.nodes, lb, le, pin, sin_, iin, pout, sout, iout,
                                                              w.perm_final, w.ts0, P);
    if (max_size > kBig) {
      int32_t cb = (int32_t)(n / kChunk + nl + 1);
      cb = std::min(cb, w.chunk_cap);
      k_big_plan<<<1, 32, 0, s>>>(w.nodes, lb, le, w.chunks, w.chunk_cap, w.counters, w.big_list, w.counters + 1,
                                   w.node_chunk0, w.acc);
      k_big_moments<<<cb, kBuildThreads, 0, s>>>(w.chunks, w.counters, lb, pin, sin_, w.ts0, w.acc);
      k_big_decide<<<nblk(n / kBig + 1, 64), 64, 0, s>>>(w.nodes, lb, w.big_list, w.counters + 1, w.acc, P);
      k_big_count<<<cb, kBuildThreads, 0, s>>>(w.chunks, w.counters, w.nodes, pin, w.chunk_nl);
      k_big_offsets<<<1, 256, 0, s>>>(w.chunks, w.counters, w.nodes, w.big_list, w.counters + 1, w.node_chunk0,
                                      w.chunk_nl, w.chunk_loff);
      k_big_scatter<<<cb, kBuildThreads, 0, s>>>(w.chunks, w.counters, w.nodes, pin, sin_, iin, pout, sout, iout,
                                                 w.perm_final, w.chunk_loff);
    }
    k_split_flags<<<nblk(nl, 256), 256, 0, s>>>(w.nodes, lb, le, w.flags);
    rc = scan_exclusive(w.flags, w.rank, nl, w.tile_sums, w.counters + 2, s);
    if (rc) return rc;
    KDS_CK(cudaMemsetAsync(&w.status->max_size, 0, sizeof(int32_t), s));
    k_make_children<<<nblk(nl, 256), 256, 0, s>>>(w.nodes, lb, le, w.rank, (int32_t)w.cap_nodes, w.status);
    KDS_CK(cudaGetLastError());
    int32_t nsplit = 0;
    KDS_CK(cudaMemcpyAsync(&nsplit, w.counters + 2, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    KDS_CK(cudaMemcpyAsync(&hst, w.status, sizeof(LevelStatus), cudaMemcpyDeviceToHost, s));
    KDS_CK(cudaStreamSynchronize(s));
    if (hst.error == 2) { set_error("kds_tree_build: coordinate >= 32768 m, non-finite stamp or dt >= 65536 s"); return KDS_ERR_RANGE; }
    if (hst.error == 1) { set_error("kds_tree_build: node capacity exceeded"); return KDS_ERR_CAPACITY; }
    if ((int64_t)le + 2 * nsplit > w.cap_nodes) { set_error("kds_tree_build: node capacity exceeded"); return KDS_ERR_CAPACITY; }
    lb = le;
    le = le + 2 * nsplit;
    max_size = hst.max_size;
    cur ^= 1;
  }
  const int32_t total = le;
  // prune: bottom-up per level
  for (int l = (int)level_begin.size() - 1; l >= 0; --l) {
    int32_t b = level_begin[l];
    int32_t e = (l + 1 < (int)level_begin.size()) ? level_begin[l + 1] : total;
    k_alive<<<nblk(e - b, 256), 256, 0, s>>>(w.nodes, b, e, w.alive, P.prune_incidence);
  }
  rc = scan_exclusive(w.alive, w.rank, total, w.tile_sums, w.counters + 2, s);
  if (rc) return rc;
  k_leaf_flags<<<nblk(total, 256), 256, 0, s>>>(w.nodes, total, w.alive, w.leaf_flag);
  rc = scan_exclusive(w.leaf_flag, w.leaf_rank, total, w.tile_sums, w.counters + 3, s);
  if (rc) return rc;
  int32_t cnt[2];
  KDS_CK(cudaMemcpyAsync(cnt, w.counters + 2, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  KDS_CK(cudaStreamSynchronize(s));
  int32_t num_nodes = cnt[0], num_leaves = cnt[1];
  double ts0 = 0.0;
  KDS_CK(cudaMemcpy(&ts0, w.ts0, sizeof(double), cudaMemcpyDeviceToHost));
  if (num_leaves < prm->tree_min_good_leaves) {
    set_error("kds_tree_build: %d good leaves < tree_min_good_leaves %d", num_leaves, prm->tree_min_good_leaves);
    return KDS_ERR_TREE_REJECTED;
  }
  kds_tree* t = new kds_tree();
  rc = tree_alloc(t->d, num_nodes, num_leaves, n);
  if (rc) { delete t; return rc; }
  t->d.num_unpruned = total;
  t->d.ts_start = ts0;
  t->d.depth = depth;
  k_compact<<<nblk(total, 256), 256, 0, s>>>(w.nodes, total, w.alive, w.rank, w.leaf_flag, w.leaf_rank, t->d);
  k_copy_perm<<<nblk(n, 256), 256, 0, s>>>(w.perm_final, t->d.perm, n);
  rc = tree_gather_leaves(t->d, s);
  if (rc) { tree_release(t->d); delete t; return rc; }
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) { tree_release(t->d); delete t; return cuda_status(e, "tree build", __FILE__, __LINE__); }
  *out = t;
  return KDS_OK;
}

int tree_import(const float* mean, const float* dir, const double* dts_mean, const double* dts_cov,
                const int64_t* s0, const int64_t* e0, const int32_t* left, const int32_t* right, int64_t num_nodes,
                double ts_start, kds_tree** out) {
  *out = nullptr;
  if (num_nodes <= 0 || num_nodes > ((int64_t)1 << 30) || !mean || !dir || !left || !right) {
    set_error("kds_tree_import: bad arguments");
    return KDS_ERR_INVALID_ARG;
  }
  // count leaves on the host (the node array is host memory)
  int64_t nleaves = 0;
  for (int64_t i = 0; i < num_nodes; ++i)
    if (left[i] < 0 && right[i] < 0) ++nleaves;
  kds_tree* t = new kds_tree();
  int rc = tree_alloc(t->d, num_nodes, nleaves, 0);
  if (rc) { delete t; return rc; }
  t->d.ts_start = ts_start;
  t->d.num_unpruned = num_nodes;
  cudaStream_t s = cudaStreamPerThread;
  // staging
  size_t nb = num_nodes;
  void* stg = nullptr;
  size_t bytes = nb * (3 * 4 * 2 + 8 * 2 + 8 * 2 + 4 * 2) + 64;
  cudaError_t ce = cudaMalloc(&stg, bytes);
  if (ce != cudaSuccess) { cudaGetLastError(); tree_release(t->d); delete t; set_error("import staging OOM"); return KDS_ERR_OOM; }
  char* p = (char*)stg;
  float* dm = (float*)p; p += nb * 12;
  float* dd = (float*)p; p += nb * 12;
  double* ddm = (double*)p; p += nb * 8;
  double* ddc = (double*)p; p += nb * 8;
  int64_t* ds = (int64_t*)p; p += nb * 8;
  int64_t* de = (int64_t*)p; p += nb * 8;
  int32_t* dl = (int32_t*)p; p += nb * 4;
  int32_t* dr = (int32_t*)p; p += nb * 4;
  int32_t* dbad = (int32_t*)p;
  cudaMemcpyAsync(dm, mean, nb * 12, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dd, dir, nb * 12, cudaMemcpyHostToDevice, s);
  if (dts_mean) cudaMemcpyAsync(ddm, dts_mean, nb * 8, cudaMemcpyHostToDevice, s);
  if (dts_cov) cudaMemcpyAsync(ddc, dts_cov, nb * 8, cudaMemcpyHostToDevice, s);
  if (s0) cudaMemcpyAsync(ds, s0, nb * 8, cudaMemcpyHostToDevice, s);
  if (e0) cudaMemcpyAsync(de, e0, nb * 8, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dl, left, nb * 4, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dr, right, nb * 4, cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(dbad, 0, 4, s);
  k_import<<<nblk(num_nodes, 256), 256, 0, s>>>(t->d, dm, dd, dts_mean ? ddm : nullptr, dts_cov ? ddc : nullptr,
                                                 s0 ? ds : nullptr, e0 ? de : nullptr, dl, dr, dbad);
  // leaf list by scan over leaf flags, reusing the staging arrays (dl as flag, dr as rank)
  int32_t* flag = (int32_t*)ds;  // ds/de no longer needed after k_import on this stream
  int32_t* rank = (int32_t*)de;
  int32_t* tiles = dl;
  int32_t* total = dbad + 1;
  k_leaf_flags_plain<<<nblk(num_nodes, 256), 256, 0, s>>>(t->d.nodes, (int32_t)num_nodes, flag);
  int rc2 = scan_exclusive(flag, rank, (int32_t)num_nodes, tiles, total, s);
  k_leaf_scatter_plain<<<nblk(num_nodes, 256), 256, 0, s>>>(flag, rank, (int32_t)num_nodes, t->d.leaf_idx);
  tree_gather_leaves(t->d, s);
  int32_t bad = 0;
  cudaMemcpyAsync(&bad, dbad, 4, cudaMemcpyDeviceToHost, s);
  ce = cudaStreamSynchronize(s);
  cudaFree(stg);
  if (ce != cudaSuccess || rc2) {
    tree_release(t->d);
    delete t;
    return ce != cudaSuccess ? cuda_status(ce, "tree import", __FILE__, __LINE__) : rc2;
  }
  if (bad) {
    tree_release(t->d);
    delete t;
    set_error("kds_tree_import: child index out of range or not after its parent (BFS order required)");
    return KDS_ERR_BAD_TREE;
  }
  *out = t;
  return KDS_OK;
}

int tree_apply_velocities(kds_tree* t, const float* v, int skip_leaves, cudaStream_t s) {
  if (t->d.num_nodes == 0) return KDS_OK;
  Vel6 vv;
  for (int i = 0; i < 6; ++i) vv.v[i] = v[i];
  k_apply_velocities<<<nblk(t->d.num_nodes, 256), 256, 0, s>>>(t->d, vv, skip_leaves);
  KDS_CK(cudaGetLastError());
  return tree_gather_leaves(t->d, s);
}

int tree_apply_isometry(kds_tree* t, const float* X, cudaStream_t s) {
  if (t->d.num_nodes == 0) return KDS_OK;
  Iso12 iso;
  for (int i = 0; i < 12; ++i) iso.m[i] = X[i];
  k_apply_isometry<<<nblk(t->d.num_nodes, 256), 256, 0, s>>>(t->d, iso);
  KDS_CK(cudaGetLastError());
  return tree_gather_leaves(t->d, s);
}

int tree_extract_leaves(const kds_tree* t, const float* v6, float* out_host, cudaStream_t s) {
  if (t->d.num_leaves == 0) return KDS_OK;
  float* d = nullptr;
  KDS_CK(cudaMalloc(&d, sizeof(float) * 6 * t->d.num_leaves));
  Vel6 vv;
  for (int i = 0; i < 6; ++i) vv.v[i] = v6 ? v6[i] : 0.f;
  k_extract_leaves<<<nblk(t->d.num_leaves, 256), 256, 0, s>>>(t->d, vv, v6 ? 1 : 0, d);
  cudaError_t e = cudaMemcpyAsync(out_host, d, sizeof(float) * 6 * t->d.num_leaves, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_status(e, "extract leaves", __FILE__, __LINE__);
  return KDS_OK;
}

int tree_export(const kds_tree* t, float* mean, float* dir, double* dts_mean, double* dts_cov, int64_t* s0,
                int64_t* e0, int32_t* left, int32_t* right, int32_t* level, int64_t* leaves, int64_t* perm) {
  const TreeDev& d = t->d;
  int64_t nn = d.num_nodes;
  std::vector<DNode> hn(nn);
  KDS_CK(cudaMemcpy(hn.data(), d.nodes, sizeof(DNode) * nn, cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < nn; ++i) {
    if (mean) { mean[3 * i] = hn[i].a.x; mean[3 * i + 1] = hn[i].a.y; mean[3 * i + 2] = hn[i].a.z; }
    if (dir) { dir[3 * i] = hn[i].a.w; dir[3 * i + 1] = hn[i].b.x; dir[3 * i + 2] = hn[i].b.y; }
    int32_t l, r;
    std::memcpy(&l, &hn[i].b.z, 4);
    std::memcpy(&r, &hn[i].b.w, 4);
    if (left) left[i] = l;
    if (right) right[i] = r;
  }
  if (dts_mean) KDS_CK(cudaMemcpy(dts_mean, d.dts_mean, sizeof(double) * nn, cudaMemcpyDeviceToHost));
  if (dts_cov) KDS_CK(cudaMemcpy(dts_cov, d.dts_cov, sizeof(double) * nn, cudaMemcpyDeviceToHost));
  if (s0 || e0) {
    std::vector<int64_t> rg(2 * nn);
    KDS_CK(cudaMemcpy(rg.data(), d.range, sizeof(int64_t) * 2 * nn, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < nn; ++i) {
      if (s0) s0[i] = rg[2 * i];
      if (e0) e0[i] = rg[2 * i + 1];
    }
  }
  if (level) KDS_CK(cudaMemcpy(level, d.level, sizeof(int32_t) * nn, cudaMemcpyDeviceToHost));
  if (leaves && d.num_leaves) {
    std::vector<int32_t> li(d.num_leaves);
    KDS_CK(cudaMemcpy(li.data(), d.leaf_idx, sizeof(int32_t) * d.num_leaves, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < d.num_leaves; ++i) leaves[i] = li[i];
  }
  if (perm && d.perm && d.num_points) {
    std::vector<int32_t> pi(d.num_points);
    KDS_CK(cudaMemcpy(pi.data(), d.perm, sizeof(int32_t) * d.num_points, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < d.num_points; ++i) perm[i] = pi[i];
  }
  return KDS_OK;
}

}  // namespace kds
