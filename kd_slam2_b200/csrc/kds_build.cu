// GPU surfel KD-tree build for one or many clouds at once (a forest).  Compiled with
// -fmad=false: every double/float expression rounds each multiply and add separately,
// so the result is bit-identical to the CPU oracle's canonical build.
//
// Replaces TreeGenerator_::makeTree (kd/tree/tree_generator_impl_.h:7-19), which the
// reference runs on the CPU only.  The tree is built level by level for all trees of
// the batch together:
//   * per-node moments [xx,xy,xz,yy,yz,zz,x,y,z,dt,dt^2] are exact, order-free 128-bit
//     fixed-point sums: each product of two floats (or double stamp term) is decomposed
//     into sign/mantissa/exponent and its floor(v * 2^64) is formed with integer shifts,
//     so warps, blocks and atomics may add them in any order;
//   * FP64 covariance, cyclic Jacobi eigensolver, FlatLeafPolicy_ decision
//     (kd/tree/flat_leaf_policy_.h:52-108) in FP64;
//   * stable partition by Node_::whichSide in float (kd/tree/node_.h:53-56);
//   * children numbered by a scan over the level's split flags: nodes of one level
//     are grouped by tree, so each tree's nodes in global order are its BFS order
//     (kd/tree/tree_cpu_impl_.h:136-158), kept by prune (kd/tree/tree_cpu_.h:172-207).
// Nodes with <= kBig points are processed by one warp each; larger ones by blocks over
// kChunk-point chunks with 128-bit atomics.  The level bounds live in device memory;
// the host checks for completion only every kLevelsPerSync levels.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <vector>

#include "kds_internal.cuh"

namespace kds {

namespace {

constexpr int kBig = 1024;
constexpr int kRootFrame = 15;  // doubles per root: eigenvalues, eigenvectors, mean (decide)
constexpr int kChunk = 1024;
constexpr int kThreads = 256;
constexpr int kGridBlocks = 148 * 4;
constexpr int kLevelBlocks = 148 * 3;  // k_decide: 3 blocks per SM at its register count
constexpr int kLevelsPerSync = 4;
constexpr int kMaxDepth = 64;
constexpr int kUnroll = 2;  // rounds of 32 points in flight per lane in the warp-per-node partition
constexpr int kSmallBlocks = 148 * 4;  // two waves: other streams' kernels interleave at block boundaries

// ---------------------------------------------------------------------------
// 128-bit two's complement fixed point (units of 2^-64)
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
__host__ __device__ __forceinline__ U128 u128_sub(U128 a, U128 b) {
  U128 r;
  r.lo = a.lo - b.lo;
  r.hi = a.hi - b.hi - (a.lo < b.lo ? 1ull : 0ull);
  return r;
}
__host__ __device__ __forceinline__ double fx_to_d(U128 q) {
  long long hi = (long long)q.hi;
  return ((double)hi * 0x1p64 + (double)q.lo) * 0x1p-64;
}

// floor(v * 2^64) for v = (-1)^sign * mant * 2^exp2 (exact integer arithmetic)
__device__ __forceinline__ U128 fx_parts(unsigned sign, unsigned long long mant, int exp2) {
  U128 mag = u128_zero();
  bool rem = false;
  if (mant == 0ull) return mag;
  int sh = exp2 + 64;
  if (sh >= 64) {
    mag.hi = mant << (sh - 64);
  } else if (sh > 0) {
    mag.lo = mant << sh;
    mag.hi = mant >> (64 - sh);
  } else if (sh == 0) {
    mag.lo = mant;
  } else {
    int r = -sh;
    if (r >= 64) {
      rem = true;
    } else {
      mag.lo = mant >> r;
      rem = (mant & ((1ull << r) - 1ull)) != 0ull;
    }
  }
  if (!sign) return mag;
  U128 neg;  // -mag - rem: ~mag when rem, else ~mag + 1
  neg.lo = ~mag.lo;
  neg.hi = ~mag.hi;
  if (!rem) {
    neg.lo += 1ull;
    if (neg.lo == 0ull) neg.hi += 1ull;
  }
  return neg;
}
__device__ __forceinline__ void f_parts(float f, unsigned& s, unsigned& m, int& e) {
  unsigned b = __float_as_uint(f);
  s = b >> 31;
  unsigned E = (b >> 23) & 0xffu;
  m = b & 0x7fffffu;
  if (E == 0u) {
    e = -149;
  } else {
    m |= 0x800000u;
    e = (int)E - 150;
  }
}
__device__ __forceinline__ U128 fx_f(float a) {
  unsigned s, m;
  int e;
  f_parts(a, s, m, e);
  return fx_parts(s, m, e);
}
__device__ __forceinline__ U128 fx_ff(float a, float b) {
  unsigned sa, ma, sb, mb;
  int ea, eb;
  f_parts(a, sa, ma, ea);
  f_parts(b, sb, mb, eb);
  return fx_parts(sa ^ sb, (unsigned long long)ma * (unsigned long long)mb, ea + eb);
}
__device__ __forceinline__ U128 fx_d(double d) {
  unsigned long long b = (unsigned long long)__double_as_longlong(d);
  unsigned s = (unsigned)(b >> 63);
  int E = (int)((b >> 52) & 0x7ffull);
  unsigned long long m = b & ((1ull << 52) - 1ull);
  int e;
  if (E == 0) {
    e = -1074;
  } else {
    m |= 1ull << 52;
    e = E - 1075;
  }
  return fx_parts(s, m, e);
}

// floor(d * 2^64) for a non-negative double below 2^52 (the stamp terms dt and dt^2: dt >= 0
// by construction, dt < 2^16 checked): two clamped shifts instead of fx_parts' branches,
// the same bits.
__device__ __forceinline__ unsigned long long shl_c(unsigned long long v, unsigned n) {
  unsigned long long r;
  asm("shl.b64 %0, %1, %2;" : "=l"(r) : "l"(v), "r"(n));  // n >= 64 gives 0
  return r;
}
__device__ __forceinline__ unsigned long long shr_c(unsigned long long v, unsigned n) {
  unsigned long long r;
  asm("shr.u64 %0, %1, %2;" : "=l"(r) : "l"(v), "r"(n));  // n >= 64 gives 0
  return r;
}
__device__ __forceinline__ U128 fx_d_nonneg(double d) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(d);
  const int E = (int)((b >> 52) & 0x7ffull);
  if ((b >> 63) || E >= 1075) return fx_d(d);  // negative, >= 2^52 or not finite: general path
  unsigned long long m = b & ((1ull << 52) - 1ull);
  int sh;  // d * 2^64 = m * 2^sh
  if (E == 0) {
    sh = -1074 + 64;
  } else {
    m |= 1ull << 52;
    sh = E - 1075 + 64;
  }
  U128 r;  // sh < 64 here
  r.lo = sh >= 0 ? shl_c(m, (unsigned)sh) : shr_c(m, (unsigned)(-sh));
  r.hi = shr_c(m, (unsigned)(64 - sh));
  return r;
}

struct Moments {
  U128 s[11];
};

// Fast path of the same floors.  A float x with x == 0 or 2^-25 <= |x| < 2^15 has no
// bit below 2^-48, so x = X * 2^-48 with an integer |X| < 2^63.  Then
// floor(x * y * 2^64) = floor(X * Y / 2^32) (an arithmetic shift of the 128-bit
// product) and floor(x * 2^64) = X * 2^16, both exact.
__device__ __forceinline__ bool fx_grid48(float x, long long& X) {
  X = __float2ll_rn(x * 0x1p48f);
  const float a = fabsf(x);
  return a == 0.0f || a >= 0x1p-25f;
}
__device__ __forceinline__ U128 fx_prod48(long long X, long long Y) {
  const unsigned long long lo = (unsigned long long)X * (unsigned long long)Y;
  const long long hi = __mul64hi(X, Y);
  U128 r;
  r.lo = (lo >> 32) | ((unsigned long long)hi << 32);
  r.hi = (unsigned long long)(hi >> 32);
  return r;
}
__device__ __forceinline__ U128 fx_single48(long long X) {
  U128 r;
  r.lo = (unsigned long long)X << 16;
  r.hi = (unsigned long long)(X >> 48);
  return r;
}

__device__ __forceinline__ void moments_add_point(Moments& M, float4 p, double st, double ts0) {
  long long X, Y, Z;
  const bool gx = fx_grid48(p.x, X), gy = fx_grid48(p.y, Y), gz = fx_grid48(p.z, Z);
  if (gx && gy && gz) {
    M.s[0] = u128_add(M.s[0], fx_prod48(X, X));
    M.s[1] = u128_add(M.s[1], fx_prod48(X, Y));
    M.s[2] = u128_add(M.s[2], fx_prod48(X, Z));
    M.s[3] = u128_add(M.s[3], fx_prod48(Y, Y));
    M.s[4] = u128_add(M.s[4], fx_prod48(Y, Z));
    M.s[5] = u128_add(M.s[5], fx_prod48(Z, Z));
    M.s[6] = u128_add(M.s[6], fx_single48(X));
    M.s[7] = u128_add(M.s[7], fx_single48(Y));
    M.s[8] = u128_add(M.s[8], fx_single48(Z));
  } else {
    M.s[0] = u128_add(M.s[0], fx_ff(p.x, p.x));
    M.s[1] = u128_add(M.s[1], fx_ff(p.x, p.y));
    M.s[2] = u128_add(M.s[2], fx_ff(p.x, p.z));
    M.s[3] = u128_add(M.s[3], fx_ff(p.y, p.y));
    M.s[4] = u128_add(M.s[4], fx_ff(p.y, p.z));
    M.s[5] = u128_add(M.s[5], fx_ff(p.z, p.z));
    M.s[6] = u128_add(M.s[6], fx_f(p.x));
    M.s[7] = u128_add(M.s[7], fx_f(p.y));
    M.s[8] = u128_add(M.s[8], fx_f(p.z));
  }
  double dt = st - ts0;
  M.s[9] = u128_add(M.s[9], fx_d_nonneg(dt));
  M.s[10] = u128_add(M.s[10], fx_d_nonneg(dt * dt));
}

// ---------------------------------------------------------------------------
struct BNode {
  int32_t start, end;
  int32_t level;
  int32_t tree;
  int32_t split;      // 1: inner node
  int32_t mid;
  int32_t left, right;
  int32_t has_parent;
  int32_t par_has;    // propagated normal received from the parent
  int32_t has_prop;   // propagated normal handed to the children
  int32_t parent;     // parent node, -1 for a root
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

struct LevelState {
  int32_t lb, le;        // node range of the current level
  int32_t cur;           // point buffer holding the current level
  int32_t depth;         // number of levels processed
  int32_t max_size;      // largest node of the current level
  int32_t max_next;      // largest node of the next level (being built)
  int32_t error;         // 1: node capacity, 2: input out of range
  int32_t num_chunks, num_big;
  int32_t pad_;
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
    if (a[0][1] == 0.0 && a[0][2] == 0.0 && a[1][2] == 0.0) break;
    for (int pq = 0; pq < 3; ++pq) {
      int p = (pq == 2) ? 1 : 0;
      int q = (pq == 0) ? 1 : 2;
      int r = 3 - p - q;
      double apq = a[p][q];
      // negligible off-diagonal: set to zero (same rule in the CPU oracle)
      if (fabs(apq) <= 1e-18 * (fabs(a[p][p]) + fabs(a[q][q]))) {
        a[p][q] = 0.0;
        a[q][p] = 0.0;
        continue;
      }
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
// label_policy_base_impl_.h:12-97) on FP64 statistics.
// Sd: the node's 11 moment sums converted to double (fx_to_d of the exact sums).
// root (nullable): for a root node, its frame as TreeCPU_'s constructor stores it
// (kd/tree/tree_cpu_.h:72-86): [0..2] eigenvalues ascending, [3..11] eigenvectors
// column-major (columns 0 and 2 reoriented as in fillMetadata, then column 0 negated if
// the determinant is negative), [12..14] mean; zero where the node has < 3 points.
__device__ __noinline__ void decide(const double* Sd, int64_t n, BNode& nd, const BuildParams& P, double* root) {
  for (int i = 0; i < 3; ++i) { nd.mean[i] = 0.f; nd.dir[i] = 0.f; }
  nd.dts_mean = 0.0;
  nd.dts_cov = 0.0;
  double mean_d[3] = {0, 0, 0};
  double e0[3] = {0, 0, 0}, e2[3] = {0, 0, 0};
  double lam[3] = {0, 0, 0};
  bool is_bad = true;
  if (n > 0) {
    double dn = (double)n;
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
      if (root) {
        const double e1[3] = {V[0][1], V[1][1], V[2][1]};
        // det [e0 e1 e2] = e0 . (e1 x e2)
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

// block-wide exclusive scan of one int per thread; *total = block sum
__device__ __forceinline__ int block_scan(int v, int* sm, int* total) {
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

// The node range [b, e) of this block when gridDim.x blocks split the current level.
__device__ __forceinline__ void level_range(const LevelState* ls, int& b, int& e) {
  const int lb = ls->lb, le = ls->le;
  const int nl = le - lb;
  const int per = (nl + gridDim.x - 1) / gridDim.x;
  b = lb + blockIdx.x * per;
  e = min(b + per, le);
}

// ---------------------------------------------------------------------------
// Kernels

__global__ void k_ingest(const float* xyz, const double* st, int64_t n, float4* pts, double* sts, LevelState* ls) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    double s = st ? st[i] : 0.0;
    bool ok = fabsf(x) < 32768.f && fabsf(y) < 32768.f && fabsf(z) < 32768.f && isfinite(s);
    if (!ok) ls->error = 2;
    pts[i] = make_float4(x, y, z, __int_as_float((int32_t)i));
    sts[i] = s;
  }
}

// Order-preserving map of finite doubles to unsigned 64-bit keys.
__device__ __forceinline__ unsigned long long dkey(double d) {
  unsigned long long b = (unsigned long long)__double_as_longlong(d);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dkey_inv(unsigned long long k) {
  unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

// ts_start of each tree = min stamp (label_policy_base_impl_.h:28-35); blockIdx.y = tree.
__global__ void k_tree_min(const double* sts, const int64_t* off, unsigned long long* tsmin) {
  const int r = blockIdx.y;
  const int64_t b = off[r], e = off[r + 1];
  unsigned long long m = ~0ull;
  for (int64_t i = b + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < e; i += (int64_t)gridDim.x * blockDim.x)
    m = min(m, dkey(sts[i]));
  for (int off2 = 16; off2 > 0; off2 >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, off2));
  if ((threadIdx.x & 31) == 0 && m != ~0ull) atomicMin(&tsmin[r], m);
}

// decodes ts_start and checks the dt range of every point; blockIdx.y = tree.
__global__ void k_tree_check(const double* sts, const int64_t* off, const unsigned long long* tsmin, double* ts0,
                             LevelState* ls) {
  const int r = blockIdx.y;
  const int64_t b = off[r], e = off[r + 1];
  const double t0 = (e > b) ? dkey_inv(tsmin[r]) : 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) ts0[r] = t0;
  for (int64_t i = b + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < e; i += (int64_t)gridDim.x * blockDim.x)
    if (!(sts[i] - t0 < 65536.0)) ls->error = 2;
}

__global__ void k_init_roots(BNode* nodes, const int64_t* off, int R, LevelState* ls, int32_t* level_begin) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < R) {
    BNode nd;
    memset(&nd, 0, sizeof(nd));
    nd.start = (int32_t)off[r];
    nd.end = (int32_t)off[r + 1];
    nd.tree = r;
    nd.left = nd.right = -1;
    nd.parent = -1;
    nodes[r] = nd;
    atomicMax(&ls->max_size, nd.end - nd.start);
  }
  if (r == 0) {
    ls->lb = 0;
    ls->le = R;
    ls->cur = 0;
    ls->depth = 0;
    ls->max_next = 0;
    level_begin[0] = 0;
  }
}

// A point moves through the levels as one 16 B record (x, y, z, w = its input index as int
// bits), double-buffered by level parity; its stamp stays in input order and is read by
// index where a sum needs it.
struct PointBufs {
  float4* p[2];
  double* st;     // stamps, input order
  int32_t* perm;  // final point order (global indices)
};

// Every node's 11 exact moment sums are kept in mom[node].  The roots' sums are
// computed from their points; a split node hands its children their sums: the smaller
// child's from one pass over its points after the partition, the other's as the
// parent's minus the smaller's (exact integer arithmetic).  So below the roots each point
// is summed once per level only when it lands in the smaller child of its parent.

// L1 prefetch of the line holding p (no register, no effect on results).
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// Warp-cooperative exact sums of points [b, e) of one point buffer.
// Warp total of the 11 sums in reduce-scatter form: the 16 slots (11 used) are halved
// over lane bits 4..1 (8 + 4 + 2 + 1 exchanges instead of 5 x 11), then added with
// lane ^ 1.  Lanes 2k and 2k + 1 return the total of sum k (k < 11; slots 11-15 are 0).
__device__ __forceinline__ U128 warp_sum_moments(const Moments& M, int lane) {
  U128 v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = k < 11 ? M.s[k] : u128_zero();
  U128 w8[8], w4[4], w2[2];
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
#pragma unroll
  for (int j = 0; j < 8; ++j) w8[j] = u128_add(b4 ? v[8 + j] : v[j], shfl_xor_u128(b4 ? v[j] : v[8 + j], 16));
#pragma unroll
  for (int j = 0; j < 4; ++j) w4[j] = u128_add(b3 ? w8[4 + j] : w8[j], shfl_xor_u128(b3 ? w8[j] : w8[4 + j], 8));
#pragma unroll
  for (int j = 0; j < 2; ++j) w2[j] = u128_add(b2 ? w4[2 + j] : w4[j], shfl_xor_u128(b2 ? w4[j] : w4[2 + j], 4));
  U128 w1 = u128_add(b1 ? w2[1] : w2[0], shfl_xor_u128(b1 ? w2[0] : w2[1], 2));
  return u128_add(w1, shfl_xor_u128(w1, 1));
}

// Sums of the points [b, e) by one warp; returns warp_sum_moments of them.
__device__ __forceinline__ U128 warp_moments(const float4* p, const double* st, int b, int e, double t0, int lane) {
  constexpr int U = 2;  // loads in flight per lane (the 11 sums already hold 44 registers)
  Moments M;
  for (int k = 0; k < 11; ++k) M.s[k] = u128_zero();
  for (int k0 = b; k0 < e; k0 += 32 * U) {
    float4 pv[U];
    double sv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = k0 + u * 32 + lane;
      if (i < e) pv[u] = p[i];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = k0 + u * 32 + lane;
      if (i < e) sv[u] = st[__float_as_int(pv[u].w)];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = k0 + u * 32 + lane;
      if (i < e) moments_add_point(M, pv[u], sv[u], t0);
    }
  }
  return warp_sum_moments(M, lane);
}

// Level 0: warp per root of at most kBig points.
__global__ void __launch_bounds__(kThreads) k_root_moments(const BNode* nodes, int R, PointBufs B, const double* ts0,
                                                           U128* mom) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < R; r += nw) {
    const int s = nodes[r].start, e = nodes[r].end;
    if (e - s > kBig) continue;
    const U128 q = warp_moments(B.p[0], B.st, s, e, ts0[nodes[r].tree], lane);
    if (!(lane & 1) && lane < 22) mom[(size_t)r * 11 + (lane >> 1)] = q;
  }
}

// Thread per node of the level: the leaf/split decision from its sums.  Block b takes
// the b-th contiguous range of the level's nodes and writes its count of split nodes
// (the children's numbering scans these counts).
__global__ void k_decide(BNode* nodes, const LevelState* ls, const U128* mom, BuildParams P, int32_t* bsum,
                         int32_t* bbig, double* root_frame) {
  __shared__ int sm[32];
  int b, e;
  level_range(ls, b, e);
  int v = 0, nc = 0, nb = 0;
  for (int i = b + threadIdx.x; i < e; i += blockDim.x) {
    BNode nd = nodes[i];
    const int n = nd.end - nd.start;
    double Sd[11];
    for (int k = 0; k < 11; ++k) Sd[k] = fx_to_d(mom[(size_t)i * 11 + k]);
    decide(Sd, n, nd, P, nd.level == 0 ? root_frame + (size_t)nd.tree * kRootFrame : nullptr);
    nodes[i] = nd;
    v += nd.split ? 1 : 0;
    if (n > kBig) {
      nc += (n + kChunk - 1) / kChunk;
      nb += 1;
    }
  }
  int total, tc, tb;
  block_scan(v, sm, &total);
  block_scan(nc, sm, &tc);
  block_scan(nb, sm, &tb);
  if (threadIdx.x == 0) {
    bsum[blockIdx.x] = total;
    bbig[2 * blockIdx.x] = tc;  // as k_big_sums
    bbig[2 * blockIdx.x + 1] = tb;
  }
}

// The level's split count from k_decide's per-block counts, then the next level (one
// whole block).
__device__ void level_advance_block(LevelState* ls, const int32_t* bsum, int nblocks, int32_t* level_begin) {
  __shared__ int sm[32];
  int v = 0;
  for (int k = threadIdx.x; k < nblocks; k += blockDim.x) v += bsum[k];
  int total;
  block_scan(v, sm, &total);
  if (threadIdx.x != 0 || ls->lb >= ls->le) return;
  ls->lb = ls->le;
  ls->le = ls->le + 2 * total;
  ls->cur ^= 1;
  ls->depth += 1;
  if (ls->depth < kMaxDepth + 1) level_begin[ls->depth] = ls->lb;
  ls->max_size = ls->max_next;
  ls->max_next = 0;
}

// The last block of the level's last kernel advances the level (done: a counter that
// starts at 0 and is left at 0; nullptr: not the last kernel).  Every block of the
// calling kernel must reach this.
__device__ __forceinline__ void advance_if_last(LevelState* ls, const int32_t* bsum, int nblocks,
                                                int32_t* level_begin, unsigned* done) {
  if (!done) return;
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(done, 1u) == gridDim.x - 1 ? 1 : 0;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  level_advance_block(ls, bsum, nblocks, level_begin);
  if (threadIdx.x == 0) *done = 0u;
}

// The first 18 words of a BNode (start .. dir): one coalesced load by lanes 0-17.
constexpr int kNodeHeadWords = 18;
static_assert(offsetof(BNode, dir) + 3 * sizeof(float) == kNodeHeadWords * 4, "BNode head layout");
static_assert(offsetof(BNode, start) == 0 && offsetof(BNode, end) == 4 && offsetof(BNode, tree) == 12 &&
                  offsetof(BNode, split) == 16 && offsetof(BNode, left) == 24 && offsetof(BNode, right) == 28 &&
                  offsetof(BNode, mean) == 48,
              "BNode head layout");

// Warp per node of at most kBig points, after its children are numbered: stable
// partition by whichSide (or leaf point order), the children's ranges and sums.
// Latency-bound at deep levels (many small nodes per warp), so each node's record
// and sums are fetched in one round of loads, one node ahead.
__global__ void __launch_bounds__(kThreads, 2) k_small_part(BNode* nodes, LevelState* ls, PointBufs B,
                                                         const double* ts0, U128* mom, const int32_t* bsum,
                                                         int nblocks, int32_t* level_begin, unsigned* done) {
  const int lb = ls->lb, le = ls->le, cur = ls->cur;
  const float4* pin = B.p[cur];
  const double* sts = B.st;
  float4* pout = B.p[cur ^ 1];
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int wslot = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;  // consecutive nodes on different SMs
  const bool sum_lane = !(lane & 1) && lane < 22;                  // holds sum lane / 2
  int maxc = 0;
  int word = 0;
  U128 pm = u128_zero();
  auto fetch = [&](int ni) {
    if (ni < le) {
      if (lane < kNodeHeadWords) word = reinterpret_cast<const int*>(nodes + ni)[lane];
      if (sum_lane) pm = mom[(size_t)ni * 11 + (lane >> 1)];
    }
  };
  fetch(lb + wslot);
  for (int ni = lb + wslot; ni < le; ni += nwarps) {
    const int s = __shfl_sync(0xffffffffu, word, 0), e = __shfl_sync(0xffffffffu, word, 1);
    const int tree = __shfl_sync(0xffffffffu, word, 3), split = __shfl_sync(0xffffffffu, word, 4);
    const int li = __shfl_sync(0xffffffffu, word, 6), ri = __shfl_sync(0xffffffffu, word, 7);
    float mean[3], dir[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      mean[k] = __int_as_float(__shfl_sync(0xffffffffu, word, 12 + k));
      dir[k] = __int_as_float(__shfl_sync(0xffffffffu, word, 15 + k));
    }
    const U128 psum = pm;
    fetch(ni + nwarps);  // the next node's record and sums are in flight meanwhile
    if (e - s > kBig) continue;
    if (!split) {
      for (int i = s + lane; i < e; i += 32) B.perm[i] = __float_as_int(pin[i].w);
      if (lane == 0) nodes[ni].mid = e;
      continue;
    }
    const int K = (e - s + 31) >> 5;
    const bool one = K <= kUnroll;  // the whole node fits one round of loads: keep it
    // every round of the node in flight at once (into L1), instead of one dependent
    // round trip per kUnroll rounds
    for (int k = kUnroll; k < K; ++k) {
      const int i = s + (k << 5) + lane;
      if (i < e) prefetch_l1(pin + i);
    }
    unsigned bits = 0u;
    float4 pv[kUnroll];
    for (int k0 = 0; k0 < K; k0 += kUnroll) {
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        int i = s + ((k0 + u) << 5) + lane;
        if (i < e) pv[u] = pin[i];
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        int i = s + ((k0 + u) << 5) + lane;
        if (i < e) {
          prefetch_l1(sts + __float_as_int(pv[u].w));  // the stamp, if this point lands in the smaller child
          if (which_side_f(mean, dir, pv[u])) bits |= 1u << (k0 + u);
        }
      }
    }
    int nl = __popc(bits);
    for (int off = 16; off > 0; off >>= 1) nl += __shfl_xor_sync(0xffffffffu, nl, off);
    const int mid = s + nl;
    // the smaller child is summed while its points move; the other is the parent minus it
    const bool small_left = mid - s <= e - mid;
    const double t0 = ts0[tree];
    Moments MS;
    for (int k = 0; k < 11; ++k) MS.s[k] = u128_zero();
    const unsigned lt = (1u << lane) - 1u;
    int cl = 0, cr = 0;
    for (int k0 = 0; k0 < K; k0 += kUnroll) {
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        int i = s + ((k0 + u) << 5) + lane;
        if (i < e && !one) pv[u] = pin[i];
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        int i = s + ((k0 + u) << 5) + lane;
        bool valid = i < e;
        bool left = valid && ((bits >> (k0 + u)) & 1u);
        unsigned bl = __ballot_sync(0xffffffffu, left);
        unsigned br = __ballot_sync(0xffffffffu, valid && !left);
        if (valid) {
          int dst = left ? (s + cl + __popc(bl & lt)) : (s + nl + cr + __popc(br & lt));
          pout[dst] = pv[u];
          if (left == small_left) moments_add_point(MS, pv[u], sts[__float_as_int(pv[u].w)], t0);
        }
        cl += __popc(bl);
        cr += __popc(br);
      }
    }
    const U128 q = warp_sum_moments(MS, lane);
    if (sum_lane) {
      const int k = lane >> 1;
      const U128 other = u128_sub(psum, q);
      mom[(size_t)li * 11 + k] = small_left ? q : other;
      mom[(size_t)ri * 11 + k] = small_left ? other : q;
    }
    if (lane == 0) {
      nodes[ni].mid = mid;
      nodes[li].start = s;
      nodes[li].end = mid;
      nodes[ri].start = mid;
      nodes[ri].end = e;
      maxc = max(maxc, max(mid - s, e - mid));
    }
  }
  if (lane == 0 && maxc > 0) atomicMax(&ls->max_next, maxc);
  advance_if_last(ls, bsum, nblocks, level_begin, done);
}

// ---- large nodes ------------------------------------------------------------------
struct Chunk {
  int32_t node;
  int32_t begin;
  int32_t end;
  int32_t big;  // ordinal among the level's large nodes
};

// Large nodes of the level and their kChunk-point chunks, listed in node order by
// kLevelBlocks blocks over contiguous node ranges: per-block counts first, then each
// block writes its list at the prefix of the blocks before it.
__global__ void k_big_sums(const BNode* nodes, const LevelState* ls, int32_t* bbig) {
  __shared__ int sm[32];
  if (ls->max_size <= kBig) return;  // no large node on this level
  int b, e;
  level_range(ls, b, e);
  int nc = 0, nb = 0;
  for (int i = b + threadIdx.x; i < e; i += blockDim.x) {
    const int n = nodes[i].end - nodes[i].start;
    if (n > kBig) {
      nc += (n + kChunk - 1) / kChunk;
      nb += 1;
    }
  }
  int tc, tb;
  block_scan(nc, sm, &tc);
  block_scan(nb, sm, &tb);
  if (threadIdx.x == 0) {
    bbig[2 * blockIdx.x] = tc;
    bbig[2 * blockIdx.x + 1] = tb;
  }
}

__global__ void k_big_plan(const BNode* nodes, LevelState* ls, const int32_t* bbig, Chunk* chunks, int32_t chunk_cap,
                           int32_t* big_list, int32_t* node_chunk0, U128* acc, U128* accl) {
  __shared__ int sm[32];
  if (ls->max_size <= kBig) {  // no large node on this level
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ls->num_chunks = 0;
      ls->num_big = 0;
    }
    return;
  }
  int b, e;
  level_range(ls, b, e);
  int carry_c, carry_b, all_c, all_b;  // chunks / large nodes of the blocks before this one, of all
  {
    int vc = 0, vb = 0, ac = 0, ab = 0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
      if (k < (int)blockIdx.x) {
        vc += bbig[2 * k];
        vb += bbig[2 * k + 1];
      }
      ac += bbig[2 * k];
      ab += bbig[2 * k + 1];
    }
    block_scan(vc, sm, &carry_c);
    block_scan(vb, sm, &carry_b);
    block_scan(ac, sm, &all_c);
    block_scan(ab, sm, &all_b);
  }
  for (int base = b; base < e; base += blockDim.x) {
    int i = base + threadIdx.x;
    int n = 0;
    if (i < e) n = nodes[i].end - nodes[i].start;
    bool big = n > kBig;
    int nc = big ? (n + kChunk - 1) / kChunk : 0;
    int tc, tb;
    int oc = block_scan(nc, sm, &tc) + carry_c;
    int ob = block_scan(big ? 1 : 0, sm, &tb) + carry_b;
    if (big) {
      big_list[ob] = i;
      node_chunk0[ob] = oc;
      int s = nodes[i].start, en = nodes[i].end;
      for (int k = 0; k < nc; ++k) {
        int c = oc + k;
        if (c < chunk_cap) {
          chunks[c].node = i;
          chunks[c].begin = s + k * kChunk;
          chunks[c].end = min(s + (k + 1) * kChunk, en);
          chunks[c].big = ob;
        }
      }
      for (int k = 0; k < 11; ++k) {
        acc[(size_t)ob * 11 + k] = u128_zero();
        accl[(size_t)ob * 11 + k] = u128_zero();
      }
    }
    carry_c += tc;
    carry_b += tb;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ls->num_chunks = min(all_c, chunk_cap);
    ls->num_big = all_b;
    if (all_c > chunk_cap) ls->error = 1;
  }
}

// Block sum of per-thread sums into one 128-bit accumulator set (any order: exact).
__device__ __forceinline__ void block_add_moments(const Moments& M, U128 (*sm)[11], U128* dst) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const U128 q = warp_sum_moments(M, lane);
  if (!(lane & 1) && lane < 22) sm[w][lane >> 1] = q;
  __syncthreads();
  if (threadIdx.x < 11) {
    U128 t = u128_zero();
    for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) t = u128_add(t, sm[ww][threadIdx.x]);
    atomic_add_u128(&dst[threadIdx.x], t);
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kThreads) k_big_moments(const Chunk* chunks, const LevelState* ls,
                                                          const PointBufs B, const double* ts0, const BNode* nodes,
                                                          U128* acc) {
  __shared__ U128 sm[kThreads / 32][11];
  const int nc = ls->num_chunks, cur = ls->cur;
  const float4* pts = B.p[cur];
  const double* st = B.st;
  for (int ci = blockIdx.x; ci < nc; ci += gridDim.x) {
    Chunk c = chunks[ci];
    double t0 = ts0[nodes[c.node].tree];
    Moments M;
    for (int k = 0; k < 11; ++k) M.s[k] = u128_zero();
    for (int i = c.begin + threadIdx.x; i < c.end; i += blockDim.x) {
      const float4 pp = pts[i];
      moments_add_point(M, pp, st[__float_as_int(pp.w)], t0);
    }
    block_add_moments(M, sm, acc + (size_t)c.big * 11);
  }
}

// Level 0: the sums of the large roots, from the chunk accumulators.
__global__ void k_big_to_mom(const LevelState* ls, const int32_t* big_list, const U128* acc, U128* mom) {
  const int nb = ls->num_big;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nb * 11; t += gridDim.x * blockDim.x)
    mom[(size_t)big_list[t / 11] * 11 + t % 11] = acc[t];
}

__global__ void k_big_count(const Chunk* chunks, const LevelState* ls, const BNode* nodes, const PointBufs B,
                            int32_t* chunk_nl) {
  __shared__ int cnt;
  const int nc = ls->num_chunks;
  const float4* pts = B.p[ls->cur];
  for (int ci = blockIdx.x; ci < nc; ci += gridDim.x) {
    Chunk c = chunks[ci];
    const BNode& nd = nodes[c.node];
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    int local = 0;
    if (nd.split)
      for (int i = c.begin + threadIdx.x; i < c.end; i += blockDim.x)
        local += which_side_f(nd.mean, nd.dir, pts[i]) ? 1 : 0;
    atomicAdd(&cnt, local);
    __syncthreads();
    if (threadIdx.x == 0) chunk_nl[ci] = cnt;
    __syncthreads();
  }
}

// Block per large node: the exclusive scan of its chunks' left counts (each chunk's left
// offset inside the node), then the node's split point and its children's ranges.
__global__ void k_big_offsets(BNode* nodes, LevelState* ls, const int32_t* big_list,
                              const int32_t* node_chunk0, const int32_t* chunk_nl, int32_t* chunk_loff) {
  __shared__ int sm[32];
  const int nb = ls->num_big, nc = ls->num_chunks;
  for (int b = blockIdx.x; b < nb; b += gridDim.x) {
    const int c0 = node_chunk0[b];
    const int c1 = (b + 1 < nb) ? node_chunk0[b + 1] : nc;
    int carry = 0;
    for (int base = c0; base < c1; base += blockDim.x) {
      const int c = base + threadIdx.x;
      const int v = c < c1 ? chunk_nl[c] : 0;
      int tot;
      const int ex = block_scan(v, sm, &tot);
      if (c < c1) chunk_loff[c] = carry + ex;
      carry += tot;
    }
    if (threadIdx.x == 0) {
      BNode& nd = nodes[big_list[b]];
      nd.mid = nd.split ? nd.start + carry : nd.end;
      if (nd.split) {
        nodes[nd.left].start = nd.start;
        nodes[nd.left].end = nd.mid;
        nodes[nd.right].start = nd.mid;
        nodes[nd.right].end = nd.end;
        atomicMax(&ls->max_next, max(nd.mid - nd.start, nd.end - nd.mid));
      }
    }
  }
}

// Stable scatter of one chunk by warp ballots: warp w of the block moves points
// [begin + 128 w, begin + 128 (w + 1)) in four rounds of 32, so left and right runs are
// written contiguously.  The points that go to the node's smaller child are summed on
// the way (the sums of the large node's smaller child); each warp adds its sums with
// 128-bit atomics, so the chunk needs one block barrier (for the warps' left counts).
__global__ void __launch_bounds__(kThreads) k_big_scatter(const Chunk* chunks, const LevelState* ls,
                                                          const BNode* nodes, PointBufs B,
                                                          const int32_t* chunk_loff, const double* ts0, U128* accl) {
  constexpr int kPer = kChunk / kThreads;  // rounds of 32 points per warp
  constexpr int kWarpsB = kThreads / 32;
  static_assert(kPer * kThreads == kChunk, "chunk = block x rounds");
  __shared__ int swl[2][kWarpsB];  // left counts of the chunk's warps, by chunk parity
  const int nc = ls->num_chunks, cur = ls->cur;
  const float4* pin = B.p[cur];
  const double* sts = B.st;
  float4* pout = B.p[cur ^ 1];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  int par = 0;
  for (int ci = blockIdx.x; ci < nc; ci += gridDim.x) {
    const Chunk c = chunks[ci];
    const BNode& nd = nodes[c.node];
    if (!nd.split) {
      for (int i = c.begin + threadIdx.x; i < c.end; i += blockDim.x) B.perm[i] = __float_as_int(pin[i].w);
      continue;  // uniform per block
    }
    const float mean[3] = {nd.mean[0], nd.mean[1], nd.mean[2]};
    const float dir[3] = {nd.dir[0], nd.dir[1], nd.dir[2]};
    const int wb = c.begin + w * 32 * kPer;  // this warp's first point
    float4 pv[kPer];
    unsigned bl[kPer], bv[kPer];
    int nl = 0;
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int i = wb + u * 32 + lane;
      if (i < c.end) pv[u] = pin[i];
    }
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int i = wb + u * 32 + lane;
      bv[u] = __ballot_sync(0xffffffffu, i < c.end);
      bl[u] = __ballot_sync(0xffffffffu, i < c.end && which_side_f(mean, dir, pv[u]));
      nl += __popc(bl[u]);
    }
    if (lane == 0) swl[par][w] = nl;
    __syncthreads();
    int lpre = 0;  // left points of the chunk's earlier warps
    for (int k = 0; k < w; ++k) lpre += swl[par][k];
    const int nl_total = nd.mid - nd.start;
    const int before = min(wb, c.end) - nd.start;  // the node's points before this warp's
    int lo = nd.start + chunk_loff[ci] + lpre;
    int ro = nd.mid + before - (chunk_loff[ci] + lpre);
    const bool small_left = nl_total <= nd.end - nd.mid;
    const double t0 = ts0[nd.tree];
    Moments M;
    for (int k = 0; k < 11; ++k) M.s[k] = u128_zero();
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const unsigned br = bv[u] & ~bl[u];
      if ((bv[u] >> lane) & 1u) {
        const bool left = (bl[u] >> lane) & 1u;
        const int dst = left ? lo + __popc(bl[u] & lt) : ro + __popc(br & lt);
        pout[dst] = pv[u];
        if (left == small_left) moments_add_point(M, pv[u], sts[__float_as_int(pv[u].w)], t0);
      }
      lo += __popc(bl[u]);
      ro += __popc(br);
    }
    {  // the warp's sums straight into its node's accumulators (exact integers: any order)
      const U128 q = warp_sum_moments(M, lane);
      if (!(lane & 1) && lane < 22) atomic_add_u128(&accl[(size_t)c.big * 11 + (lane >> 1)], q);
    }
    par ^= 1;  // the barrier above keeps warps within one split chunk of each other
  }
}

// Children's sums of the large split nodes: the smaller from accl, the other = parent - it.
__global__ void k_big_childmom(const BNode* nodes, LevelState* ls, const int32_t* big_list, const U128* accl,
                               U128* mom, const int32_t* bsum, int nblocks, int32_t* level_begin, unsigned* done) {
  const int nb = ls->num_big;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nb * 11; t += gridDim.x * blockDim.x) {
    const int b = t / 11, k = t % 11;
    const int i = big_list[b];
    if (!nodes[i].split) continue;
    const U128 q = accl[t];  // the smaller child's sums
    const U128 other = u128_sub(mom[(size_t)i * 11 + k], q);
    const bool small_left = nodes[i].mid - nodes[i].start <= nodes[i].end - nodes[i].mid;
    mom[(size_t)nodes[i].left * 11 + k] = small_left ? q : other;
    mom[(size_t)nodes[i].right * 11 + k] = small_left ? other : q;
  }
  advance_if_last(ls, bsum, nblocks, level_begin, done);
}

// ---- children ------------------------------------------------------------------------

__global__ void k_level_children(BNode* nodes, LevelState* ls, const int32_t* bsum, int32_t cap) {
  __shared__ int sm[32];
  int b, e;
  level_range(ls, b, e);
  const int le = ls->le;
  int pre;  // split nodes of the blocks before this one
  {
    int v = 0;
    for (int k = threadIdx.x; k < (int)blockIdx.x; k += blockDim.x) v += bsum[k];
    block_scan(v, sm, &pre);
  }
  int carry = 0;
  for (int base = b; base < e; base += blockDim.x) {
    int i = base + threadIdx.x;
    bool sp = (i < e) && nodes[i].split;
    int tot;
    int r = block_scan(sp ? 1 : 0, sm, &tot) + carry + pre;
    carry += tot;
    if (i < e) {
      BNode& nd = nodes[i];
      if (!sp) {
        nd.left = -1;
        nd.right = -1;
      } else {
        int li = le + 2 * r;
        if (li + 1 >= cap) {
          ls->error = 1;
          nd.split = 0;
          nd.left = nd.right = -1;
        } else {
          nd.left = li;
          nd.right = li + 1;
          for (int k = 0; k < 2; ++k) {
            BNode c;
            memset(&c, 0, sizeof(c));  // start/end: set by the partition
            c.level = nd.level + 1;
            c.tree = nd.tree;
            c.left = c.right = -1;
            c.parent = i;
            c.has_parent = 1;
            c.par_has = nd.has_prop;
            for (int j = 0; j < 3; ++j) c.par_prop[j] = nd.prop[j];
            nodes[li + k] = c;
          }
        }
      }
    }
  }
}

// ---- deep levels: whole subtrees in shared memory --------------------------------------
// Once every node of a level has at most kDeepMax points, each of them is the root of a
// subtree that one warp builds to the end in its own slice of shared memory: the points
// are loaded once, and every depth below runs the same steps as the level kernels --
// decide (lane per node, from the node's exact sums), children numbered by a warp scan,
// stable ballot partition by whichSide (the warp per node) with the smaller child summed
// on the way (the other = parent - smaller).  The arithmetic and the partition order are
// those of k_decide / k_small_part, so the nodes are bit-identical to a level-by-level
// build.  The warps of a block share nothing and never wait for each other.  Nodes below
// the roots are written as DeepNode records tagged (subtree, depth, rank); k_deep_place
// then puts them at their breadth-first positions: depth by depth, subtree by subtree in
// the roots' order, by rank inside a subtree -- the order in which the level kernels
// would have numbered them.
constexpr int kDeepMax = 256;      // largest subtree root (points)
// The subtree pass runs only while the level has at most this many nodes: it finishes a
// few thousand subtrees in about one subtree's latency, which beats the level kernels'
// launches for single trees and small batches; for large forests (hundreds of thousands
// of tiny subtrees, where a warp's decide runs on a few lanes) the level kernels, with a
// thread per node of the whole level, are faster.
constexpr int kDeepMaxRoots = 8192;
constexpr int kDeepNodes = 192;    // nodes of one depth: at most 2 x (kDeepMax / 3) split children
constexpr int kDeepWarpsPerBlock = 4;
constexpr int kDeepThreads = 32 * kDeepWarpsPerBlock;
constexpr int kDeepBlocksPerSM = 4;
static_assert(kDeepMax <= kBig, "deep subtree roots are summed by k_root_moments");
static_assert(2 * (kDeepMax / 3) <= kDeepNodes, "node capacity of one depth");

struct DeepNode {
  float mean[3], dir[3];
  double dts_mean, dts_cov;
  double prop[3];
  int32_t start, end;     // point offsets inside the subtree
  int32_t sub;            // subtree ordinal: its root is node lb + sub
  int32_t depth;          // >= 1: levels below the root
  int32_t rank;           // breadth-first position among the subtree's nodes of this depth
  int32_t q;              // split nodes: children ranks 2q, 2q + 1; leaves: -1
  int32_t parent_rank;    // rank of the parent at depth - 1
  int32_t has_prop;
};
static_assert(sizeof(DeepNode) == 96, "DeepNode layout");
static_assert(sizeof(DeepNode) <= 11 * sizeof(U128), "a DeepNode fits the sums slot of one node");

struct DeepWarpSmem {                // one warp's slice
  float4 pts[2][kDeepMax];           // the 16 B point records (w = input index)
  uint32_t range[2][kDeepNodes];     // node start | end << 16 (subtree offsets), by depth parity
  int32_t prank[2][kDeepNodes];      // parent's rank, by depth parity
  int32_t list[kDeepNodes];          // q -> rank of the q-th split node of the depth
  uint8_t split[kDeepNodes];
};

__global__ void __launch_bounds__(kDeepThreads, kDeepBlocksPerSM)
    k_deep_build(BNode* nodes, LevelState* ls, PointBufs B, const double* ts0, const U128* mom, BuildParams P,
                 double* root_frame, DeepNode* dn, int32_t dn_cap, int32_t* dn_count, U128* ring, int32_t* counts,
                 int32_t dcap) {
  extern __shared__ __align__(16) unsigned char deep_smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  DeepWarpSmem& S = reinterpret_cast<DeepWarpSmem*>(deep_smem_raw)[wib];
  const int lb = ls->lb, le = ls->le, cur0 = ls->cur;
  const int nroots = le - lb;
  const unsigned full = 0xffffffffu, lt = (1u << lane) - 1u;
  const int gw = blockIdx.x * kDeepWarpsPerBlock + wib, nw = gridDim.x * kDeepWarpsPerBlock;
  U128* myring = ring + (size_t)gw * 2 * kDeepNodes * 11;
  const float4* pin = B.p[cur0];
  const double* sts = B.st;
  for (int sub = gw; sub < nroots; sub += nw) {
    const int R = lb + sub;
    const BNode root = nodes[R];
    const int n = root.end - root.start;
    const int pbase = root.start;
    const double t0 = ts0[root.tree];
    for (int i = lane; i < n; i += 32) S.pts[0][i] = pin[pbase + i];
    if (lane == 0) {
      S.range[0][0] = (uint32_t)n << 16;
      S.prank[0][0] = -1;
    }
    __syncwarp();
    int cnt = 1, c = 0, base = 0, base_prev = 0;
    for (int d = 0; cnt > 0; ++d, c ^= 1) {
      // ---- decide: lane per node of this depth; record slots for the depth's nodes
      if (d > 0) {
        base_prev = base;
        int b = 0;
        if (lane == 0) b = atomicAdd(dn_count, cnt);
        base = __shfl_sync(full, b, 0);
        if (base + cnt > dn_cap) {
          if (lane == 0) ls->error = 1;  // out of record slots: the build reports KDS_ERR_CAPACITY
          break;
        }
      }
      const U128* psums = d == 0 ? mom + (size_t)R * 11 : myring + (size_t)(d & 1) * kDeepNodes * 11;
      for (int r = lane; r < cnt; r += 32) {
        const uint32_t rg = S.range[c][r];
        const int st = (int)(rg & 0xffffu), en = (int)(rg >> 16);
        BNode nd;
        if (d == 0) {
          nd = root;
        } else {
          memset(&nd, 0, sizeof(nd));
          nd.level = root.level + d;
          nd.tree = root.tree;
          nd.has_parent = 1;
          if (d == 1) {  // the root's decision, written at depth 0
            for (int k = 0; k < 3; ++k) nd.par_prop[k] = nodes[R].prop[k];
            nd.par_has = nodes[R].has_prop;
          } else {
            const DeepNode& pn = dn[base_prev + S.prank[c][r]];
            nd.par_has = pn.has_prop;
            for (int k = 0; k < 3; ++k) nd.par_prop[k] = pn.prop[k];
          }
        }
        double Sd[11];
        const U128* ms = d == 0 ? psums : psums + (size_t)r * 11;
        for (int k = 0; k < 11; ++k) Sd[k] = fx_to_d(ms[k]);
        decide(Sd, en - st, nd, P, nd.level == 0 ? root_frame + (size_t)nd.tree * kRootFrame : nullptr);
        S.split[r] = nd.split ? 1 : 0;
        if (d == 0) {
          nodes[R] = nd;  // left / right follow in k_deep_place
        } else {
          DeepNode x;
          for (int k = 0; k < 3; ++k) {
            x.mean[k] = nd.mean[k];
            x.dir[k] = nd.dir[k];
            x.prop[k] = nd.prop[k];
          }
          x.dts_mean = nd.dts_mean;
          x.dts_cov = nd.dts_cov;
          x.start = st;
          x.end = en;
          x.sub = sub;
          x.depth = d;
          x.rank = r;
          x.q = -1;
          x.parent_rank = S.prank[c][r];
          x.has_prop = nd.has_prop;
          dn[base + r] = x;
        }
      }
      __syncwarp();
      // ---- children numbering: split ranks by a warp scan in rank order
      int nsplit = 0;
      for (int r0 = 0; r0 < cnt; r0 += 32) {
        const int r = r0 + lane;
        const bool f = r < cnt && S.split[r];
        const unsigned bf = __ballot_sync(full, f);
        if (f) {
          const int q = nsplit + __popc(bf & lt);
          S.list[q] = r;
          if (d > 0) dn[base + r].q = q;
        }
        nsplit += __popc(bf);
      }
      if (2 * nsplit > kDeepNodes) {  // cannot happen (split nodes hold >= 3 points); refuse rather than overrun
        if (lane == 0) ls->error = 1;
        break;
      }
      if (nsplit > 0 && lane == 0) {
        if (d + 1 < dcap) counts[(size_t)(d + 1) * nroots + sub] = 2 * nsplit;
        else ls->error = 1;
      }
      __syncwarp();
      // ---- the leaves' point order (lane per leaf)
      for (int r = lane; r < cnt; r += 32) {
        if (S.split[r]) continue;
        const uint32_t rg = S.range[c][r];
        const int st = (int)(rg & 0xffffu), en = (int)(rg >> 16);
        for (int i = st; i < en; ++i) B.perm[pbase + i] = __float_as_int(S.pts[c][i].w);
      }
      // ---- partition of the split nodes, the warp per node
      for (int q = 0; q < nsplit; ++q) {
        const int r = S.list[q];
        const uint32_t rg = S.range[c][r];
        const int st = (int)(rg & 0xffffu), en = (int)(rg >> 16);
        float mean[3], dir[3];
        if (d == 0) {
          for (int k = 0; k < 3; ++k) { mean[k] = nodes[R].mean[k]; dir[k] = nodes[R].dir[k]; }
        } else {
          const DeepNode& x = dn[base + r];
          for (int k = 0; k < 3; ++k) { mean[k] = x.mean[k]; dir[k] = x.dir[k]; }
        }
        int nl = 0;
        for (int k0 = st; k0 < en; k0 += 32) {
          const int i = k0 + lane;
          const bool left = i < en && which_side_f(mean, dir, S.pts[c][i]);
          nl += __popc(__ballot_sync(full, left));
        }
        const int mid = st + nl;
        const bool small_left = mid - st <= en - mid;
        Moments MS;
        for (int k = 0; k < 11; ++k) MS.s[k] = u128_zero();
        int cl = 0, cr = 0;
        for (int k0 = st; k0 < en; k0 += 32) {
          const int i = k0 + lane;
          const bool valid = i < en;
          float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
          if (valid) p = S.pts[c][i];
          const bool left = valid && which_side_f(mean, dir, p);
          const unsigned bl = __ballot_sync(full, left);
          const unsigned br = __ballot_sync(full, valid && !left);
          if (valid) {
            const int dst = left ? (st + cl + __popc(bl & lt)) : (mid + cr + __popc(br & lt));
            S.pts[c ^ 1][dst] = p;
            if (left == small_left) moments_add_point(MS, p, sts[__float_as_int(p.w)], t0);
          }
          cl += __popc(bl);
          cr += __popc(br);
        }
        const U128 qs = warp_sum_moments(MS, lane);
        if (!(lane & 1) && lane < 22) {
          const int k = lane >> 1;
          const U128 ps = d == 0 ? psums[k] : psums[(size_t)r * 11 + k];
          const U128 other = u128_sub(ps, qs);
          U128* nxt = myring + (size_t)((d + 1) & 1) * kDeepNodes * 11;
          nxt[(size_t)(2 * q) * 11 + k] = small_left ? qs : other;
          nxt[(size_t)(2 * q + 1) * 11 + k] = small_left ? other : qs;
        }
        if (lane == 0) {
          S.range[c ^ 1][2 * q] = (uint32_t)st | ((uint32_t)mid << 16);
          S.range[c ^ 1][2 * q + 1] = (uint32_t)mid | ((uint32_t)en << 16);
          S.prank[c ^ 1][2 * q] = r;
          S.prank[c ^ 1][2 * q + 1] = r;
        }
      }
      cnt = 2 * nsplit;
      if (d + 1 >= dcap) cnt = 0;
      __syncwarp();
    }
    __syncwarp();
  }
}

// Deep nodes to their breadth-first positions: node (subtree s, depth d, rank r) goes to
// le + off[d * nroots + s] + r, where off is the exclusive scan of the per-(depth,
// subtree) node counts in depth-major order.  The roots get their children's indices.
__global__ void k_deep_place(BNode* nodes, LevelState* ls, const DeepNode* dn, const int32_t* dn_count,
                             int32_t dn_cap, const int32_t* off, int32_t dcap, int32_t cap_nodes) {
  if (ls->error) return;  // the build fails; records may be missing
  const int lb = ls->lb, le = ls->le;
  const int nroots = le - lb;
  const int nd_total = min(*dn_count, dn_cap);
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nroots; i += stride) {
    BNode& rt = nodes[lb + i];
    if (rt.split && dcap > 1) {
      rt.left = le + off[(size_t)1 * nroots + i];
      rt.right = rt.left + 1;
    } else {
      rt.left = rt.right = -1;
    }
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nd_total; i += stride) {
    const DeepNode x = dn[i];
    const int s = x.sub, d = x.depth;
    const BNode& rt = nodes[lb + s];
    BNode o;
    memset(&o, 0, sizeof(o));
    o.start = rt.start + x.start;
    o.end = rt.start + x.end;
    o.level = rt.level + d;
    o.tree = rt.tree;
    o.split = x.q >= 0 ? 1 : 0;
    o.mid = o.end;
    o.left = o.right = -1;
    if (x.q >= 0 && d + 1 < dcap) {
      o.left = le + off[(size_t)(d + 1) * nroots + s] + 2 * x.q;
      o.right = o.left + 1;
    }
    o.has_parent = 1;
    o.has_prop = x.has_prop;
    o.parent = d == 1 ? lb + s : le + off[(size_t)(d - 1) * nroots + s] + x.parent_rank;
    for (int k = 0; k < 3; ++k) {
      o.mean[k] = x.mean[k];
      o.dir[k] = x.dir[k];
      o.prop[k] = x.prop[k];
    }
    o.dts_mean = x.dts_mean;
    o.dts_cov = x.dts_cov;
    const int g = le + off[(size_t)d * nroots + s] + x.rank;
    if (g >= cap_nodes) {
      ls->error = 1;
      continue;
    }
    nodes[g] = o;
  }
}

// One thread: the level state after the deep levels (every level done), the begin of
// each deep level, the depth, and the node capacity check.
__global__ void k_deep_finish(LevelState* ls, const int32_t* off, const int32_t* total, int32_t dcap,
                              int32_t cap_nodes, int32_t* level_begin) {
  if (blockIdx.x != 0 || threadIdx.x != 0 || ls->error) return;
  const int lb = ls->lb, le = ls->le;
  const int nroots = le - lb;
  const int tot = *total;
  int dmax = 0;  // deepest local depth holding nodes
  for (int d = 1; d < dcap; ++d) {
    const int b = off[(size_t)d * nroots];
    const int e = d + 1 < dcap ? off[(size_t)(d + 1) * nroots] : tot;
    if (e > b) {
      dmax = d;
      if (ls->depth + d < kMaxDepth + 1) level_begin[ls->depth + d] = le + b;
    }
  }
  if (le + tot > cap_nodes) ls->error = 1;
  ls->depth += dmax + 1;
  ls->lb = ls->le = le + tot;
  if (ls->depth < kMaxDepth + 1) level_begin[ls->depth] = ls->lb;
}

// ---- prune and per-tree compaction -----------------------------------------------------
// Prune in one launch (alive[] zeroed before): a leaf lives if it passes
// IsGoodLeafPredicate_ (kd/tree/tree_predicates_.h:18-29, in float), an inner node if
// any child lives, i.e. if a good leaf lies below it (kd/tree/tree_cpu_.h:172-196).  Each
// good leaf marks its ancestors up to the first one already marked: whoever marks a node
// first goes on to its parent, so every ancestor ends marked whatever the order.
__global__ void k_alive(const BNode* nodes, int32_t total, int32_t* alive, float incidence) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const BNode& nd = nodes[i];
    if (nd.left >= 0 || nd.right >= 0) continue;
    F3 d = f3(nd.dir[0], nd.dir[1], nd.dir[2]);
    F3 m = f3(nd.mean[0], nd.mean[1], nd.mean[2]);
    if (!(dot3x(d, d) > 0.0f && fabsf(dot3x(m, d)) > incidence)) continue;
    alive[i] = 1;
    for (int p = nd.parent; p >= 0; p = nodes[p].parent) {
      if (((volatile int32_t*)alive)[p]) break;
      alive[p] = 1;
    }
  }
}

// group = (level, tree); nodes of one group are contiguous in global order
// Counts per (level, tree) group; lanes with the same group combine their counts
// before one atomic per group and warp.
__global__ void k_group_counts(const BNode* nodes, int32_t total, const int32_t* alive, int R, int32_t* cnt,
                               int32_t* lcnt, int32_t* ucnt, int32_t* leaf_flag) {
  const int lane = threadIdx.x & 31;
  for (int base = blockIdx.x * blockDim.x; base < total; base += gridDim.x * blockDim.x) {
    const int i = base + threadIdx.x;
    const bool valid = i < total;
    int tree = -1, g = -1;
    bool al = false, leaf = false;
    if (valid) {
      const BNode& nd = nodes[i];
      tree = nd.tree;
      g = nd.level * R + nd.tree;
      al = alive[i] != 0;
      leaf = al && nd.left < 0 && nd.right < 0;
      leaf_flag[i] = leaf ? 1 : 0;
    }
    const unsigned pt = __match_any_sync(0xffffffffu, tree);
    if (valid && lane == __ffs(pt) - 1) atomicAdd(&ucnt[tree], __popc(pt));
    const unsigned pg = __match_any_sync(0xffffffffu, g);
    const unsigned ba = __ballot_sync(0xffffffffu, al);
    const unsigned bl = __ballot_sync(0xffffffffu, leaf);
    if (valid && lane == __ffs(pg) - 1) {
      const int c = __popc(pg & ba), lc = __popc(pg & bl);
      if (c) atomicAdd(&cnt[g], c);
      if (lc) atomicAdd(&lcnt[g], lc);
    }
  }
}

// Exclusive prefix over groups in (level, tree) order (one block, scans with carry),
// and per-tree level offsets (one thread per tree).
__global__ void k_group_tables(int depth, int R, const int32_t* cnt, const int32_t* lcnt, int32_t* gp, int32_t* lgp,
                               int32_t* to, int32_t* lto, int32_t* tot_nodes, int32_t* tot_leaves) {
  __shared__ int sm[32];
  const int G = depth * R;
  int carry = 0, lcarry = 0;
  for (int base = 0; base < G; base += blockDim.x) {
    const int g = base + threadIdx.x;
    const int c = g < G ? cnt[g] : 0, lc = g < G ? lcnt[g] : 0;
    int tc, tl;
    const int o = block_scan(c, sm, &tc);
    const int lo = block_scan(lc, sm, &tl);
    if (g < G) {
      gp[g] = carry + o;
      lgp[g] = lcarry + lo;
    }
    carry += tc;
    lcarry += tl;
  }
  for (int t = threadIdx.x; t < R; t += blockDim.x) {
    int s = 0, ls = 0;
    for (int l = 0; l < depth; ++l) {
      const int g = l * R + t;
      to[g] = s;
      lto[g] = ls;
      s += cnt[g];
      ls += lcnt[g];
    }
    tot_nodes[t] = s;
    tot_leaves[t] = ls;
  }
}

__global__ void k_compact_forest(const BNode* nodes, int32_t total, const int32_t* alive, const int32_t* rank,
                                 const int32_t* leaf_flag, const int32_t* lrank, int R, const int32_t* gp,
                                 const int32_t* lgp, const int32_t* to, const int32_t* lto, TreeDev* trees) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    if (!alive[i]) continue;
    const BNode& nd = nodes[i];
    TreeDev& T = trees[nd.tree];
    if (T.nodes == nullptr) continue;  // rejected tree
    int g = nd.level * R + nd.tree;
    int o = to[g] + (rank[i] - gp[g]);
    int gc = (nd.level + 1) * R + nd.tree;
    int l = (nd.left >= 0 && alive[nd.left]) ? to[gc] + (rank[nd.left] - gp[gc]) : -1;
    int r = (nd.right >= 0 && alive[nd.right]) ? to[gc] + (rank[nd.right] - gp[gc]) : -1;
    DNode d;
    d.a = make_float4(nd.mean[0], nd.mean[1], nd.mean[2], nd.dir[0]);
    d.b = make_float4(nd.dir[1], nd.dir[2], __int_as_float(l), __int_as_float(r));
    T.nodes[o] = d;
    T.dts_f[o] = (float)nd.dts_mean;
    T.dts_mean[o] = nd.dts_mean;
    T.dts_cov[o] = nd.dts_cov;
    int64_t base = nd.start;  // ranges are global; made tree-relative below
    T.range[2 * o] = base;
    T.range[2 * o + 1] = nd.end;
    T.level[o] = nd.level;
    if (leaf_flag[i]) T.leaf_idx[lto[g] + (lrank[i] - lgp[g])] = o;
  }
}

// tree-relative point ranges and point order; blockIdx.y = tree
__global__ void k_finish_trees(TreeDev* trees, const int64_t* off, const int32_t* perm_final) {
  const int r = blockIdx.y;
  TreeDev& T = trees[r];
  if (T.nodes == nullptr) return;
  const int64_t o0 = off[r];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < T.num_nodes;
       i += (int64_t)gridDim.x * blockDim.x) {
    T.range[2 * i] -= o0;
    T.range[2 * i + 1] -= o0;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < T.num_points;
       i += (int64_t)gridDim.x * blockDim.x)
    T.perm[i] = perm_final[o0 + i] - (int32_t)o0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < T.num_leaves;
       i += (int64_t)gridDim.x * blockDim.x) {
    int o = T.leaf_idx[i];
    DNode d = T.nodes[o];
    T.leaf_md[i] = make_float4(d.a.x, d.a.y, d.a.z, T.dts_f[o]);
    T.leaf_nrm[i] = make_float4(d.a.w, d.b.x, d.b.y, 0.f);
  }
}

inline int nblk(int64_t n, int t) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + t - 1) / t, 1 << 20)); }

template <class T> T* carve(char*& p, size_t count) {
  size_t bytes = (count * sizeof(T) + 255) & ~(size_t)255;
  T* r = reinterpret_cast<T*>(p);
  p += bytes;
  return r;
}
template <class T> size_t carve_size(size_t count) { return (count * sizeof(T) + 255) & ~(size_t)255; }

struct BuildWs {
  void* block = nullptr;
  PointBufs B;
  BNode* nodes;
  int32_t *alive, *rank, *leaf_flag, *lrank, *tile_sums;
  Chunk* chunks;
  int32_t *chunk_nl, *chunk_loff, *big_list, *node_chunk0;
  U128* acc;
  U128* accl;  // left-child sums of the level's large nodes
  U128* mom;   // exact sums of every node (11 per node)
  double* ts0;
  double* root_frame;  // kRootFrame per cloud (k_decide at level 0)
  unsigned long long* tsmin;
  int64_t* off;
  LevelState* ls;
  int32_t* level_begin;
  unsigned* done;  // last-block counter of the level's last kernel
  int32_t* bsum;
  int32_t* bbig;  // per-block (chunks, large nodes) of the level
  int32_t *cnt, *lcnt, *ucnt, *gp, *lgp, *to, *lto, *tot_nodes, *tot_leaves, *scan_tot;
  TreeDev* trees;
  int64_t cap_nodes;
  int32_t chunk_cap;
};

// Bytes of the build workspace for n points in R clouds.
size_t ws_bytes(int64_t n, int R) {
  const int64_t cn = 2 * n + 4096 + 4 * (int64_t)R;
  const int64_t chunk_cap = n / kChunk + n / kBig + 16;
  const int64_t ntiles = cn / 4096 + 2;
  const int64_t G = (int64_t)(kMaxDepth + 2) * R;
  return 2 * carve_size<float4>(n) + carve_size<double>(n) + carve_size<int32_t>(n) +
         carve_size<BNode>(cn) + 4 * carve_size<int32_t>(cn) + carve_size<int32_t>(ntiles) +
         carve_size<Chunk>(chunk_cap) + 4 * carve_size<int32_t>(chunk_cap) +
         2 * carve_size<U128>((size_t)11 * (n / kBig + 2)) + carve_size<U128>((size_t)11 * cn) + 2 * carve_size<double>(R) +
         carve_size<double>((size_t)kRootFrame * R) + carve_size<int64_t>(R + 1) +
         carve_size<LevelState>(1) + carve_size<int32_t>(kMaxDepth + 2) + carve_size<unsigned>(1) +
         carve_size<int32_t>(kLevelBlocks) +
         carve_size<int32_t>(2 * kLevelBlocks) +
         7 * carve_size<int32_t>(G) + 3 * carve_size<int32_t>(R) + carve_size<int32_t>(8) + carve_size<TreeDev>(R) +
         256;
}

int ws_alloc(BuildWs& w, int64_t n, int R, cudaStream_t s) {
  w.cap_nodes = 2 * n + 4096 + 4 * (int64_t)R;
  w.chunk_cap = (int32_t)(n / kChunk + n / kBig + 16);
  const int64_t cn = w.cap_nodes;
  const int64_t ntiles = cn / 4096 + 2;
  const int64_t G = (int64_t)(kMaxDepth + 2) * R;
  const size_t bytes = ws_bytes(n, R);
  cudaError_t e = cudaMallocAsync(&w.block, bytes, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    w.block = nullptr;
    set_error("cudaMallocAsync of %zu bytes for the tree build workspace failed: %s", bytes, cudaGetErrorString(e));
    return KDS_ERR_OOM;
  }
  char* p = (char*)w.block;
  w.B.p[0] = carve<float4>(p, n);
  w.B.p[1] = carve<float4>(p, n);
  w.B.st = carve<double>(p, n);
  w.B.perm = carve<int32_t>(p, n);
  w.nodes = carve<BNode>(p, cn);
  w.alive = carve<int32_t>(p, cn);
  w.rank = carve<int32_t>(p, cn);
  w.leaf_flag = carve<int32_t>(p, cn);
  w.lrank = carve<int32_t>(p, cn);
  w.tile_sums = carve<int32_t>(p, ntiles);
  w.chunks = carve<Chunk>(p, w.chunk_cap);
  w.chunk_nl = carve<int32_t>(p, w.chunk_cap);
  w.chunk_loff = carve<int32_t>(p, w.chunk_cap);
  w.big_list = carve<int32_t>(p, w.chunk_cap);
  w.node_chunk0 = carve<int32_t>(p, w.chunk_cap);
  w.acc = carve<U128>(p, (size_t)11 * (n / kBig + 2));
  w.accl = carve<U128>(p, (size_t)11 * (n / kBig + 2));
  w.mom = carve<U128>(p, (size_t)11 * cn);
  w.ts0 = carve<double>(p, R);
  w.root_frame = carve<double>(p, (size_t)kRootFrame * R);
  w.tsmin = carve<unsigned long long>(p, R);
  w.off = carve<int64_t>(p, R + 1);
  w.ls = carve<LevelState>(p, 1);
  w.level_begin = carve<int32_t>(p, kMaxDepth + 2);
  w.done = carve<unsigned>(p, 1);
  w.bsum = carve<int32_t>(p, kLevelBlocks);
  w.bbig = carve<int32_t>(p, 2 * kLevelBlocks);
  w.cnt = carve<int32_t>(p, G);
  w.lcnt = carve<int32_t>(p, G);
  w.gp = carve<int32_t>(p, G);
  w.lgp = carve<int32_t>(p, G);
  w.to = carve<int32_t>(p, G);
  w.lto = carve<int32_t>(p, G);
  w.ucnt = carve<int32_t>(p, G);
  w.tot_nodes = carve<int32_t>(p, R);
  w.tot_leaves = carve<int32_t>(p, R);
  w.scan_tot = carve<int32_t>(p, R);
  w.trees = carve<TreeDev>(p, R);
  return KDS_OK;
}

}  // namespace

namespace {

// The deep levels of a build whose current level (h, read at the last sync) has no node
// above kDeepMax points: k_deep_build, the depth-major scan of the per-(depth, subtree)
// node counts, k_deep_place, k_deep_finish.  The node records of the deep levels are
// staged in the unused part of the sums array (slots from le on).
int deep_pass(BuildWs& w, const BuildParams& P, const LevelState& h, cudaStream_t s) {
  const int lb = h.lb, le = h.le;
  const int nroots = le - lb;
  if (nroots <= 0) return KDS_OK;
  const int dcap = std::max(1, P.max_level - h.depth);
  DeepNode* dn = reinterpret_cast<DeepNode*>(w.mom + (size_t)le * 11);
  const int64_t dn_cap64 = ((w.cap_nodes - le) * (int64_t)(11 * sizeof(U128))) / (int64_t)sizeof(DeepNode);
  const int32_t dn_cap = (int32_t)std::min<int64_t>(dn_cap64, INT32_MAX);
  const int grid = (int)std::min<int64_t>((nroots + kDeepWarpsPerBlock - 1) / kDeepWarpsPerBlock,
                                          148 * kDeepBlocksPerSM);
  const int64_t nwarps = (int64_t)grid * kDeepWarpsPerBlock;
  const int64_t ncount = (int64_t)dcap * nroots;
  if (ncount > INT32_MAX / 2) { set_error("kds_tree_build: too many deep subtrees"); return KDS_ERR_CAPACITY; }
  const size_t bc = carve_size<int32_t>(ncount), bt = carve_size<int32_t>(ncount / 4096 + 2),
               br = carve_size<U128>((size_t)nwarps * 2 * kDeepNodes * 11);
  void* blk = nullptr;
  cudaError_t e = cudaMallocAsync(&blk, 2 * bc + bt + 3 * 256 + br, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("cudaMallocAsync for the deep tree levels failed: %s", cudaGetErrorString(e));
    return KDS_ERR_OOM;
  }
  char* p = (char*)blk;
  int32_t* counts = carve<int32_t>(p, ncount);
  int32_t* off = carve<int32_t>(p, ncount);
  int32_t* tiles = carve<int32_t>(p, ncount / 4096 + 2);
  int32_t* total = carve<int32_t>(p, 1);
  int32_t* dn_count = carve<int32_t>(p, 1);
  carve<int32_t>(p, 1);
  U128* ring = carve<U128>(p, (size_t)nwarps * 2 * kDeepNodes * 11);
  int rc = KDS_OK;
  static std::atomic<bool> attr_set{false};  // a property of the kernel, per process (builds may run on two threads)
  if (!attr_set.load()) {
    e = cudaFuncSetAttribute((const void*)k_deep_build, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(DeepWarpSmem) * kDeepWarpsPerBlock));
    if (e == cudaSuccess) attr_set.store(true);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(counts, 0, sizeof(int32_t) * ncount, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(dn_count, 0, sizeof(int32_t), s);
  if (e == cudaSuccess) {
    k_deep_build<<<grid, kDeepThreads, sizeof(DeepWarpSmem) * kDeepWarpsPerBlock, s>>>(w.nodes, w.ls, w.B, w.ts0, w.mom, P, w.root_frame, dn,
                                                              dn_cap, dn_count, ring, counts, dcap);
    count_launch();
    rc = scan_exclusive(counts, off, (int32_t)ncount, tiles, total, s);
    const int pg = (int)std::min<int64_t>(nblk(std::max<int64_t>(w.cap_nodes - le, nroots), kThreads), kGridBlocks * 4);
    k_deep_place<<<pg, kThreads, 0, s>>>(w.nodes, w.ls, dn, dn_count, dn_cap, off, dcap, (int32_t)w.cap_nodes);
    k_deep_finish<<<1, 32, 0, s>>>(w.ls, off, total, dcap, (int32_t)w.cap_nodes, w.level_begin);
    count_launch();
    count_launch();
    e = cudaGetLastError();
  }
  cudaFreeAsync(blk, s);
  if (e != cudaSuccess) return cuda_status(e, "deep tree levels", __FILE__, __LINE__);
  return rc;
}

}  // namespace

size_t forest_workspace_bytes(int64_t n, int R) { return ws_bytes(std::max<int64_t>(n, 1), std::max(R, 1)); }

// Builds R trees from R clouds stored back to back (offsets[R+1] on the host).
// out[r] = NULL and status[r] = KDS_ERR_TREE_REJECTED where makeTree returns nullptr.
// Page-locked staging for the build's small device-to-host reads (the level state at each
// host check, the per-tree counts at the end) instead of pageable host memory: one block
// per host thread, grown on demand, released when the thread exits.
struct PinnedStage {
  void* p = nullptr;
  size_t cap = 0;
  ~PinnedStage() {
    if (p) cudaFreeHost(p);
  }
  void* get(size_t bytes) {
    if (bytes > cap) {
      if (p) cudaFreeHost(p);
      p = nullptr;
      cap = 0;
      const size_t c = std::max<size_t>(bytes, 64 * 1024);
      if (cudaMallocHost(&p, c) != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        return nullptr;
      }
      cap = c;
    }
    return p;
  }
};

void* pinned_stage(size_t bytes) {
  thread_local PinnedStage st;
  return st.get(bytes);
}

int tree_build_forest(const float* xyz, const double* stamps, const int64_t* offsets, int32_t R, int32_t mem,
                      const kds_tree_params* prm, cudaStream_t s, kds_tree** out, int32_t* status) {
  for (int r = 0; r < R; ++r) { out[r] = nullptr; status[r] = KDS_ERR_TREE_REJECTED; }
  if (R <= 0) { set_error("kds_tree_build: no clouds"); return KDS_ERR_INVALID_ARG; }
  const int64_t N = offsets[R] - offsets[0];
  if (offsets[0] != 0 || N < 0 || N > ((int64_t)1 << 30)) {
    set_error("kds_tree_build: bad point count / offsets");
    return KDS_ERR_INVALID_ARG;
  }
  std::vector<int64_t> off(offsets, offsets + R + 1);
  int32_t max_size = 0;
  for (int r = 0; r < R; ++r) {
    if (off[r + 1] < off[r]) { set_error("kds_tree_build: offsets must be non-decreasing"); return KDS_ERR_INVALID_ARG; }
    max_size = std::max<int32_t>(max_size, (int32_t)(off[r + 1] - off[r]));
  }
  BuildParams P;
  P.propagate_normal = prm->propagate_normal;
  P.leaf_min_points = prm->leaf_min_points;
  P.leaf_max_points = prm->leaf_max_points;
  P.leaf_density = prm->leaf_density;
  P.leaf_min_normal_incidence = prm->leaf_min_normal_incidence;
  P.leaf_normal_eigenratio = prm->leaf_normal_eigenratio;
  P.prune_incidence = prm->prune_min_normal_incidence;
  P.max_level = prm->max_level > 0 ? std::min(prm->max_level, kMaxDepth) : 48;
  if (N == 0) return KDS_OK;  // every cloud rejected (fewer points than leaf_min_points)

  BuildWs w;
  int rc = ws_alloc(w, std::max<int64_t>(N, 1), R, s);
  if (rc) return rc;
  struct Guard {
    BuildWs* w;
    cudaStream_t s;
    void* h_xyz = nullptr;
    void* h_st = nullptr;
    ~Guard() {
      if (w->block) cudaFreeAsync(w->block, s);
      if (h_xyz) cudaFreeAsync(h_xyz, s);
      if (h_st) cudaFreeAsync(h_st, s);
    }
  } guard{&w, s};
  const float* d_xyz = xyz;
  const double* d_st = stamps;
  if (mem == KDS_MEM_HOST) {
    KDS_CK(cudaMallocAsync(&guard.h_xyz, sizeof(float) * 3 * N, s));
    KDS_CK(cudaMemcpyAsync(guard.h_xyz, xyz, sizeof(float) * 3 * N, cudaMemcpyHostToDevice, s));
    d_xyz = (const float*)guard.h_xyz;
    if (stamps) {
      KDS_CK(cudaMallocAsync(&guard.h_st, sizeof(double) * N, s));
      KDS_CK(cudaMemcpyAsync(guard.h_st, stamps, sizeof(double) * N, cudaMemcpyHostToDevice, s));
      d_st = (const double*)guard.h_st;
    }
  }
  KDS_CK(cudaMemsetAsync(w.ls, 0, sizeof(LevelState), s));
  KDS_CK(cudaMemsetAsync(w.done, 0, sizeof(unsigned), s));
  KDS_CK(cudaMemcpyAsync(w.off, off.data(), sizeof(int64_t) * (R + 1), cudaMemcpyHostToDevice, s));
  k_ingest<<<nblk(N, kThreads), kThreads, 0, s>>>(d_xyz, d_st, N, w.B.p[0], w.B.st, w.ls);
  count_launch();
  {
    KDS_CK(cudaMemsetAsync(w.tsmin, 0xff, sizeof(unsigned long long) * R, s));
    dim3 g((unsigned)std::min<int64_t>(std::max<int64_t>((max_size + kThreads - 1) / kThreads, 1), 64), (unsigned)R);
    k_tree_min<<<g, kThreads, 0, s>>>(w.B.st, w.off, w.tsmin);
    k_tree_check<<<g, kThreads, 0, s>>>(w.B.st, w.off, w.tsmin, w.ts0, w.ls);
    count_launch();
    count_launch();
  }
  k_init_roots<<<(R + 127) / 128, 128, 0, s>>>(w.nodes, w.off, R, w.ls, w.level_begin);
  count_launch();
  KDS_CK(cudaGetLastError());

  // pinned: [level state | per-tree nodes, leaves, unpruned nodes | ts0 | root frames]
  const size_t st_ls = (sizeof(LevelState) + 255) & ~(size_t)255;
  const size_t st_cnt = ((size_t)12 * R + 255) & ~(size_t)255;
  char* stage = (char*)pinned_stage(st_ls + st_cnt + sizeof(double) * (size_t)(1 + kRootFrame) * R);
  if (!stage) { set_error("kds_tree_build: page-locked staging of the level state failed"); return KDS_ERR_OOM; }
  LevelState& hls = *reinterpret_cast<LevelState*>(stage);
  int32_t* h_cnt = reinterpret_cast<int32_t*>(stage + st_ls);
  double* h_dbl = reinterpret_cast<double*>(stage + st_ls + st_cnt);
  int32_t host_max = max_size;
  const int cb = std::min<int>(w.chunk_cap, kGridBlocks * 2);
  // Grids of the level kernels sized to the level: a level has at most twice the nodes
  // of the one before, and the host learns the current level's size at each sync.  The
  // node-range kernels (k_decide, k_level_children, k_big_plan) share
  // one block count per level; every kernel's result is independent of its grid.
  int64_t level_nodes = R;
  int32_t global_levels = -1;  // levels built level by level; -1: no shared-memory pass
  hls.lb = 0;
  hls.le = R;
  hls.depth = 0;
  for (int round = 0; round < kMaxDepth; ++round) {
    if (host_max <= kDeepMax && level_nodes <= kDeepMaxRoots) {
      // every node of the current level fits one block: the rest of every subtree is
      // built in shared memory, then the host reads the final level state
      if (round == 0) {  // the roots' sums (every root has at most kBig points)
        k_root_moments<<<kGridBlocks, kThreads, 0, s>>>(w.nodes, R, w.B, w.ts0, w.mom);
        count_launch();
      }
      global_levels = hls.depth;
      rc = deep_pass(w, P, hls, s);
      if (rc) return rc;
      KDS_CK(cudaMemcpyAsync(&hls, w.ls, sizeof(LevelState), cudaMemcpyDeviceToHost, s));
      KDS_CK(cudaStreamSynchronize(s));
      if (hls.error == 2) { set_error("kds_tree_build: coordinate >= 32768 m, non-finite stamp or dt >= 65536 s"); return KDS_ERR_RANGE; }
      if (hls.error == 1) { set_error("kds_tree_build: node capacity exceeded"); return KDS_ERR_CAPACITY; }
      break;
    }
    // sync after every level once the subtree pass is within reach: the largest node within
    // a few halvings of kDeepMax and the level small enough (nodes at most double per level)
    const int nlev = (host_max <= 4 * kDeepMax && level_nodes * 4 <= kDeepMaxRoots) ? 1 : kLevelsPerSync;
    for (int k = 0; k < nlev; ++k) {
      const bool level0 = round == 0 && k == 0;
      const int64_t nodes_bound = level_nodes << k;
      const int lvl_blocks = (int)std::max<int64_t>(1, std::min<int64_t>(kLevelBlocks, (nodes_bound + kThreads - 1) / kThreads));
      const int small_blocks =
          (int)std::max<int64_t>(1, std::min<int64_t>(kSmallBlocks, (nodes_bound + kThreads / 32 - 1) / (kThreads / 32)));
      if (level0) {  // the roots' sums
        k_root_moments<<<kGridBlocks, kThreads, 0, s>>>(w.nodes, R, w.B, w.ts0, w.mom);
        count_launch();
        if (host_max > kBig) {
          k_big_sums<<<lvl_blocks, kThreads, 0, s>>>(w.nodes, w.ls, w.bbig);
          k_big_plan<<<lvl_blocks, kThreads, 0, s>>>(w.nodes, w.ls, w.bbig, w.chunks, w.chunk_cap, w.big_list,
                                                     w.node_chunk0, w.acc, w.accl);
          k_big_moments<<<cb, kThreads, 0, s>>>(w.chunks, w.ls, w.B, w.ts0, w.nodes, w.acc);
          k_big_to_mom<<<64, 256, 0, s>>>(w.ls, w.big_list, w.acc, w.mom);
          for (int c = 0; c < 4; ++c) count_launch();
        }
      }
      k_decide<<<lvl_blocks, kThreads, 0, s>>>(w.nodes, w.ls, w.mom, P, w.bsum, w.bbig, w.root_frame);
      k_level_children<<<lvl_blocks, kThreads, 0, s>>>(w.nodes, w.ls, w.bsum, (int32_t)w.cap_nodes);
      const bool big = host_max > kBig;  // the large-node kernels run after the partition
      k_small_part<<<small_blocks, kThreads, 0, s>>>(w.nodes, w.ls, w.B, w.ts0, w.mom, w.bsum, lvl_blocks,
                                                     w.level_begin, big ? nullptr : w.done);
      for (int c = 0; c < 3; ++c) count_launch();
      if (big) {
        if (!level0) {  // k_decide counted the large nodes per block
          k_big_plan<<<lvl_blocks, kThreads, 0, s>>>(w.nodes, w.ls, w.bbig, w.chunks, w.chunk_cap, w.big_list,
                                                     w.node_chunk0, w.acc, w.accl);
          count_launch();
        }
        k_big_count<<<cb, kThreads, 0, s>>>(w.chunks, w.ls, w.nodes, w.B, w.chunk_nl);
        k_big_offsets<<<kGridBlocks, kThreads, 0, s>>>(w.nodes, w.ls, w.big_list, w.node_chunk0, w.chunk_nl,
                                                       w.chunk_loff);
        k_big_scatter<<<cb, kThreads, 0, s>>>(w.chunks, w.ls, w.nodes, w.B, w.chunk_loff, w.ts0, w.accl);
        k_big_childmom<<<64, 256, 0, s>>>(w.nodes, w.ls, w.big_list, w.accl, w.mom, w.bsum, lvl_blocks,
                                          w.level_begin, w.done);
        for (int c = 0; c < 5; ++c) count_launch();
      }
    }
    KDS_CK(cudaGetLastError());
    KDS_CK(cudaMemcpyAsync(&hls, w.ls, sizeof(LevelState), cudaMemcpyDeviceToHost, s));
    KDS_CK(cudaStreamSynchronize(s));
    if (hls.error == 2) { set_error("kds_tree_build: coordinate >= 32768 m, non-finite stamp or dt >= 65536 s"); return KDS_ERR_RANGE; }
    if (hls.error == 1) { set_error("kds_tree_build: node capacity exceeded"); return KDS_ERR_CAPACITY; }
    if (hls.lb >= hls.le) break;
    host_max = hls.max_size;
    level_nodes = hls.le - hls.lb;
  }
  if (hls.lb < hls.le) { set_error("kds_tree_build: depth limit"); return KDS_ERR_CAPACITY; }
  const int depth = hls.depth;
  const int32_t total = hls.le;
  // prune
  KDS_CK(cudaMemsetAsync(w.alive, 0, sizeof(int32_t) * total, s));
  k_alive<<<(int)std::min<int64_t>(nblk(total, kThreads), kGridBlocks * 4), kThreads, 0, s>>>(w.nodes, total, w.alive,
                                                                                          P.prune_incidence);
  count_launch();
  const int64_t G = (int64_t)(kMaxDepth + 2) * R;
  KDS_CK(cudaMemsetAsync(w.cnt, 0, sizeof(int32_t) * G, s));
  KDS_CK(cudaMemsetAsync(w.lcnt, 0, sizeof(int32_t) * G, s));
  KDS_CK(cudaMemsetAsync(w.ucnt, 0, sizeof(int32_t) * G, s));
  k_group_counts<<<nblk(total, kThreads), kThreads, 0, s>>>(w.nodes, total, w.alive, R, w.cnt, w.lcnt, w.ucnt,
                                                            w.leaf_flag);
  count_launch();
  rc = scan_exclusive(w.alive, w.rank, total, w.tile_sums, w.scan_tot, s);
  if (rc) return rc;
  rc = scan_exclusive(w.leaf_flag, w.lrank, total, w.tile_sums, w.scan_tot, s);
  if (rc) return rc;
  k_group_tables<<<1, 1024, 0, s>>>(depth, R, w.cnt, w.lcnt, w.gp, w.lgp, w.to, w.lto, w.tot_nodes, w.tot_leaves);
  count_launch();
  KDS_CK(cudaMemcpyAsync(h_cnt, w.tot_nodes, sizeof(int32_t) * R, cudaMemcpyDeviceToHost, s));
  KDS_CK(cudaMemcpyAsync(h_cnt + R, w.tot_leaves, sizeof(int32_t) * R, cudaMemcpyDeviceToHost, s));
  KDS_CK(cudaMemcpyAsync(h_cnt + 2 * R, w.ucnt, sizeof(int32_t) * R, cudaMemcpyDeviceToHost, s));
  KDS_CK(cudaMemcpyAsync(h_dbl, w.ts0, sizeof(double) * R, cudaMemcpyDeviceToHost, s));
  KDS_CK(cudaMemcpyAsync(h_dbl + R, w.root_frame, sizeof(double) * kRootFrame * R, cudaMemcpyDeviceToHost, s));
  KDS_CK(cudaStreamSynchronize(s));
  const std::vector<int32_t> tn(h_cnt, h_cnt + R), tl(h_cnt + R, h_cnt + 2 * R), tu(h_cnt + 2 * R, h_cnt + 3 * R);
  const std::vector<double> ts0(h_dbl, h_dbl + R), rf(h_dbl + R, h_dbl + R + (size_t)kRootFrame * R);
  std::vector<TreeDev> td(R);
  std::vector<kds_tree*> made(R, nullptr);
  for (int r = 0; r < R; ++r) {
    int64_t np = off[r + 1] - off[r];
    if (np < prm->leaf_min_points || np == 0 || tl[r] < prm->tree_min_good_leaves) continue;
    kds_tree* t = new kds_tree();
    rc = tree_alloc(t->d, tn[r], tl[r], np, s);
    if (rc) {
      delete t;
      for (int q = 0; q < r; ++q)
        if (made[q]) { tree_release(made[q]->d); delete made[q]; }
      return rc;
    }
    t->d.num_unpruned = tu[r];
    t->d.ts_start = ts0[r];
    t->d.depth = depth;
    t->d.global_levels = global_levels >= 0 ? global_levels : depth;
    const double* f = &rf[(size_t)kRootFrame * r];
    for (int i = 0; i < 3; ++i) {
      t->root_eigenvalues[i] = (float)f[i];
      t->root_mean[i] = (float)f[12 + i];
    }
    for (int i = 0; i < 9; ++i) t->root_eigenvectors[i] = (float)f[3 + i];
    made[r] = t;
    td[r] = t->d;
  }
  KDS_CK(cudaMemcpyAsync(w.trees, td.data(), sizeof(TreeDev) * R, cudaMemcpyHostToDevice, s));
  k_compact_forest<<<nblk(total, kThreads), kThreads, 0, s>>>(w.nodes, total, w.alive, w.rank, w.leaf_flag, w.lrank,
                                                              R, w.gp, w.lgp, w.to, w.lto, w.trees);
  count_launch();
  dim3 fg((unsigned)std::min<int64_t>(nblk(max_size, kThreads), 256), (unsigned)R);
  k_finish_trees<<<fg, kThreads, 0, s>>>(w.trees, w.off, w.B.perm);
  count_launch();
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    for (auto* t : made)
      if (t) { tree_release(t->d); delete t; }
    return cuda_status(e, "tree build", __FILE__, __LINE__);
  }
  for (int r = 0; r < R; ++r) {
    out[r] = made[r];
    status[r] = made[r] ? KDS_OK : KDS_ERR_TREE_REJECTED;
  }
  return KDS_OK;
}

int tree_build(const float* xyz, const double* stamps, int64_t n, int32_t mem, const kds_tree_params* prm,
               cudaStream_t s, kds_tree** out) {
  *out = nullptr;
  if (n < 0 || n > ((int64_t)1 << 30)) {
    set_error("kds_tree_build: bad point count %lld", (long long)n);
    return KDS_ERR_INVALID_ARG;
  }
  if (n < prm->leaf_min_points || n == 0) {
    set_error("kds_tree_build: %lld points < leaf_min_points", (long long)n);
    return KDS_ERR_TREE_REJECTED;
  }
  int64_t off[2] = {0, n};
  int32_t st = 0;
  int rc = tree_build_forest(xyz, stamps, off, 1, mem, prm, s, out, &st);
  if (rc) return rc;
  if (st != KDS_OK) {
    set_error("kds_tree_build: too few good leaves (tree_min_good_leaves %d)", prm->tree_min_good_leaves);
    return KDS_ERR_TREE_REJECTED;
  }
  return KDS_OK;
}

}  // namespace kds
