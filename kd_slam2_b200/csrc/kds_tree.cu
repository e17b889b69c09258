// Surfel KD-tree utilities on the GPU: allocation, import/export, morph, rigid
// transform and leaf extraction.  The build itself is in kds_build.cu.  Compiled with
// -fmad=false so the morph and transform kernels round like the CPU oracle.
#include <cuda_runtime.h>

#include <cstddef>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "kds_internal.cuh"

namespace kds {

namespace {

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

__global__ void k_gather_leaves(TreeDev t) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= t.num_leaves) return;
  int o = t.leaf_idx[i];
  DNode d = t.nodes[o];
  t.leaf_md[i] = make_float4(d.a.x, d.a.y, d.a.z, t.dts_f[o]);
  t.leaf_nrm[i] = make_float4(d.a.w, d.b.x, d.b.y, 0.f);
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

static_assert(sizeof(kds_kdnode3f) == 56 && offsetof(kds_kdnode3f, idx_start) == 24 &&
                  offsetof(kds_kdnode3f, dts_mean) == 40 && offsetof(kds_kdnode3f, dts_covariance) == 48,
              "KDNode3f record layout");

// kd_slam2_msgs/msg/KDNode3f records -> device node arrays (the bag reader's per-node
// copy, lib/kd_io/rosbag2_message_reader.cpp:180-188), with the same checks as k_import.
__global__ void k_import_msg(TreeDev t, const kds_kdnode3f* rec, int32_t* bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= t.num_nodes) return;
  const kds_kdnode3f k = rec[i];
  const int l = k.idx_left, r = k.idx_right;
  if (l >= t.num_nodes || r >= t.num_nodes || (l >= 0 && l <= i) || (r >= 0 && r <= i)) *bad = 1;
  DNode d;
  d.a = make_float4(k.mean[0], k.mean[1], k.mean[2], k.direction[0]);
  d.b = make_float4(k.direction[1], k.direction[2], __int_as_float(l), __int_as_float(r));
  t.nodes[i] = d;
  t.dts_mean[i] = k.dts_mean;
  t.dts_f[i] = (float)k.dts_mean;
  t.dts_cov[i] = k.dts_covariance;
  t.range[2 * i] = (int64_t)k.idx_start;
  t.range[2 * i + 1] = (int64_t)k.idx_end;
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

template <class T> T* carve(char*& p, size_t count) {
  size_t bytes = (count * sizeof(T) + 255) & ~(size_t)255;
  T* r = reinterpret_cast<T*>(p);
  p += bytes;
  return r;
}
template <class T> size_t carve_size(size_t count) { return (count * sizeof(T) + 255) & ~(size_t)255; }

}  // namespace

// Exclusive scan of n int32 into out; *total receives the sum (device).
int scan_exclusive(const int32_t* in, int32_t* out, int32_t n, int32_t* tile_sums, int32_t* total,
                   cudaStream_t s) {
  int nt = nblk(n, kScanTile);
  k_scan_tiles<<<nt, kScanThreads, 0, s>>>(in, n, tile_sums); ::kds::count_launch();
  k_scan_top<<<1, kScanThreads, 0, s>>>(tile_sums, nt, total); ::kds::count_launch();
  k_scan_apply<<<nt, kScanThreads, 0, s>>>(in, n, tile_sums, out); ::kds::count_launch();
  KDS_CK(cudaGetLastError());
  return KDS_OK;
}

// ---------------------------------------------------------------------------
int tree_alloc(TreeDev& t, int64_t nodes, int64_t leaves, int64_t points, cudaStream_t s) {
  size_t bytes = carve_size<DNode>(nodes) + carve_size<float>(nodes) + 2 * carve_size<double>(nodes) +
                 carve_size<int64_t>(2 * nodes) + carve_size<int32_t>(nodes) + carve_size<int32_t>(leaves) +
                 2 * carve_size<float4>(leaves) + carve_size<int32_t>(points) + 256;
  void* blk = nullptr;
  cudaError_t e = cudaMallocAsync(&blk, bytes, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("cudaMalloc of %zu bytes for a tree failed: %s", bytes, cudaGetErrorString(e));
    return KDS_ERR_OOM;
  }
  char* p = (char*)blk;
  t.block = blk;
  t.stream = s;
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
  if (t.block) {
    // stream-ordered free on the stream the tree was made on; fall back to a plain
    // free if that stream is gone
    if (cudaFreeAsync(t.block, t.stream) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(t.block);
    }
  }
  t = TreeDev();
}

int tree_gather_leaves(TreeDev& t, cudaStream_t s) {
  if (t.num_leaves == 0) return KDS_OK;
  k_gather_leaves<<<nblk(t.num_leaves, 256), 256, 0, s>>>(t); ::kds::count_launch();
  KDS_CK(cudaGetLastError());
  return KDS_OK;
}

static int import_finish(kds_tree* t, int32_t* flag, int32_t* rank, int32_t* tiles, int32_t* dbad, void* stg,
                         cudaStream_t s, const char* who, kds_tree** out);

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
  int rc = tree_alloc(t->d, num_nodes, nleaves, 0, cudaStreamPerThread);
  if (rc) { delete t; return rc; }
  t->d.ts_start = ts_start;
  t->d.num_unpruned = num_nodes;
  cudaStream_t s = cudaStreamPerThread;
  // staging
  size_t nb = num_nodes;
  void* stg = nullptr;
  size_t bytes = nb * (3 * 4 * 2 + 8 * 2 + 8 * 2 + 4 * 2) + 64;
  // staging from the stream-ordered pool: no device-wide synchronisation on release
  cudaError_t ce = cudaMallocAsync(&stg, bytes, s);
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
                                                 s0 ? ds : nullptr, e0 ? de : nullptr, dl, dr, dbad); ::kds::count_launch();
  // leaf list by scan over leaf flags, reusing the staging arrays (dl as flag, dr as rank)
  int32_t* flag = (int32_t*)ds;  // ds/de no longer needed after k_import on this stream
  int32_t* rank = (int32_t*)de;
  return import_finish(t, flag, rank, dl, dbad, stg, s, "kds_tree_import", out);
}

// Leaf list of an imported tree (scan over leaf flags), the leaf arrays, and the result
// of the node checks; frees the staging block and hands the tree out (or releases it).
// flag, rank, tiles: num_nodes int32 scratch each; dbad[0] the check flag, dbad[1] scratch.
static int import_finish(kds_tree* t, int32_t* flag, int32_t* rank, int32_t* tiles, int32_t* dbad, void* stg,
                         cudaStream_t s, const char* who, kds_tree** out) {
  const int64_t num_nodes = t->d.num_nodes;
  int32_t* total = dbad + 1;
  k_leaf_flags_plain<<<nblk(num_nodes, 256), 256, 0, s>>>(t->d.nodes, (int32_t)num_nodes, flag); ::kds::count_launch();
  int rc2 = scan_exclusive(flag, rank, (int32_t)num_nodes, tiles, total, s);
  k_leaf_scatter_plain<<<nblk(num_nodes, 256), 256, 0, s>>>(flag, rank, (int32_t)num_nodes, t->d.leaf_idx); ::kds::count_launch();
  tree_gather_leaves(t->d, s);
  int32_t bad = 0;
  cudaMemcpyAsync(&bad, dbad, 4, cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(stg, s);
  cudaError_t ce = cudaStreamSynchronize(s);
  if (ce != cudaSuccess || rc2) {
    tree_release(t->d);
    delete t;
    return ce != cudaSuccess ? cuda_status(ce, "tree import", __FILE__, __LINE__) : rc2;
  }
  if (bad) {
    tree_release(t->d);
    delete t;
    set_error("%s: child index out of range or not after its parent (BFS order required)", who);
    return KDS_ERR_BAD_TREE;
  }
  *out = t;
  return KDS_OK;
}

int tree_from_msg(const kds_kdtree3f* msg, kds_tree** out) {
  *out = nullptr;
  const int64_t n = msg->num_nodes;
  if (n <= 0 || n > ((int64_t)1 << 30) || !msg->nodes) {
    set_error("kds_tree_from_msg: bad node array");
    return KDS_ERR_INVALID_ARG;
  }
  int64_t nleaves = 0;
  for (int64_t i = 0; i < n; ++i)
    if (msg->nodes[i].idx_left < 0 && msg->nodes[i].idx_right < 0) ++nleaves;
  kds_tree* t = new kds_tree();
  cudaStream_t s = cudaStreamPerThread;
  int rc = tree_alloc(t->d, n, nleaves, 0, s);
  if (rc) { delete t; return rc; }
  t->d.ts_start = msg->ts_start;
  t->d.num_unpruned = n;
  for (int i = 0; i < 3; ++i) {
    t->root_mean[i] = msg->root_mean[i];
    t->root_eigenvalues[i] = msg->root_eigenvalues[i];
  }
  for (int i = 0; i < 9; ++i) t->root_eigenvectors[i] = msg->root_eigenvectors[i];
  // staging: the raw records, then three int32 arrays and two flags
  void* stg = nullptr;
  const size_t rec_bytes = (((size_t)n * sizeof(kds_kdnode3f)) + 255) & ~(size_t)255;
  cudaError_t ce = cudaMallocAsync(&stg, rec_bytes + (size_t)n * 12 + 64, s);
  if (ce != cudaSuccess) {
    cudaGetLastError();
    tree_release(t->d);
    delete t;
    set_error("kds_tree_from_msg: staging OOM");
    return KDS_ERR_OOM;
  }
  kds_kdnode3f* drec = (kds_kdnode3f*)stg;
  int32_t* flag = (int32_t*)((char*)stg + rec_bytes);
  int32_t* rank = flag + n;
  int32_t* tiles = rank + n;
  int32_t* dbad = tiles + n;
  cudaMemcpyAsync(drec, msg->nodes, (size_t)n * sizeof(kds_kdnode3f), cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(dbad, 0, 4, s);
  k_import_msg<<<nblk(n, 256), 256, 0, s>>>(t->d, drec, dbad); ::kds::count_launch();
  return import_finish(t, flag, rank, tiles, dbad, stg, s, "kds_tree_from_msg", out);
}

int tree_apply_velocities(kds_tree* t, const float* v, int skip_leaves, cudaStream_t s) {
  if (t->d.num_nodes == 0) return KDS_OK;
  Vel6 vv;
  for (int i = 0; i < 6; ++i) vv.v[i] = v[i];
  k_apply_velocities<<<nblk(t->d.num_nodes, 256), 256, 0, s>>>(t->d, vv, skip_leaves); ::kds::count_launch();
  KDS_CK(cudaGetLastError());
  return tree_gather_leaves(t->d, s);
}

int tree_apply_isometry(kds_tree* t, const float* X, cudaStream_t s) {
  if (t->d.num_nodes == 0) return KDS_OK;
  Iso12 iso;
  for (int i = 0; i < 12; ++i) iso.m[i] = X[i];
  k_apply_isometry<<<nblk(t->d.num_nodes, 256), 256, 0, s>>>(t->d, iso); ::kds::count_launch();
  KDS_CK(cudaGetLastError());
  return tree_gather_leaves(t->d, s);
}

// Gathers [mean, dir] per leaf, optionally morphed by v6.  out_device: the caller's
// device buffer (no allocation, asynchronous on s); otherwise out_host through a
// stream-ordered temporary, returning when the host copy is complete.
int tree_extract_leaves(const kds_tree* t, const float* v6, float* out_host, float* out_device, cudaStream_t s) {
  if (t->d.num_leaves == 0) return KDS_OK;
  Vel6 vv;
  for (int i = 0; i < 6; ++i) vv.v[i] = v6 ? v6[i] : 0.f;
  float* d = out_device;
  if (!d) KDS_CK(cudaMallocAsync(&d, sizeof(float) * 6 * t->d.num_leaves, s));
  k_extract_leaves<<<nblk(t->d.num_leaves, 256), 256, 0, s>>>(t->d, vv, v6 ? 1 : 0, d); ::kds::count_launch();
  cudaError_t e = cudaGetLastError();
  if (out_device) return e == cudaSuccess ? KDS_OK : cuda_status(e, "extract leaves", __FILE__, __LINE__);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out_host, d, sizeof(float) * 6 * t->d.num_leaves, cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(d, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
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

namespace kds {

// Device-to-device copy of a whole tree into a new block allocated on stream s: every
// node and leaf array, the point permutation and the host-side fields.  The arrays are
// copied one by one because the two blocks may carve at different base alignments.
int tree_clone(const kds_tree* src, cudaStream_t s, kds_tree** out) {
  *out = nullptr;
  const TreeDev& a = src->d;
  kds_tree* t = new kds_tree();
  int rc = tree_alloc(t->d, a.num_nodes, a.num_leaves, a.num_points, s);
  if (rc != KDS_OK) {
    delete t;
    return rc;
  }
  TreeDev& b = t->d;
  const int64_t nn = a.num_nodes, nl = a.num_leaves, np = a.num_points;
  cudaError_t e = cudaSuccess;
  auto cp = [&](void* dst, const void* from, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(dst, from, bytes, cudaMemcpyDeviceToDevice, s);
  };
  cp(b.nodes, a.nodes, sizeof(DNode) * nn);
  cp(b.dts_f, a.dts_f, sizeof(float) * nn);
  cp(b.dts_mean, a.dts_mean, sizeof(double) * nn);
  cp(b.dts_cov, a.dts_cov, sizeof(double) * nn);
  cp(b.range, a.range, sizeof(int64_t) * 2 * nn);
  cp(b.level, a.level, sizeof(int32_t) * nn);
  cp(b.leaf_idx, a.leaf_idx, sizeof(int32_t) * nl);
  cp(b.leaf_md, a.leaf_md, sizeof(float4) * nl);
  cp(b.leaf_nrm, a.leaf_nrm, sizeof(float4) * nl);
  if (a.perm && b.perm) cp(b.perm, a.perm, sizeof(int32_t) * np);
  if (e != cudaSuccess) {
    cudaGetLastError();
    tree_release(t->d);
    delete t;
    return cuda_status(e, "tree_clone copies", __FILE__, __LINE__);
  }
  b.num_unpruned = a.num_unpruned;
  b.ts_start = a.ts_start;
  b.depth = a.depth;
  b.accepted = a.accepted;
  for (int i = 0; i < 3; ++i) {
    t->root_mean[i] = src->root_mean[i];
    t->root_eigenvalues[i] = src->root_eigenvalues[i];
  }
  for (int i = 0; i < 9; ++i) t->root_eigenvectors[i] = src->root_eigenvectors[i];
  *out = t;
  return KDS_OK;
}

}  // namespace kds
