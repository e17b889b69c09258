// Raw scan -> tree-build input on the device: toPointsVector's stamps
// (lib/kd_io/scan_utils_impl_.h:9-33) and Voxelizer_::voxelize
// (kd/utils/voxelizer_impl_.h:111-145, with add() :68-109 and the Accumulator :11-58).
//
// The reference bins points in a hash map and emits the voxels in the map's iteration
// order (implementation-defined).  Here the voxels come out sorted by their integer
// index (x, y, z, t) -- a canonical order; trees built from the two agree node for node,
// only the point permutation differs.  Within a voxel the points are summed in input
// order in float (stamps in double), as the Accumulator adds them, so each voxel mean is
// the reference's bit for bit: a stable sort of (voxel, input index) followed by one
// thread per voxel.  The sort is CUB's radix sort (two stable 64-bit passes).
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "kds_internal.cuh"

namespace kds {

namespace {

constexpr unsigned long long kInvalidKey = ~0ull;

// order-preserving map of doubles to unsigned keys (for the stamps' minimum)
__device__ __forceinline__ unsigned long long dkey_of(double d) {
  unsigned long long b = (unsigned long long)__double_as_longlong(d);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double d_of_key(unsigned long long k) {
  unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

struct VoxArgs {
  const float* xyz;
  const double* st;     // per-point stamps or NULL
  int64_t n;
  double msg_t;
  double scan_duration;
  float inv_space;      // Scalar(1) / space_res
  float inv_time;       // Scalar(1) / time_res, or 0
  float lo2, hi2;       // float bounds of add(): pow(max(0, range_min - b), 2), pow(range_max + b, 2)
  double rmin2, rmax2;  // double bounds of voxelize(): pow(range_min, 2), pow(range_max, 2)
};

// Eigen's squaredNorm of a 3-vector: (x*x + y*y) + z*z
__device__ __forceinline__ float sq_norm(float x, float y, float z) {
  return __fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z));
}

// toPointsVector's stamp of point i
__device__ __forceinline__ double stamp_of(const VoxArgs& a, int64_t i) {
  if (a.st) return a.st[i];
  if (a.scan_duration > 0.0) {
    const double alpha = atan2((double)a.xyz[3 * i + 1], (double)a.xyz[3 * i]);
    return a.msg_t + (alpha + M_PI) / (2.0 * M_PI) * a.scan_duration;
  }
  return a.msg_t;
}

__global__ void k_stamps_min(VoxArgs a, double* stamps, unsigned long long* tmin) {
  unsigned long long m = ~0ull;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
    const double t = stamp_of(a, i);
    stamps[i] = t;
    m = min(m, dkey_of(t));
  }
  for (int off = 16; off > 0; off >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) atomicMin(tmin, m);
}

// (int) of a scaled coordinate: truncation, held inside +-2^30, biased to sort as unsigned
__device__ __forceinline__ unsigned cell_of(float v) {
  const float c = fminf(fmaxf(v, -1073741824.f), 1073741824.f);
  return (unsigned)__float2int_rz(c) ^ 0x80000000u;
}

// voxel key halves of every point (invalid: outside add()'s bounds)
__global__ void k_vox_keys(VoxArgs a, const double* stamps, const unsigned long long* tmin,
                           unsigned long long* khi, unsigned long long* klo, int32_t* idx) {
  const double t0 = d_of_key(*tmin);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
    const float x = a.xyz[3 * i], y = a.xyz[3 * i + 1], z = a.xyz[3 * i + 2];
    const float n2 = sq_norm(x, y, z);
    idx[i] = (int32_t)i;
    if (n2 > a.hi2 || n2 < a.lo2 || !(n2 == n2)) {
      khi[i] = kInvalidKey;
      klo[i] = kInvalidKey;
      continue;
    }
    const unsigned ix = cell_of(__fmul_rn(x, a.inv_space)), iy = cell_of(__fmul_rn(y, a.inv_space));
    const unsigned iz = cell_of(__fmul_rn(z, a.inv_space));
    unsigned it = 0x80000000u;
    if (a.inv_time > 0.f) {
      const double ts = __dmul_rn(stamps[i] - t0, (double)a.inv_time);
      it = (unsigned)__double2int_rz(fmin(fmax(ts, -1073741824.0), 1073741824.0)) ^ 0x80000000u;
    }
    khi[i] = ((unsigned long long)ix << 32) | iy;
    klo[i] = ((unsigned long long)iz << 32) | it;
  }
}

__global__ void k_gather_u64(const unsigned long long* src, const int32_t* idx, int64_t n, unsigned long long* dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[idx[i]];
}

// 1 where a sorted entry starts a new voxel (valid entries only)
__global__ void k_vox_heads(const unsigned long long* khi, const unsigned long long* klo, int64_t n, int32_t* head) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const bool valid = khi[i] != kInvalidKey || klo[i] != kInvalidKey;
    head[i] = valid && (i == 0 || khi[i] != khi[i - 1] || klo[i] != klo[i - 1]) ? 1 : 0;
  }
}

// voxel v starts at sorted position start[v]
__global__ void k_vox_starts(const int32_t* head, const int32_t* vid, int64_t n, int32_t* start) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (head[i]) start[vid[i]] = (int32_t)i;
}

// Accumulator::add in input order, normalize(), and voxelize()'s range test of the mean
__global__ void k_vox_means(VoxArgs a, const double* stamps, const unsigned long long* khi,
                            const unsigned long long* klo, const int32_t* order, const int32_t* start,
                            const int32_t* nvox_p, int64_t n, float4* mean, double* mst, int32_t* keep) {
  const int32_t nvox = *nvox_p;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += gridDim.x * blockDim.x) {
    const int32_t b = start[v];
    float sx = 0.f, sy = 0.f, sz = 0.f;
    double ss = 0.0;
    int cnt = 0;
    for (int64_t k = b; k < n && (k == b || (khi[k] == khi[b] && klo[k] == klo[b])); ++k) {
      const int32_t i = order[k];
      sx = __fadd_rn(sx, a.xyz[3 * i]);
      sy = __fadd_rn(sy, a.xyz[3 * i + 1]);
      sz = __fadd_rn(sz, a.xyz[3 * i + 2]);
      ss = __dadd_rn(ss, stamps[i]);
      ++cnt;
    }
    const float inv = __fdiv_rn(1.f, (float)cnt);
    const float mx = __fmul_rn(sx, inv), my = __fmul_rn(sy, inv), mz = __fmul_rn(sz, inv);
    mean[v] = make_float4(mx, my, mz, 0.f);
    mst[v] = __dmul_rn(ss, (double)inv);
    const double n2 = (double)sq_norm(mx, my, mz);
    keep[v] = (n2 > a.rmax2 || n2 < a.rmin2) ? 0 : 1;
  }
}

// no voxel grid: the points inside [range_min, range_max], in input order
__global__ void k_range_keep(VoxArgs a, int32_t* keep) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
    const double n2 = (double)sq_norm(a.xyz[3 * i], a.xyz[3 * i + 1], a.xyz[3 * i + 2]);
    keep[i] = (n2 < a.rmin2 || n2 > a.rmax2) ? 0 : 1;
  }
}

__global__ void k_scatter_points(const float* xyz, const double* st, const int32_t* keep, const int32_t* pos,
                                 int64_t n, float* oxyz, double* ost) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (!keep[i]) continue;
    const int32_t o = pos[i];
    oxyz[3 * o] = xyz[3 * i];
    oxyz[3 * o + 1] = xyz[3 * i + 1];
    oxyz[3 * o + 2] = xyz[3 * i + 2];
    if (ost) ost[o] = st[i];
  }
}

__global__ void k_scatter_voxels(const float4* mean, const double* mst, const int32_t* keep, const int32_t* pos,
                                 const int32_t* nvox_p, float* oxyz, double* ost) {
  const int32_t nvox = *nvox_p;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += gridDim.x * blockDim.x) {
    if (!keep[v]) continue;
    const int32_t o = pos[v];
    oxyz[3 * o] = mean[v].x;
    oxyz[3 * o + 1] = mean[v].y;
    oxyz[3 * o + 2] = mean[v].z;
    if (ost) ost[o] = mst[v];
  }
}

// kept voxels: the exclusive scan of the keep flags at nvox
__global__ void k_voxel_count(const int32_t* pos, const int32_t* nvox, int32_t* nout) { *nout = pos[*nvox]; }

inline int grid_for(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 8); }

}  // namespace

int points_voxelize(const float* xyz, const double* stamps, int64_t n, int32_t mem, double msg_t,
                    double scan_duration, const kds_voxel_params* prm, cudaStream_t s, float* out_xyz,
                    double* out_stamps, int64_t* out_n) {
  if (!out_n || n < 0 || n > ((int64_t)1 << 30) || (n > 0 && (!xyz || !out_xyz)) || !prm) {
    set_error("kds_points_voxelize: bad arguments");
    return KDS_ERR_INVALID_ARG;
  }
  *out_n = 0;
  if (n == 0) return KDS_OK;
  const bool host = mem == KDS_MEM_HOST;
  const bool vox = prm->space_res > 0.f;
  VoxArgs a;
  a.n = n;
  a.msg_t = msg_t;
  a.scan_duration = scan_duration;
  a.inv_space = vox ? 1.f / prm->space_res : 0.f;
  a.inv_time = prm->time_res > 0.f ? 1.f / prm->time_res : 0.f;
  const float b = prm->use_boundary ? (float)std::sqrt((double)(prm->space_res * 3)) : 0.f;
  a.hi2 = (float)std::pow(prm->range_max + b, 2);
  a.lo2 = (float)std::pow(std::max(0.f, prm->range_min - b), 2);
  a.rmin2 = std::pow(prm->range_min, 2);
  a.rmax2 = std::pow(prm->range_max, 2);

  size_t cub_sort = 0, cub_scan = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, cub_sort, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                  (int32_t*)nullptr, (int32_t*)nullptr, (int)n, 0, 64, s);
  cub::DeviceScan::ExclusiveSum(nullptr, cub_scan, (int32_t*)nullptr, (int32_t*)nullptr, (int)n + 1, s);
  // one device block: inputs and outputs (host case), stamps, keys, sort buffers, scans
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t N = (size_t)n;
  const size_t bytes = (host ? al(12 * N) + al(8 * N) + al(12 * N) + al(8 * N) : 0) + al(8 * N) + 4 * al(8 * N) +
                       2 * al(4 * N) + 3 * al(4 * (N + 1)) + al(16 * N) + al(8 * N) + al(std::max(cub_sort, cub_scan)) +
                       al(64);
  void* blk = nullptr;
  cudaError_t e = cudaMallocAsync(&blk, bytes, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("kds_points_voxelize: device memory (%zu bytes): %s", bytes, cudaGetErrorString(e));
    return KDS_ERR_OOM;
  }
  char* p = (char*)blk;
  auto take = [&](size_t x) { char* r = p; p += al(x); return (void*)r; };
  const float* d_xyz = xyz;
  const double* d_st = stamps;
  float* d_oxyz = out_xyz;
  double* d_ost = out_stamps;
  if (host) {
    d_xyz = (const float*)take(12 * N);
    d_st = stamps ? (const double*)take(8 * N) : nullptr;
    d_oxyz = (float*)take(12 * N);
    d_ost = out_stamps ? (double*)take(8 * N) : nullptr;
  }
  double* d_stamp = (double*)take(8 * N);
  unsigned long long* khi = (unsigned long long*)take(8 * N);
  unsigned long long* klo = (unsigned long long*)take(8 * N);
  unsigned long long* khi2 = (unsigned long long*)take(8 * N);
  unsigned long long* klo2 = (unsigned long long*)take(8 * N);
  int32_t* idx = (int32_t*)take(4 * N);
  int32_t* idx2 = (int32_t*)take(4 * N);
  int32_t* flag = (int32_t*)take(4 * (N + 1));
  int32_t* pos = (int32_t*)take(4 * (N + 1));
  int32_t* start = (int32_t*)take(4 * (N + 1));
  float4* vmean = (float4*)take(16 * N);
  double* vst = (double*)take(8 * N);
  void* cub_tmp = take(std::max(cub_sort, cub_scan));
  unsigned long long* tmin = (unsigned long long*)take(64);
  int32_t* nvox = (int32_t*)(tmin + 1);
  int32_t* nout = nvox + 1;
  int32_t h_nout = 0;
  const int g = grid_for(n);
  do {
    if (host) {
      if ((e = cudaMemcpyAsync((void*)d_xyz, xyz, 12 * N, cudaMemcpyHostToDevice, s))) break;
      if (stamps && (e = cudaMemcpyAsync((void*)d_st, stamps, 8 * N, cudaMemcpyHostToDevice, s))) break;
    }
    a.xyz = d_xyz;
    a.st = d_st;
    if ((e = cudaMemsetAsync(tmin, 0xff, 8, s))) break;
    k_stamps_min<<<g, 256, 0, s>>>(a, d_stamp, tmin);
    count_launch();
    a.st = d_stamp;  // from here on the stamps are toPointsVector's
    if (!vox) {
      k_range_keep<<<g, 256, 0, s>>>(a, flag);
      count_launch();
      if ((e = cudaMemsetAsync(flag + n, 0, 4, s))) break;
      if ((e = cub::DeviceScan::ExclusiveSum(cub_tmp, cub_scan, flag, pos, (int)n + 1, s))) break;
      k_scatter_points<<<g, 256, 0, s>>>(d_xyz, d_stamp, flag, pos, n, d_oxyz, d_ost);
      count_launch();
      if ((e = cudaMemcpyAsync(&h_nout, pos + n, 4, cudaMemcpyDeviceToHost, s))) break;
    } else {
      k_vox_keys<<<g, 256, 0, s>>>(a, d_stamp, tmin, khi, klo, idx);
      count_launch();
      // LSD: stable by the low half (z, t), then stable by the high half (x, y)
      size_t ts = cub_sort;
      if ((e = cub::DeviceRadixSort::SortPairs(cub_tmp, ts, klo, klo2, idx, idx2, (int)n, 0, 64, s))) break;
      k_gather_u64<<<g, 256, 0, s>>>(khi, idx2, n, khi2);
      count_launch();
      ts = cub_sort;
      if ((e = cub::DeviceRadixSort::SortPairs(cub_tmp, ts, khi2, khi, idx2, idx, (int)n, 0, 64, s))) break;
      k_gather_u64<<<g, 256, 0, s>>>(klo, idx, n, klo2);  // the low halves in the final order
      count_launch();
      k_vox_heads<<<g, 256, 0, s>>>(khi, klo2, n, flag);
      count_launch();
      if ((e = cudaMemsetAsync(flag + n, 0, 4, s))) break;
      if ((e = cub::DeviceScan::ExclusiveSum(cub_tmp, cub_scan, flag, pos, (int)n + 1, s))) break;
      k_vox_starts<<<g, 256, 0, s>>>(flag, pos, n, start);
      count_launch();
      if ((e = cudaMemcpyAsync(nvox, pos + n, 4, cudaMemcpyDeviceToDevice, s))) break;
      k_vox_means<<<g, 256, 0, s>>>(a, d_stamp, khi, klo2, idx, start, nvox, n, vmean, vst, flag);
      count_launch();
      // keep flags in flag[0, nvox); the scan runs over n + 1 entries, and only
      // positions below nvox are read (entries past nvox hold stale heads)
      if ((e = cub::DeviceScan::ExclusiveSum(cub_tmp, cub_scan, flag, pos, (int)n + 1, s))) break;
      k_scatter_voxels<<<g, 256, 0, s>>>(vmean, vst, flag, pos, nvox, d_oxyz, d_ost);
      count_launch();
      k_voxel_count<<<1, 1, 0, s>>>(pos, nvox, nout);
      count_launch();
      if ((e = cudaMemcpyAsync(&h_nout, nout, 4, cudaMemcpyDeviceToHost, s))) break;
    }
    if ((e = cudaGetLastError())) break;
    if ((e = cudaStreamSynchronize(s))) break;
    if (host && h_nout > 0) {
      if ((e = cudaMemcpyAsync(out_xyz, d_oxyz, 12 * (size_t)h_nout, cudaMemcpyDeviceToHost, s))) break;
      if (out_stamps && (e = cudaMemcpyAsync(out_stamps, d_ost, 8 * (size_t)h_nout, cudaMemcpyDeviceToHost, s))) break;
      if ((e = cudaStreamSynchronize(s))) break;
    }
  } while (false);
  cudaFreeAsync(blk, s);
  if (e != cudaSuccess) {
    const int rc = cuda_status(e, "kds_points_voxelize", __FILE__, __LINE__);
    cudaGetLastError();
    return rc;
  }
  *out_n = h_nout;
  return KDS_OK;
}

}  // namespace kds
