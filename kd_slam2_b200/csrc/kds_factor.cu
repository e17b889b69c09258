// Multi-view bundle-adjustment factor assembly on the device: the block updates that
// MultiViewICPFactor_::compute and MultiViewCTICPFactor_::compute make with each pair's
// H, b (kd/map/multiview_icp_factor_impl_.h:30-62, multiview_cticp_factor_impl_.h:33-83),
// applied to every job of a batch at once, straight from the batch's device outputs.
//
// The host lays out the structure only: each factor-local block (r, c), r <= c, goes to
// the global block (var[r], var[c]), stored as the upper triangle (row variable <= column
// variable, the transpose where the factor's order is the other way round).  The
// contributions of every global block (and of every variable's b) are listed in factor
// order, so the device sums them in FP64 in a fixed order: the result does not depend
// on scheduling.  A factor counts when inlierRatio() > disable_inlier_ratio
// (kd/icp/icp_stats_.h:28-31, evaluated in float as there); this is decided on the device
// from the job's statistics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "kds_align.cuh"
#include "kds_internal.cuh"

namespace kds {

namespace {

// 6x6 sources inside a job's outputs
enum Src : int32_t {
  kH00 = 0,   // H[0:6, 0:6] (ICP: all of H; CT: H_pp)
  kH01 = 1,   // CT H[0:6, 6:12] = H_pv
  kH11 = 2,   // CT H[6:12, 6:12] = H_vv
  kHvB = 3,   // H_dual_vel_B
  kHpvB = 4,  // H_dual_cross_pose_vel_B
  kHvAB = 5,  // H_dual_cross_vel_AB
};
// 6-vectors
enum SrcB : int32_t { kB0 = 0, kB1 = 1, kBvB = 2 };

struct Contrib {
  int32_t job;
  int32_t src;
  int32_t sign;       // +1 / -1
  int32_t transpose;  // 1: add the source transposed
};

__device__ __forceinline__ double src_entry(const JobOut& o, int D, int src, int r, int c) {
  switch (src) {
    case kH00: return o.H[r * D + c];
    case kH01: return o.H[r * D + 6 + c];
    case kH11: return o.H[(6 + r) * D + 6 + c];
    case kHvB: return o.H_vel_B[r * 6 + c];
    case kHpvB: return o.H_cross_pose_vel_B[r * 6 + c];
    default: return o.H_cross_vel_AB[r * 6 + c];
  }
}

// enabled[f] = inlierRatio() > ratio, in float as ICPStats_ computes it
__global__ void k_factor_enabled(const JobOut* outs, const int32_t* fjob, int32_t nf, float ratio,
                                 int32_t* enabled) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const kds_stats& st = outs[fjob[f]].stats;
  const int leaves = st.num_inliers + st.num_outliers + st.num_bad + st.num_err_normal + st.num_err_fn;
  const float r = leaves ? (float)st.num_inliers / (float)leaves : 0.f;
  enabled[f] = r > ratio ? 1 : 0;
}

// thread per (global block, entry): its contributions in factor order, FP64
__global__ void k_factor_blocks(const JobOut* outs, const int32_t* jdim, const Contrib* con, const int32_t* cbeg,
                                const int32_t* cfac, const int32_t* enabled, int32_t nblocks, double* H) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nblocks * 36) return;
  const int blk = t / 36, e = t % 36, r = e / 6, c = e % 6;
  double acc = 0.0;
  for (int k = cbeg[blk]; k < cbeg[blk + 1]; ++k) {
    if (!enabled[cfac[k]]) continue;
    const Contrib q = con[k];
    const JobOut& o = outs[q.job];
    const double v = q.transpose ? src_entry(o, jdim[q.job], q.src, c, r) : src_entry(o, jdim[q.job], q.src, r, c);
    acc = q.sign > 0 ? acc + v : acc - v;
  }
  H[t] = acc;
}

// thread per (variable, entry)
__global__ void k_factor_b(const JobOut* outs, const Contrib* con, const int32_t* cbeg, const int32_t* cfac,
                           const int32_t* enabled, int32_t nvars, double* b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nvars * 6) return;
  const int var = t / 6, e = t % 6;
  double acc = 0.0;
  for (int k = cbeg[var]; k < cbeg[var + 1]; ++k) {
    if (!enabled[cfac[k]]) continue;
    const Contrib q = con[k];
    const JobOut& o = outs[q.job];
    const double v = q.src == kB0 ? o.b[e] : (q.src == kB1 ? o.b[6 + e] : o.b_vel_B[e]);
    acc = q.sign > 0 ? acc + v : acc - v;
  }
  b[t] = acc;
}

struct HEntry {
  int32_t gr, gc;  // global block (row variable <= column variable)
  int32_t factor;
  int32_t seq;     // order inside the factor
  Contrib c;
};

}  // namespace

int batch_assemble(Runner& R, const kds_factor* F, int32_t nf, int32_t nvars, float ratio, cudaStream_t s,
                   int32_t* num_blocks, int32_t* block_rc, double* H_out, double* b_out, int32_t* enabled_out) {
  if (nf < 0 || nvars <= 0 || (nf > 0 && !F) || !num_blocks) {
    set_error("kds_batch_assemble: bad arguments");
    return KDS_ERR_INVALID_ARG;
  }
  std::vector<HEntry> hs;
  std::vector<std::pair<int32_t, HEntry>> bs;  // (variable, contribution)
  std::vector<int32_t> fjob(nf), jdim(R.num_jobs, 6);
  for (int j = 0; j < R.num_jobs; ++j) jdim[j] = R.h_jobs[j].kind == 0 ? 6 : 12;
  for (int f = 0; f < nf; ++f) {
    const kds_factor& q = F[f];
    if (q.job < 0 || q.job >= R.num_jobs) {
      set_error("kds_batch_assemble: factor %d names job %d of %d", f, q.job, R.num_jobs);
      return KDS_ERR_INVALID_ARG;
    }
    const int kind = R.h_jobs[q.job].kind;
    const int nv = kind == 0 ? 2 : 4;
    if (kind == 1) {
      set_error("kds_batch_assemble: factor %d: a CT-ICP factor needs a KDS_JOB_LINEARIZE_DUAL job", f);
      return KDS_ERR_INVALID_ARG;
    }
    for (int k = 0; k < nv; ++k)
      if (q.var[k] < 0 || q.var[k] >= nvars) {
        set_error("kds_batch_assemble: factor %d: variable %d out of range", f, q.var[k]);
        return KDS_ERR_INVALID_ARG;
      }
    fjob[f] = q.job;
    int seq = 0;
    auto addH = [&](int r, int c, int src, int sign, int tr) {
      int gr = q.var[r], gc = q.var[c];
      if (gr > gc) { std::swap(gr, gc); tr ^= 1; }
      hs.push_back({gr, gc, f, seq++, {q.job, src, sign, tr}});
      if (gr == gc && r != c)  // both variables of an off-diagonal block are one: its transpose lands here too
        hs.push_back({gr, gc, f, seq++, {q.job, src, sign, tr ^ 1}});
    };
    auto addB = [&](int r, int src, int sign) { bs.push_back({q.var[r], {0, 0, f, seq++, {q.job, src, sign, 0}}}); };
    if (kind == 0) {  // ICP: x0 fixed pose, x1 moving pose (multiview_icp_factor_impl_.h:46-61)
      addH(0, 0, kH00, +1, 0);
      addH(0, 1, kH00, -1, 0);
      addH(1, 1, kH00, +1, 0);
      addB(0, kB0, +1);
      addB(1, kB0, -1);
    } else {  // CT dual: x0 pose_A, v0 vel_A, x1 pose_B, v1 vel_B (multiview_cticp_factor_impl_.h:62-83)
      addH(0, 0, kH00, +1, 0);
      addH(0, 1, kHpvB, -1, 0);
      addH(0, 2, kH00, -1, 0);
      addH(0, 3, kH01, -1, 0);
      addH(1, 1, kHvB, +1, 0);
      addH(1, 2, kHpvB, +1, 1);
      addH(1, 3, kHvAB, +1, 1);
      addH(2, 2, kH00, +1, 0);
      addH(2, 3, kH01, +1, 0);
      addH(3, 3, kH11, +1, 0);
      addB(0, kB0, +1);
      addB(1, kBvB, -1);
      addB(2, kB0, -1);
      addB(3, kB1, -1);
    }
  }
  std::stable_sort(hs.begin(), hs.end(), [](const HEntry& a, const HEntry& b) {
    return a.gr != b.gr ? a.gr < b.gr : a.gc < b.gc;  // factor order kept within a block
  });
  std::stable_sort(bs.begin(), bs.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  std::vector<int32_t> hbeg, rc, hfac, bbeg(nvars + 1, 0), bfac;
  std::vector<Contrib> hcon, bcon;
  for (size_t k = 0; k < hs.size(); ++k) {
    if (k == 0 || hs[k].gr != hs[k - 1].gr || hs[k].gc != hs[k - 1].gc) {
      hbeg.push_back((int32_t)k);
      rc.push_back(hs[k].gr);
      rc.push_back(hs[k].gc);
    }
    hcon.push_back(hs[k].c);
    hfac.push_back(hs[k].factor);
  }
  const int32_t nb = (int32_t)rc.size() / 2;
  hbeg.push_back((int32_t)hs.size());
  for (auto& e : bs) {
    ++bbeg[e.first + 1];
    bcon.push_back(e.second.c);
    bfac.push_back(e.second.factor);
  }
  for (int v = 0; v < nvars; ++v) bbeg[v + 1] += bbeg[v];
  const int32_t cap = *num_blocks;
  *num_blocks = nb;
  if (cap < nb || (nb > 0 && (!block_rc || !H_out))) {
    if (cap == 0 && !block_rc && !H_out) return KDS_OK;  // count query
    set_error("kds_batch_assemble: %d blocks do not fit in %d", nb, cap);
    return KDS_ERR_CAPACITY;
  }
  if (!rc.empty()) memcpy(block_rc, rc.data(), sizeof(int32_t) * rc.size());
  // device buffers: one block from the stream-ordered pool
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t sz_fjob = al(sizeof(int32_t) * std::max(nf, 1)), sz_en = sz_fjob;
  const size_t sz_jdim = al(sizeof(int32_t) * std::max(R.num_jobs, 1));
  const size_t sz_hcon = al(sizeof(Contrib) * std::max<size_t>(hcon.size(), 1));
  const size_t sz_hbeg = al(sizeof(int32_t) * hbeg.size()), sz_hfac = al(sizeof(int32_t) * std::max<size_t>(hfac.size(), 1));
  const size_t sz_bcon = al(sizeof(Contrib) * std::max<size_t>(bcon.size(), 1));
  const size_t sz_bbeg = al(sizeof(int32_t) * bbeg.size()), sz_bfac = al(sizeof(int32_t) * std::max<size_t>(bfac.size(), 1));
  const size_t sz_H = al(sizeof(double) * 36 * std::max(nb, 1)), sz_b = al(sizeof(double) * 6 * nvars);
  const size_t total = sz_fjob + sz_en + sz_jdim + sz_hcon + sz_hbeg + sz_hfac + sz_bcon + sz_bbeg + sz_bfac + sz_H + sz_b;
  void* blk = nullptr;
  cudaError_t e = cudaMallocAsync(&blk, total, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("kds_batch_assemble: device memory (%zu bytes): %s", total, cudaGetErrorString(e));
    return KDS_ERR_OOM;
  }
  char* p = (char*)blk;
  auto take = [&](size_t n) { char* r = p; p += n; return (void*)r; };
  int32_t* d_fjob = (int32_t*)take(sz_fjob);
  int32_t* d_en = (int32_t*)take(sz_en);
  int32_t* d_jdim = (int32_t*)take(sz_jdim);
  Contrib* d_hcon = (Contrib*)take(sz_hcon);
  int32_t* d_hbeg = (int32_t*)take(sz_hbeg);
  int32_t* d_hfac = (int32_t*)take(sz_hfac);
  Contrib* d_bcon = (Contrib*)take(sz_bcon);
  int32_t* d_bbeg = (int32_t*)take(sz_bbeg);
  int32_t* d_bfac = (int32_t*)take(sz_bfac);
  double* d_H = (double*)take(sz_H);
  double* d_b = (double*)take(sz_b);
  std::vector<int32_t> en(std::max(nf, 1), 0);
  do {
    if (nf > 0 && (e = cudaMemcpyAsync(d_fjob, fjob.data(), sizeof(int32_t) * nf, cudaMemcpyHostToDevice, s))) break;
    if ((e = cudaMemcpyAsync(d_jdim, jdim.data(), sizeof(int32_t) * R.num_jobs, cudaMemcpyHostToDevice, s))) break;
    if (!hcon.empty()) {
      if ((e = cudaMemcpyAsync(d_hcon, hcon.data(), sizeof(Contrib) * hcon.size(), cudaMemcpyHostToDevice, s))) break;
      if ((e = cudaMemcpyAsync(d_hfac, hfac.data(), sizeof(int32_t) * hfac.size(), cudaMemcpyHostToDevice, s))) break;
    }
    if ((e = cudaMemcpyAsync(d_hbeg, hbeg.data(), sizeof(int32_t) * hbeg.size(), cudaMemcpyHostToDevice, s))) break;
    if (!bcon.empty()) {
      if ((e = cudaMemcpyAsync(d_bcon, bcon.data(), sizeof(Contrib) * bcon.size(), cudaMemcpyHostToDevice, s))) break;
      if ((e = cudaMemcpyAsync(d_bfac, bfac.data(), sizeof(int32_t) * bfac.size(), cudaMemcpyHostToDevice, s))) break;
    }
    if ((e = cudaMemcpyAsync(d_bbeg, bbeg.data(), sizeof(int32_t) * bbeg.size(), cudaMemcpyHostToDevice, s))) break;
    if (nf > 0) {
      k_factor_enabled<<<(nf + 255) / 256, 256, 0, s>>>(R.d_outs, d_fjob, nf, ratio, d_en);
      count_launch();
    }
    if (nb > 0) {
      k_factor_blocks<<<(nb * 36 + 255) / 256, 256, 0, s>>>(R.d_outs, d_jdim, d_hcon, d_hbeg, d_hfac, d_en, nb, d_H);
      count_launch();
    }
    k_factor_b<<<(nvars * 6 + 255) / 256, 256, 0, s>>>(R.d_outs, d_bcon, d_bbeg, d_bfac, d_en, nvars, d_b);
    count_launch();
    if ((e = cudaGetLastError())) break;
    if (nb > 0 && (e = cudaMemcpyAsync(H_out, d_H, sizeof(double) * 36 * nb, cudaMemcpyDeviceToHost, s))) break;
    if (b_out && (e = cudaMemcpyAsync(b_out, d_b, sizeof(double) * 6 * nvars, cudaMemcpyDeviceToHost, s))) break;
    if (nf > 0 && (e = cudaMemcpyAsync(en.data(), d_en, sizeof(int32_t) * nf, cudaMemcpyDeviceToHost, s))) break;
    e = cudaStreamSynchronize(s);
  } while (false);
  cudaFreeAsync(blk, s);
  if (e != cudaSuccess) {
    const int rc2 = cuda_status(e, "kds_batch_assemble", __FILE__, __LINE__);
    cudaGetLastError();
    return rc2;
  }
  if (enabled_out && nf > 0) memcpy(enabled_out, en.data(), sizeof(int32_t) * nf);
  return KDS_OK;
}

}  // namespace kds
