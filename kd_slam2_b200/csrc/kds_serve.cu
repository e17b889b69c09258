// Served registration: a request loop that takes scan-to-map ICP and CT-ICP
// registrations of uneven sizes from many sensor streams, keeps each stream's local
// surfel map resident on the device, and runs the registrations with continuous
// batching.  The reference has nothing like it (one tracker thread and one aligner
// per role, kd/tracker/tracker_proc_.h:82); every alignment it runs is the same
// computation as kds_aligner_compute (TreeAlignerBase_::compute,
// kd/icp/tree_aligner_base_.h:100-115) on a moving tree from
// TreeGenerator_::makeTree (kd/tree/tree_generator_impl_.h:7-19).
//
// Host threads drive their own CUDA streams:
//  * a build thread admits arrived requests in arrival order while their estimated
//    device memory fits under the cap, copies their points to the device and builds
//    all their moving trees -- and any pending map rebuilds -- in one forest pass (with
//    two build threads, one builds what can register next and the other builds ahead;
//    see build_loop);
//  * the Gauss-Newton thread runs ticks.  One tick = one k_linearize_pair launch per
//    kind over the tiles of every active job (two tiles of one job per block), followed
//    by a compact result copy.  Requests
//    whose trees are built join at the next tick when a slot, tile space and their
//    map version are available; finished jobs leave at the tick after they finish.
//    Ticks are double buffered: tick t+1 is queued before the results of tick t are
//    read, so the device never waits for the host.
// Each job's arithmetic is independent of the others in the tick (fixed 128-leaf
// tiles, per-job partials summed in tile order), so a result is identical alone and
// in the mix.
//
// Maps: stream s's requests are numbered q = 0, 1, ...; the window w holds requests
// [wE, (w+1)E) (E = map_every).  Requests of window w align against map version w;
// version 0 is given at kds_server_add_stream, version w+1 is a tree over the world
// points (deskewed with the estimated velocities, transformed with the estimated
// poses) of the requests of window w, built once they have all finished.
//
// The serial mode is the plain drop-in for comparison: one request at a time
// through the per-call API (kds_tree_build, kds_aligner_compute), same maps.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "kds_align.cuh"
#include "kds_internal.cuh"

namespace kds {

size_t forest_workspace_bytes(int64_t n, int R);

namespace {

// ---------------------------------------------------------------------------
// Device: points of a finished request into the world frame.
// CT: p_w = X (R(w dt) p + t dt) with dt = stamp - ts_start (the per-node morph of
// kd/tree/tree_cuda_impl_.h:132-161 applied to points); ICP: p_w = X p.
__global__ void k_to_world(const float* __restrict__ xyz, const double* __restrict__ stamps, int64_t n,
                           double ts_start, Iso12 X, Vel6 v, int warp, float* __restrict__ out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  F3 p = f3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
  if (warp) {
    const float dt = (float)((stamps ? stamps[i] : 0.0) - ts_start);
    F3 pm, nm;
    warp_x(v.v, dt, p, f3(0.f, 0.f, 0.f), pm, nm);
    p = pm;
  }
  F3 w = apply_iso_x(X.m, p);
  out[3 * i] = w.x;
  out[3 * i + 1] = w.y;
  out[3 * i + 2] = w.z;
}

int to_world(const float* xyz, const double* stamps, int64_t n, double ts_start, const double* X, const double* v,
             bool warp, float* out, cudaStream_t s) {
  if (n <= 0) return KDS_OK;
  Iso12 Xf;
  Vel6 vf;
  for (int i = 0; i < 12; ++i) Xf.m[i] = (float)X[i];
  for (int i = 0; i < 6; ++i) vf.v[i] = warp ? (float)v[i] : 0.f;
  k_to_world<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(xyz, stamps, n, ts_start, Xf, vf, warp ? 1 : 0, out);
  count_launch();
  KDS_CK(cudaGetLastError());
  return KDS_OK;
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Device bytes of a built tree (the layout of tree_alloc).
int64_t tree_bytes(const TreeDev& t) {
  return 72 * t.num_nodes + 36 * t.num_leaves + 4 * t.num_points + 4096;
}
// Estimate before the build: nodes ~ n/4, leaves ~ n/8 at 16-32 points per leaf.
int64_t tree_bytes_estimate(int64_t n) { return 18 * n + 5 * n + 4 * n + 4096; }

struct Batch {  // device copy of the points of one build pass
  void* block = nullptr;
  float* xyz = nullptr;     // 3 floats per point
  double* stamps = nullptr; // 1 double per point
  int refs = 0;
  int64_t bytes = 0;
};

struct MapVersion {
  kds_tree* tree = nullptr;
  int refs = 0;
  bool superseded = false;
};

struct Request {
  int64_t ticket = 0;
  kds_request in;
  int32_t seq = 0;
  int32_t window = 0;
  int64_t win_off = 0;
  double ts_start = 0.0;
  int64_t reserved = 0;  // bytes held under the cap
  bool host_input = true; // xyz/stamps in host memory (copied host->device)
  // build results
  bool built = false;
  int32_t build_status = KDS_OK;
  kds_tree* tree = nullptr;
  std::shared_ptr<Batch> batch;
  int64_t batch_off = 0;
  // GN
  int slot = -1, kind = 0, tile_begin = 0, tile_count = 0;
  kds_result res;
  bool done = false;
};

struct StreamState {
  int64_t max_scan_points = 0;
  float* win[2] = {nullptr, nullptr};  // world points of windows w % 2
  int32_t next_seq = 0;
  std::vector<int64_t> win_fill;       // points assigned to each window
  std::vector<int32_t> win_done;       // finished requests of each window
  // (offset, count) of the world points each finished request wrote into its window;
  // a request refused at admission finishes without points
  std::vector<std::vector<std::pair<int64_t, int64_t>>> win_ranges;
  std::map<int32_t, MapVersion> maps;  // version -> tree
  int32_t installed = -1;              // newest installed version
};

struct MapTask {
  int32_t stream = 0;
  int32_t version = 0;  // version to build (from window version - 1)
  int64_t points = 0;
  std::vector<std::pair<int64_t, int64_t>> ranges;  // window buffer ranges, ascending offsets
  cudaEvent_t ready = nullptr;  // world points written (GN stream)
};

// First-fit allocator of tile ranges in one kind's arena.
struct Arena {
  int cap = 0;
  std::map<int, int> free_;  // begin -> length
  int hw = 0;                // end of the highest allocated range
  std::map<int, int> used;   // begin -> length
  void init(int c) {
    cap = c;
    free_.clear();
    used.clear();
    free_[0] = c;
    hw = 0;
  }
  int alloc(int n) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= n) {
        int b = it->first, len = it->second;
        free_.erase(it);
        if (len > n) free_[b + n] = len - n;
        used[b] = n;
        hw = std::max(hw, b + n);
        return b;
      }
    }
    return -1;
  }
  void release(int b) {
    auto u = used.find(b);
    if (u == used.end()) return;
    int n = u->second;
    used.erase(u);
    auto it = free_.emplace(b, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
    hw = used.empty() ? 0 : used.rbegin()->first + used.rbegin()->second;
  }
};

}  // namespace
}  // namespace kds

using namespace kds;

struct kds_server {
  kds_server_params P;
  std::mutex mu;
  std::condition_variable cv_build, cv_gn, cv_done;
  std::chrono::steady_clock::time_point t0;
  bool started = false, stopping = false;
  int device = 0;
  cudaStream_t sA = nullptr, sB = nullptr;  // Gauss-Newton (high priority), builds
  cudaStream_t sB2 = nullptr;               // the second build thread's stream
  cudaStream_t sA2 = nullptr;               // a tick's ICP launches, beside the CT ones on sA
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  std::thread th_build, th_build2, th_gn;
  int thread_error = KDS_OK;
  char thread_error_text[256] = {0};

  std::vector<StreamState> streams;
  std::vector<std::unique_ptr<Request>> reqs;  // by ticket
  std::deque<Request*> pending;                // submitted, not yet built (arrival order after start)
  std::deque<Request*> ready;                  // built, waiting for a slot / map
  std::deque<MapTask> map_tasks;
  int64_t completed = 0;
  int64_t reserved = 0, peak_reserved = 0, cap = 0;
  float* zero_stamps = nullptr;  // serial mode: zero stamps for map builds
  int64_t zero_cap = 0;

  // Gauss-Newton device state (served mode)
  int S = 0;  // slots; slot S is the permanently finished sentinel
  JobIn* d_jobs = nullptr;
  JobState* d_states = nullptr;
  JobOut* d_outs = nullptr;
  LinDev* d_lins = nullptr;
  TileDev* d_tiles[2] = {nullptr, nullptr};
  int2* d_pairs[2] = {nullptr, nullptr};  // blocks of two tiles of one job, per kind
  double* d_partials[2] = {nullptr, nullptr};
  SlotResult* d_res = nullptr;
  void* d_stage = nullptr;  // admitted job records (2 tick buffers)
  void* h_stage[2] = {nullptr, nullptr};
  SlotResult* h_res[2] = {nullptr, nullptr};
  cudaEvent_t ev_tick[2] = {nullptr, nullptr};
  cudaEvent_t ev_lin[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  Arena arena[2];
  std::vector<TileDev> h_tiles[2];
  std::vector<int> free_slots;
  std::vector<Request*> slot_req;

  // profiling: distinct fixed nodes each job's descents touch (algorithmic bytes)
  unsigned long long* d_touched = nullptr;
  uint32_t* d_bitmap = nullptr;
  int64_t bitmap_words = 0;

  // statistics
  int64_t ticks = 0, build_passes = 0, map_builds = 0, built_trees = 0;
  double sum_active = 0.0, lin_ms = 0.0, alg_bytes = 0.0;
  int64_t lin_launches = 0, leaf_iterations = 0, h2d_bytes = 0, d2h_bytes = 0;
  double build_ms = 0.0;      // wall time of the build passes (summed over passes)
  double build_busy_ms = 0.0;  // wall time during which at least one build pass ran
  int32_t passes_running = 0;
  int64_t released_ahead = 0;  // trees built ahead and released to make room
  double busy_since = 0.0;
  // timeline: kind (0 build pass, 1 tick), count (points / registrations), begin, end [s]
  std::vector<std::array<double, 4>> trace;
  double tick_t0[2] = {0.0, 0.0};
  int tick_n[2] = {0, 0};
  int64_t build_points = 0;   // points built (requests and maps)
  double build_point_levels = 0.0;  // sum over passes of points x levels
  double build_global_point_levels = 0.0;  // the same for the levels built level by level
};

namespace {

void fail_thread(kds_server* s, int rc) {
  std::lock_guard<std::mutex> g(s->mu);
  if (s->thread_error == KDS_OK) {
    s->thread_error = rc;
    snprintf(s->thread_error_text, sizeof(s->thread_error_text), "%s", kds_last_error());
  }
  s->stopping = true;
  s->cv_build.notify_all();
  s->cv_gn.notify_all();
  s->cv_done.notify_all();
}

int64_t request_persistent_bytes(const kds_request& r) { return 20 * r.n + tree_bytes_estimate(r.n); }

void release_map_ref(kds_server* s, int32_t stream, int32_t version) {
  StreamState& st = s->streams[stream];
  auto it = st.maps.find(version);
  if (it == st.maps.end()) return;
  if (--it->second.refs <= 0 && it->second.superseded) {
    kds_tree_free(it->second.tree);
    st.maps.erase(it);
  }
}

void install_map(kds_server* s, int32_t stream, int32_t version, kds_tree* t) {
  StreamState& st = s->streams[stream];
  for (auto& kv : st.maps) kv.second.superseded = true;
  for (auto it = st.maps.begin(); it != st.maps.end();) {
    if (it->second.refs <= 0) {
      kds_tree_free(it->second.tree);
      it = st.maps.erase(it);
    } else {
      ++it;
    }
  }
  MapVersion mv;
  mv.tree = t;
  st.maps[version] = mv;
  st.installed = version;
}

// Counts a finished request towards its window and queues the map rebuild when the
// window is complete.  The event orders the rebuild after the world-point kernels,
// which are all on the Gauss-Newton stream.  Called with the lock held.
int window_progress(kds_server* s, Request* r, bool contributed) {
  StreamState& st = s->streams[r->in.stream];
  if (contributed) st.win_ranges[r->window].emplace_back(r->win_off, r->in.n);
  if (++st.win_done[r->window] == s->P.map_every) {
    MapTask mt;
    mt.stream = r->in.stream;
    mt.version = r->window + 1;
    mt.ranges = st.win_ranges[r->window];
    std::sort(mt.ranges.begin(), mt.ranges.end());
    for (auto& g : mt.ranges) mt.points += g.second;
    KDS_CK(cudaEventCreateWithFlags(&mt.ready, cudaEventDisableTiming));
    KDS_CK(cudaEventRecord(mt.ready, s->sA));
    s->map_tasks.push_back(mt);
    s->cv_build.notify_all();
  }
  return KDS_OK;
}

// Finishes a request: world points into its window, map rebuild when the window is
// complete, result published.  Called with the lock held, on the GN thread.
int finish_request(kds_server* s, Request* r, cudaStream_t stream, const float* dev_xyz, const double* dev_st) {
  StreamState& st = s->streams[r->in.stream];
  const bool warp = r->in.type == KDS_CTICP;
  float* dst = st.win[r->window % 2] + 3 * r->win_off;
  int rc = to_world(dev_xyz, dev_st, r->in.n, r->ts_start, r->res.X, r->res.v, warp, dst, stream);
  if (!rc) rc = window_progress(s, r, true);
  if (rc) return rc;
  r->res.t_done = seconds_since(s->t0);
  r->done = true;
  s->reserved -= r->reserved;
  r->reserved = 0;
  ++s->completed;
  s->cv_done.notify_all();
  return KDS_OK;
}

// ---------------------------------------------------------------------------
// Build threads (served mode)
// With one build thread each pass takes the pending map rebuilds first (they unblock whole
// windows), then admits arrived requests in arrival order.  With two, the work is split by
// what it unblocks:
//  * the first thread takes the map rebuilds and the requests whose map version is
//    installed: everything that can register as soon as it is built;
//  * the second takes the requests whose map is not there yet and builds their trees
//    ahead, beside the first.  It admits only while
//    the reservations stay under a quarter of the cap; when the first thread cannot fit a
//    request it releases the trees built ahead (they are rebuilt later), so a request that
//    fits under the cap alone is never held back by work that waits for it.

// Releases the trees built ahead (requests whose map version is not installed) and puts
// their requests back into the pending queue in arrival order.  Called with the lock held.
bool release_ahead(kds_server* s) {
  bool any = false;
  for (auto it = s->ready.begin(); it != s->ready.end();) {
    Request* r = *it;
    if (s->streams[r->in.stream].installed >= r->window) { ++it; continue; }
    if (r->tree) kds_tree_free(r->tree);
    r->tree = nullptr;
    if (r->batch && --r->batch->refs == 0 && r->batch->block) {
      cudaFreeAsync(r->batch->block, s->sB2);
      r->batch->block = nullptr;
    }
    r->batch.reset();
    s->reserved -= r->reserved;
    r->reserved = 0;
    r->built = false;
    it = s->ready.erase(it);
    auto pos = std::find_if(s->pending.begin(), s->pending.end(), [&](const Request* q) {
      return q->in.arrival > r->in.arrival || (q->in.arrival == r->in.arrival && q->ticket > r->ticket);
    });
    s->pending.insert(pos, r);
    ++s->released_ahead;
    any = true;
  }
  return any;
}

void build_loop(kds_server* s, cudaStream_t bst, int role) {
  const bool split = s->P.build_threads > 1;  // roles as above; role 0 takes everything otherwise
  const bool ahead = split && role == 1;
  cudaSetDevice(s->device);
  std::vector<Request*> batch;
  std::vector<MapTask> maps;
  for (;;) {
    batch.clear();
    maps.clear();
    int64_t transient = 0;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      for (;;) {
        if (s->stopping) return;
        const double now = seconds_since(s->t0);
        // map rebuilds first; they are not held under the cap
        while (!ahead && !s->map_tasks.empty() && (int)maps.size() < s->P.max_build_trees) {
          maps.push_back(s->map_tasks.front());
          s->map_tasks.pop_front();
        }
        int64_t pts = 0;  // points of the pass; the maps' share is not held under the cap
        for (auto& m : maps) pts += m.points;
        int64_t rpts = 0;  // request points of the pass
        double next_arrival = -1.0;
        bool released = false;
        auto it = s->pending.begin();
        while (it != s->pending.end() && (int)(batch.size() + maps.size()) < s->P.max_build_trees) {
          Request* r = *it;
          if (r->in.arrival > now) {
            next_arrival = r->in.arrival;
            break;
          }
          if (split && (s->streams[r->in.stream].installed < r->window) != ahead) {
            ++it;
            continue;
          }
          if (!batch.empty() && pts + r->in.n > s->P.max_build_points) break;
          const int64_t need = request_persistent_bytes(r->in);
          const int64_t ws = (int64_t)forest_workspace_bytes(rpts + r->in.n, (int)batch.size() + 1);
          if (s->reserved + need + ws > (ahead ? s->cap / 4 : s->cap)) {
            if (ahead) break;
            if (split && !released && release_ahead(s)) {
              released = true;  // the queue changed: scan again (admitted requests left it)
              it = s->pending.begin();
              continue;
            }
            if (batch.empty() && need + (int64_t)forest_workspace_bytes(r->in.n, 1) > s->cap) {
              // can never fit, even alone: refused at admission, finishes with its initial guess
              it = s->pending.erase(it);
              r->res.status = KDS_ERR_ADMISSION;
              memcpy(r->res.X, r->in.X0, sizeof(r->res.X));
              memcpy(r->res.v, r->in.v0, sizeof(r->res.v));
              if (window_progress(s, r, false)) {
                lk.unlock();
                fail_thread(s, KDS_ERR_CUDA);
                return;
              }
              r->res.t_done = seconds_since(s->t0);
              r->done = true;
              ++s->completed;
              s->cv_done.notify_all();
              continue;
            }
            break;
          }
          it = s->pending.erase(it);
          r->reserved = need;
          s->reserved += need;
          r->res.t_admit = now;
          batch.push_back(r);
          pts += r->in.n;
          rpts += r->in.n;
        }
        if (!batch.empty() || !maps.empty()) {
          if (s->passes_running++ == 0) s->busy_since = seconds_since(s->t0);
          transient = batch.empty() ? 0 : (int64_t)forest_workspace_bytes(rpts, (int)batch.size());
          s->reserved += transient;
          s->peak_reserved = std::max(s->peak_reserved, s->reserved);
          break;
        }
        // a request refused above can complete a window and queue its map rebuild (its
        // notification came while this thread held the lock): take it before waiting
        if (!ahead && !s->map_tasks.empty()) continue;
        if (next_arrival > 0.0)
          s->cv_build.wait_for(lk, std::chrono::duration<double>(std::max(0.0, next_arrival - now)));
        else
          s->cv_build.wait(lk);
      }
    }
    // one forest pass over the maps and the admitted requests
    const auto pass_t0 = std::chrono::steady_clock::now();
    const int R = (int)(maps.size() + batch.size());
    std::vector<int64_t> off(R + 1, 0);
    for (int i = 0; i < (int)maps.size(); ++i) off[i + 1] = off[i] + maps[i].points;
    for (int i = 0; i < (int)batch.size(); ++i) off[maps.size() + i + 1] = off[maps.size() + i] + batch[i]->in.n;
    const int64_t N = off[R];
    auto B = std::make_shared<Batch>();
    B->bytes = 12 * N + 8 * N + 512;
    int rc = KDS_OK;
    if (N > 0) {
      cudaError_t e = cudaMallocAsync(&B->block, (size_t)B->bytes, bst);
      if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("served build: cudaMallocAsync of %lld bytes failed", (long long)B->bytes);
        fail_thread(s, KDS_ERR_OOM);
        return;
      }
    }
    float* bx = (float*)B->block;
    double* bs = (double*)((char*)B->block + ((12 * N + 255) & ~(int64_t)255));
    B->xyz = bx;
    B->stamps = bs;
    for (int i = 0; rc == KDS_OK && i < (int)maps.size(); ++i) {
      const MapTask& m = maps[i];
      const float* win = s->streams[m.stream].win[(m.version - 1) % 2];
      cudaError_t e = cudaStreamWaitEvent(bst, m.ready, 0);
      int64_t o = off[i];
      for (size_t g = 0; e == cudaSuccess && g < m.ranges.size(); ++g) {
        e = cudaMemcpyAsync(bx + 3 * o, win + 3 * m.ranges[g].first, 12 * m.ranges[g].second,
                            cudaMemcpyDeviceToDevice, bst);
        o += m.ranges[g].second;
      }
      if (e == cudaSuccess && m.points > 0) e = cudaMemsetAsync(bs + off[i], 0, 8 * m.points, bst);
      if (e != cudaSuccess) rc = cuda_status(e, "served build: map copy", __FILE__, __LINE__);
    }
    int64_t h2d = 0;
    for (int i = 0; rc == KDS_OK && i < (int)batch.size(); ++i) {
      Request* r = batch[i];
      const int64_t o = off[maps.size() + i];
      cudaError_t e = cudaMemcpyAsync(bx + 3 * o, r->in.xyz, 12 * r->in.n, cudaMemcpyDefault, bst);
      if (e == cudaSuccess)
        e = r->in.stamps ? cudaMemcpyAsync(bs + o, r->in.stamps, 8 * r->in.n, cudaMemcpyDefault, bst)
                         : cudaMemsetAsync(bs + o, 0, 8 * r->in.n, bst);
      if (e != cudaSuccess) rc = cuda_status(e, "served build: point copy", __FILE__, __LINE__);
      if (r->host_input) h2d += (r->in.stamps ? 20 : 12) * r->in.n;
    }
    std::vector<kds_tree*> trees(R, nullptr);
    std::vector<int32_t> status(R, KDS_ERR_TREE_REJECTED);
    if (rc == KDS_OK && N > 0)
      rc = tree_build_forest(bx, bs, off.data(), R, KDS_MEM_DEVICE, &s->P.tree, bst, trees.data(), status.data());
    if (rc == KDS_OK) {
      cudaError_t e = cudaStreamSynchronize(bst);
      if (e != cudaSuccess) rc = cuda_status(e, "served build", __FILE__, __LINE__);
    }
    if (rc != KDS_OK) {
      fail_thread(s, rc);
      return;
    }
    {
      std::lock_guard<std::mutex> g(s->mu);
      s->reserved -= transient;
      s->h2d_bytes += h2d;
      ++s->build_passes;
      s->build_ms += 1e3 * seconds_since(pass_t0);
      if (--s->passes_running == 0) s->build_busy_ms += 1e3 * (seconds_since(s->t0) - s->busy_since);
      s->build_points += N;
      {
        int depth = 0, glob = 0;  // levels of the pass (the same for every tree it built)
        for (auto* t : trees)
          if (t) {
            depth = std::max(depth, (int)t->d.depth);
            glob = std::max(glob, (int)t->d.global_levels);
          }
        s->build_point_levels += (double)N * depth;
        s->build_global_point_levels += (double)N * glob;
      }
      {
        const double t1 = seconds_since(s->t0);
        s->trace.push_back({0.0, (double)N, t1 - seconds_since(pass_t0), t1});
      }
      s->built_trees += R;
      for (int i = 0; i < (int)maps.size(); ++i) {
        cudaEventDestroy(maps[i].ready);
        ++s->map_builds;
        // a rejected map keeps the previous version in service
        if (trees[i]) install_map(s, maps[i].stream, maps[i].version, trees[i]);
        else {
          StreamState& st = s->streams[maps[i].stream];
          auto it = st.maps.find(st.installed);
          if (it != st.maps.end()) {
            MapVersion alias = it->second;
            st.maps.erase(it);
            st.maps[maps[i].version] = alias;
            st.installed = maps[i].version;
          }
        }
      }
      B->refs = (int)batch.size();
      const double now = seconds_since(s->t0);
      for (int i = 0; i < (int)batch.size(); ++i) {
        Request* r = batch[i];
        r->built = true;
        r->res.t_built = now;
        r->batch = B;
        r->batch_off = off[maps.size() + i];
        r->build_status = status[maps.size() + i];
        r->tree = trees[maps.size() + i];
        if (r->tree) {
          const int64_t actual = 20 * r->in.n + tree_bytes(r->tree->d);
          s->reserved += actual - r->reserved;
          r->reserved = actual;
        }
        s->ready.push_back(r);
      }
      if (B->refs == 0 && B->block) {
        cudaFreeAsync(B->block, bst);
        B->block = nullptr;
      }
      s->cv_gn.notify_all();
      if (split) s->cv_build.notify_all();  // installed maps make queued requests the other role's
    }
  }
}

// ---------------------------------------------------------------------------
// Gauss-Newton thread (served mode)
size_t stage_bytes(const kds_server* s) {
  const size_t recs = ((size_t)s->S * (sizeof(int32_t) + sizeof(JobIn) + sizeof(LinDev)) + 3 * 256 + 255) &
                      ~(size_t)255;
  return recs + (sizeof(TileDev) + sizeof(int2)) * (size_t)(s->arena[0].cap + s->arena[1].cap) + 512;
}

// Blocks of two consecutive tiles of one job (the pair form of k_linearize: two descents
// in flight per thread, the tree top staged once per two tiles); the sentinel's free tiles
// get no block.  Returns the number of pairs written to out.
int make_pairs(const TileDev* tiles, int hw, int sentinel, int2* out) {
  int n = 0;
  for (int t = 0; t < hw;) {
    if (tiles[t].job == sentinel) { ++t; continue; }
    const bool two = t + 1 < hw && tiles[t + 1].job == tiles[t].job && tiles[t + 1].lin == tiles[t].lin;
    out[n++] = make_int2(t, two ? t + 1 : -1);
    t += two ? 2 : 1;
  }
  return n;
}

void release_slot(kds_server* s, Request* r) {
  for (int t = r->tile_begin; t < r->tile_begin + r->tile_count; ++t) {
    TileDev& T = s->h_tiles[r->kind][t];
    T.job = s->S;  // the sentinel slot is always finished
    T.lin = s->S;
    T.leaf_begin = 0;
    T.leaf_end = 0;
  }
  if (r->tile_count > 0) s->arena[r->kind].release(r->tile_begin);
  s->slot_req[r->slot] = nullptr;
  s->free_slots.push_back(r->slot);
  r->slot = -1;
}

void complete_device_request(kds_server* s, Request* r, const SlotResult* sr) {
  r->res.status = KDS_OK;
  r->res.result = sr->result;
  r->res.iterations = sr->iterations;
  r->res.stats = sr->stats;
  memcpy(r->res.X, sr->X, sizeof(r->res.X));
  memcpy(r->res.v, sr->v, sizeof(r->res.v));
}

void gn_loop(kds_server* s) {
  cudaSetDevice(s->device);
  std::vector<Request*> admitted;
  std::vector<Request*> active_prev, active_cur;
  bool prev_pending = false;
  int64_t t = 0;
  for (;;) {
    admitted.clear();
    std::vector<Request*> finished_now;  // rejected builds, finished without the GN loop
    {
      std::unique_lock<std::mutex> lk(s->mu);
      for (;;) {
        if (s->stopping) return;
        // admit built requests in order while their map version exists
        for (auto it = s->ready.begin(); it != s->ready.end();) {
          Request* r = *it;
          StreamState& st = s->streams[r->in.stream];
          if (st.installed < r->window) { ++it; continue; }
          if (!r->tree) {  // rejected tree: finishes with its initial guess
            finished_now.push_back(r);
            it = s->ready.erase(it);
            continue;
          }
          if (s->free_slots.empty()) break;
          const int nt = (int)((r->tree->d.num_leaves + kTileSurfels - 1) / kTileSurfels);
          const int kind = r->in.type == KDS_ICP ? 0 : 1;
          int tb = nt > 0 ? s->arena[kind].alloc(nt) : 0;
          if (tb < 0) { ++it; continue; }
          r->kind = kind;
          r->tile_begin = tb;
          r->tile_count = nt;
          r->slot = s->free_slots.back();
          s->free_slots.pop_back();
          s->slot_req[r->slot] = r;
          st.maps[r->window].refs++;
          admitted.push_back(r);
          it = s->ready.erase(it);
        }
        bool any_active = false;
        for (Request* r : s->slot_req)
          if (r) { any_active = true; break; }
        if (any_active || prev_pending || !finished_now.empty()) break;
        s->cv_gn.wait(lk);
      }
    }
    int rc = KDS_OK;
    // requests whose tree was rejected: world points with the initial guess
    for (Request* r : finished_now) {
      std::lock_guard<std::mutex> g(s->mu);
      r->res.status = r->build_status;
      r->res.result = 0;
      memcpy(r->res.X, r->in.X0, sizeof(r->res.X));
      memcpy(r->res.v, r->in.v0, sizeof(r->res.v));
      rc = finish_request(s, r, s->sA, r->batch->xyz + 3 * r->batch_off, r->batch->stamps + r->batch_off);
      if (rc) break;
      if (--r->batch->refs == 0) {
        cudaFreeAsync(r->batch->block, s->sA);
        r->batch->block = nullptr;
      }
      r->batch.reset();
    }
    if (rc) { fail_thread(s, rc); return; }

    // ---- enqueue tick t
    active_cur.clear();
    {
      std::lock_guard<std::mutex> g(s->mu);
      for (Request* r : s->slot_req)
        if (r) active_cur.push_back(r);
      const int buf = (int)(t & 1);
      char* h = (char*)s->h_stage[buf];
      const int na = (int)admitted.size();
      // stage: [slot ids | job records | fixed-entry records] packed for this tick, tiles at a fixed offset
      auto a256 = [](size_t x) { return (x + 255) & ~(size_t)255; };
      int32_t* h_slots = (int32_t*)h;
      JobIn* h_jobs = (JobIn*)(h + a256((size_t)na * sizeof(int32_t)));
      LinDev* h_lins = (LinDev*)((char*)h_jobs + a256((size_t)na * sizeof(JobIn)));
      const size_t rec_bytes = (size_t)((char*)(h_lins + na) - h);
      TileDev* h_t0 = (TileDev*)(h + a256((size_t)s->S * (sizeof(int32_t) + sizeof(JobIn) + sizeof(LinDev)) + 3 * 256));
      TileDev* h_t1 = h_t0 + s->arena[0].cap;
      for (int i = 0; i < na; ++i) {
        Request* r = admitted[i];
        StreamState& st = s->streams[r->in.stream];
        const kds_tree* fixed = st.maps[r->window].tree;
        const kds_aligner_params& AP = r->kind == 0 ? s->P.icp : s->P.ct;
        JobIn& J = h_jobs[i];
        memset(&J, 0, sizeof(J));
        J.m_md = r->tree->d.leaf_md;
        J.m_nrm = r->tree->d.leaf_nrm;
        J.m_num_leaves = (int32_t)r->tree->d.num_leaves;
        J.kind = r->kind;
        J.mode = KDS_JOB_COMPUTE;
        J.stats_mode = 0;
        J.lin_begin = r->slot;
        J.lin_count = 1;
        J.tile_begin = r->tile_begin;
        J.tile_count = r->tile_count;
        J.P.kernel_threshold = AP.kernel_threshold;
        J.P.damping = AP.damping;
        J.P.max_error = AP.max_error;
        J.P.min_normal_cos = AP.min_normal_cos;
        J.P.min_good_measurements = AP.min_good_measurements;
        J.P.max_iterations = AP.max_iterations;
        J.P.velocity_damping = AP.velocity_damping;
        J.P.term_crit = AP.term_crit;
        J.P.d_pert = AP.d_pert;
        J.P.d_score = AP.d_score;
        memcpy(J.X0, r->in.X0, sizeof(J.X0));
        for (int k = 0; k < 6; ++k) J.v0[k] = r->kind == 0 ? 0.0 : r->in.v0[k];
        LinDev& L = h_lins[i];
        memset(&L, 0, sizeof(L));
        L.fnodes = fixed->d.nodes;
        L.fdts = fixed->d.dts_f;
        L.f_num_nodes = (int32_t)fixed->d.num_nodes;
        L.job = r->slot;
        const double I12[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
        memcpy(L.Xf, I12, sizeof(L.Xf));
        h_slots[i] = r->slot;
        for (int k = 0; k < r->tile_count; ++k) {
          TileDev& T = s->h_tiles[r->kind][r->tile_begin + k];
          T.job = r->slot;
          T.lin = r->slot;
          T.leaf_begin = k * kTileSurfels;
          T.leaf_end = std::min((k + 1) * kTileSurfels, J.m_num_leaves);
        }
      }
      const int hw0 = s->arena[0].hw, hw1 = s->arena[1].hw;
      if (hw0) memcpy(h_t0, s->h_tiles[0].data(), sizeof(TileDev) * hw0);
      if (hw1) memcpy(h_t1, s->h_tiles[1].data(), sizeof(TileDev) * hw1);
      int2* h_p0 = (int2*)(h_t1 + s->arena[1].cap);
      int2* h_p1 = h_p0 + s->arena[0].cap;
      const int np0 = make_pairs(h_t0, hw0, s->S, h_p0), np1 = make_pairs(h_t1, hw1, s->S, h_p1);
      char* d = (char*)s->d_stage + (size_t)buf * stage_bytes(s);
      cudaStream_t A = s->sA;
      cudaError_t e = cudaSuccess;
      if (na > 0) e = cudaMemcpyAsync(d, h, rec_bytes, cudaMemcpyHostToDevice, A);
      if (e == cudaSuccess && hw0)
        e = cudaMemcpyAsync(s->d_tiles[0], h_t0, sizeof(TileDev) * hw0, cudaMemcpyHostToDevice, A);
      if (e == cudaSuccess && hw1)
        e = cudaMemcpyAsync(s->d_tiles[1], h_t1, sizeof(TileDev) * hw1, cudaMemcpyHostToDevice, A);
      if (e == cudaSuccess && np0)
        e = cudaMemcpyAsync(s->d_pairs[0], h_p0, sizeof(int2) * np0, cudaMemcpyHostToDevice, A);
      if (e == cudaSuccess && np1)
        e = cudaMemcpyAsync(s->d_pairs[1], h_p1, sizeof(int2) * np1, cudaMemcpyHostToDevice, A);
      if (e != cudaSuccess) rc = cuda_status(e, "served tick upload", __FILE__, __LINE__);
      if (!rc && na > 0) {
        const int32_t* d_slots = (const int32_t*)d;
        const JobIn* d_new_jobs = (const JobIn*)(d + ((char*)h_jobs - h));
        const LinDev* d_new_lins = (const LinDev*)(d + ((char*)h_lins - h));
        rc = launch_admit_slots(d_slots, na, d_new_jobs, d_new_lins, s->d_jobs, s->d_states, s->d_outs, s->d_lins, A);
        for (int i = 0; !rc && s->P.profile && i < na; ++i) {
          Request* r = admitted[i];
          const int64_t words = (s->streams[r->in.stream].maps[r->window].tree->d.num_nodes + 31) / 32;
          if (words > s->bitmap_words) {
            if (s->d_bitmap) cudaFree(s->d_bitmap);
            s->bitmap_words = 2 * words;
            e = cudaMalloc(&s->d_bitmap, 4 * s->bitmap_words);
            if (e != cudaSuccess) { rc = cuda_status(e, "served profiling bitmap", __FILE__, __LINE__); break; }
          }
          rc = launch_touch(r->kind, s->d_jobs, s->d_lins, r->slot, (int)r->tree->d.num_leaves, s->d_bitmap, words,
                            s->d_touched + r->slot, A);
        }
      }
      if (!rc && !active_cur.empty()) {
        if (s->P.profile) cudaEventRecord(s->ev_lin[buf][0], A);
        // the two kinds touch disjoint jobs: with both present, the ICP iterations run on a
        // second stream beside the CT ones (the profiling pass keeps them in one stream, so
        // its events time the launches alone)
        const bool fork = !s->P.profile && np0 > 0 && np1 > 0;
        cudaStream_t A0 = fork ? s->sA2 : A;
        if (fork) {
          e = cudaEventRecord(s->ev_fork, A);
          if (e == cudaSuccess) e = cudaStreamWaitEvent(A0, s->ev_fork, 0);
          if (e != cudaSuccess) rc = cuda_status(e, "served tick fork", __FILE__, __LINE__);
        }
        for (int it = 0; it < s->P.iters_per_tick && !rc; ++it) {
          rc = launch_linearize_pairs(0, np0, s->d_jobs, s->d_states, s->d_outs, s->d_lins, s->d_tiles[0],
                                      s->d_pairs[0], s->d_partials[0], A0);
          if (!rc)
            rc = launch_linearize_pairs(1, np1, s->d_jobs, s->d_states, s->d_outs, s->d_lins, s->d_tiles[1],
                                        s->d_pairs[1], s->d_partials[1], A);
        }
        if (fork && !rc) {
          e = cudaEventRecord(s->ev_join, A0);
          if (e == cudaSuccess) e = cudaStreamWaitEvent(A, s->ev_join, 0);
          if (e != cudaSuccess) rc = cuda_status(e, "served tick join", __FILE__, __LINE__);
        }
        if (s->P.profile) cudaEventRecord(s->ev_lin[buf][1], A);
        int nslots = 0;
        for (Request* r : active_cur) nslots = std::max(nslots, r->slot + 1);
        if (!rc) rc = launch_collect(nslots, s->d_states, s->d_outs, s->P.profile ? s->d_touched : nullptr, s->d_res, A);
        if (!rc) {
          e = cudaMemcpyAsync(s->h_res[buf], s->d_res, sizeof(SlotResult) * nslots, cudaMemcpyDeviceToHost, A);
          s->d2h_bytes += (int64_t)sizeof(SlotResult) * nslots;
          if (e == cudaSuccess) e = cudaEventRecord(s->ev_tick[buf], A);
          if (e != cudaSuccess) rc = cuda_status(e, "served tick", __FILE__, __LINE__);
        }
        for (Request* r : active_cur) s->leaf_iterations += r->tree->d.num_leaves;
        s->sum_active += (double)active_cur.size();
        ++s->ticks;
        s->tick_t0[buf] = seconds_since(s->t0);
        s->tick_n[buf] = (int)active_cur.size();
      }
    }
    if (rc) { fail_thread(s, rc); return; }
    const bool cur_pending = !active_cur.empty();

    // ---- results of tick t-1
    if (prev_pending) {
      const int pb = (int)((t - 1) & 1);
      cudaError_t e = cudaEventSynchronize(s->ev_tick[pb]);
      if (e != cudaSuccess) { fail_thread(s, cuda_status(e, "served tick", __FILE__, __LINE__)); return; }
      std::lock_guard<std::mutex> g(s->mu);
      s->trace.push_back({1.0, (double)s->tick_n[pb], s->tick_t0[pb], seconds_since(s->t0)});
      if (s->P.profile) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, s->ev_lin[pb][0], s->ev_lin[pb][1]) == cudaSuccess) {
          s->lin_ms += ms;
          ++s->lin_launches;
        } else {
          cudaGetLastError();
        }
      }
      for (Request* r : active_prev) {
        if (r->slot < 0 || r->done) continue;
        const SlotResult& sr = s->h_res[pb][r->slot];
        if (!sr.done) continue;
        complete_device_request(s, r, &sr);
        if (s->P.profile) {
          // per Gauss-Newton iteration: 32 B per moving surfel, 32 B per distinct fixed node
          // touched, one tile partial (M + 7 doubles) written and read
          const double M = r->kind == 0 ? 27.0 + 7.0 : 90.0 + 7.0;
          s->alg_bytes += (double)sr.iterations * (32.0 * (double)r->tree->d.num_leaves + 32.0 * (double)sr.touched +
                                                   2.0 * 8.0 * M * (double)r->tile_count);
        }
        const int slot = r->slot;
        (void)slot;
        release_slot(s, r);
        release_map_ref(s, r->in.stream, r->window);
        rc = finish_request(s, r, s->sA, r->batch->xyz + 3 * r->batch_off, r->batch->stamps + r->batch_off);
        if (rc) break;
        if (--r->batch->refs == 0) {
          cudaFreeAsync(r->batch->block, s->sA);
          r->batch->block = nullptr;
        }
        r->batch.reset();
        kds_tree_free(r->tree);
        r->tree = nullptr;
      }
      s->cv_build.notify_all();
    }
    if (rc) { fail_thread(s, rc); return; }
    active_prev.swap(active_cur);
    prev_pending = cur_pending;
    ++t;
  }
}

// ---------------------------------------------------------------------------
// Serial mode: the plain drop-in, one request at a time through the per-call API.
void serial_loop(kds_server* s) {
  cudaSetDevice(s->device);
  kds_aligner* al[2] = {nullptr, nullptr};
  int rc = kds_aligner_create(KDS_ICP, &s->P.icp, &al[0]);
  if (!rc) rc = kds_aligner_create(KDS_CTICP, &s->P.ct, &al[1]);
  if (!rc) rc = kds_aligner_set_stream(al[0], s->sA);
  if (!rc) rc = kds_aligner_set_stream(al[1], s->sA);
  void* dev = nullptr;
  int64_t dev_cap = 0;
  auto cleanup = [&]() {
    if (al[0]) kds_aligner_free(al[0]);
    if (al[1]) kds_aligner_free(al[1]);
    if (dev) cudaFree(dev);
  };
  if (rc) { fail_thread(s, rc); cleanup(); return; }
  for (;;) {
    Request* r = nullptr;
    MapTask mt;
    bool have_map = false;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      for (;;) {
        if (s->stopping) { lk.unlock(); cleanup(); return; }
        if (!s->map_tasks.empty()) {
          mt = s->map_tasks.front();
          s->map_tasks.pop_front();
          have_map = true;
          break;
        }
        if (!s->pending.empty()) {
          const double now = seconds_since(s->t0);
          Request* f = s->pending.front();
          if (f->in.arrival <= now) {
            r = f;
            s->pending.pop_front();
            r->res.t_admit = now;
            break;
          }
          s->cv_build.wait_for(lk, std::chrono::duration<double>(f->in.arrival - now));
          continue;
        }
        s->cv_build.wait(lk);
      }
    }
    if (have_map) {
      StreamState& st = s->streams[mt.stream];
      kds_tree* t = nullptr;
      rc = kds_tree_build(st.win[(mt.version - 1) % 2], (const double*)s->zero_stamps, mt.points, KDS_MEM_DEVICE,
                          &s->P.tree, s->sA, &t);
      cudaEventDestroy(mt.ready);
      if (rc == KDS_ERR_TREE_REJECTED) rc = KDS_OK;
      if (rc) break;
      std::lock_guard<std::mutex> g(s->mu);
      ++s->map_builds;
      if (t) install_map(s, mt.stream, mt.version, t);
      else {
        auto it = st.maps.find(st.installed);
        MapVersion alias = it->second;
        st.maps.erase(it);
        st.maps[mt.version] = alias;
        st.installed = mt.version;
      }
      continue;
    }
    // points to the device, tree, alignment
    const int64_t need = 20 * r->in.n + 256;
    if (need > dev_cap) {
      if (dev) cudaFree(dev);
      dev = nullptr;
      cudaError_t e = cudaMalloc(&dev, (size_t)need);
      if (e != cudaSuccess) { rc = cuda_status(e, "serial: point buffer", __FILE__, __LINE__); break; }
      dev_cap = need;
    }
    float* dx = (float*)dev;
    double* ds = (double*)((char*)dev + ((12 * r->in.n + 255) & ~(int64_t)255));
    cudaError_t e = cudaMemcpyAsync(dx, r->in.xyz, 12 * r->in.n, cudaMemcpyDefault, s->sA);
    if (e == cudaSuccess)
      e = r->in.stamps ? cudaMemcpyAsync(ds, r->in.stamps, 8 * r->in.n, cudaMemcpyDefault, s->sA)
                       : cudaMemsetAsync(ds, 0, 8 * r->in.n, s->sA);
    if (e != cudaSuccess) { rc = cuda_status(e, "serial: copy", __FILE__, __LINE__); break; }
    if (r->host_input) {
      std::lock_guard<std::mutex> g(s->mu);
      s->h2d_bytes += (r->in.stamps ? 20 : 12) * r->in.n;
    }
    kds_tree* t = nullptr;
    rc = kds_tree_build(dx, ds, r->in.n, KDS_MEM_DEVICE, &s->P.tree, s->sA, &t);
    r->res.t_built = seconds_since(s->t0);
    if (rc == KDS_ERR_TREE_REJECTED) {
      r->res.status = rc;
      r->res.result = 0;
      memcpy(r->res.X, r->in.X0, sizeof(r->res.X));
      memcpy(r->res.v, r->in.v0, sizeof(r->res.v));
      rc = KDS_OK;
    } else if (rc == KDS_OK) {
      kds_aligner* a = al[r->in.type == KDS_ICP ? 0 : 1];
      const kds_tree* fixed;
      {
        std::lock_guard<std::mutex> g(s->mu);
        fixed = s->streams[r->in.stream].maps[r->window].tree;
      }
      int32_t result = 0;
      rc = kds_aligner_set_fixed(a, fixed);
      if (!rc) rc = kds_aligner_set_moving(a, t);
      if (!rc) rc = kds_aligner_set_x(a, r->in.X0);
      if (!rc && r->in.type == KDS_CTICP) rc = kds_aligner_set_velocities(a, r->in.v0);
      if (!rc) rc = kds_aligner_compute(a, 0, &result);
      if (!rc) rc = kds_aligner_get_x(a, r->res.X);
      if (!rc) rc = kds_aligner_get_stats(a, &r->res.stats);
      if (!rc) {
        if (r->in.type == KDS_CTICP) rc = kds_aligner_get_velocities(a, r->res.v);
        else memset(r->res.v, 0, sizeof(r->res.v));
      }
      r->res.status = KDS_OK;
      r->res.result = result;
      kds_stats log[64];
      int32_t nlog = 0;
      if (!rc) rc = kds_aligner_get_stats_log(a, log, 64, &nlog);
      r->res.iterations = nlog;
      kds_tree_free(t);
    }
    if (rc) break;
    {
      std::lock_guard<std::mutex> g(s->mu);
      rc = finish_request(s, r, s->sA, dx, ds);
    }
    if (rc) break;
    {
      // the per-call API reads back pose, velocities, stats and the stats log
      std::lock_guard<std::mutex> g(s->mu);
      s->d2h_bytes += (int64_t)(sizeof(JobOut) + sizeof(kds_stats) * 64);
    }
    e = cudaStreamSynchronize(s->sA);
    if (e != cudaSuccess) { rc = cuda_status(e, "serial", __FILE__, __LINE__); break; }
  }
  fail_thread(s, rc);
  cleanup();
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
void kds_server_params_default(kds_server_params* p) {
  memset(p, 0, sizeof(*p));
  p->max_slots = 512;
  p->map_every = 5;
  p->max_build_trees = 128;
  p->serial = 0;
  p->profile = 0;
  p->hbm_cap = 0;
  p->max_build_points = 16 << 20;
  p->max_tiles = 32768;
  p->iters_per_tick = 3;
  p->build_threads = 1;
  kds_tree_params_default(&p->tree);
  kds_aligner_params_default(&p->icp);
  kds_aligner_params_default(&p->ct);
}

int kds_server_create(const kds_server_params* params, kds_server** out) {
  if (!params || !out || params->max_slots <= 0 || params->map_every <= 0 || params->max_build_trees <= 0 ||
      params->max_tiles <= 0 || params->iters_per_tick <= 0 || params->build_threads > 2) {
    set_error("kds_server_create: bad parameters");
    return KDS_ERR_INVALID_ARG;
  }
  *out = nullptr;
  int rc = ensure_init();
  if (rc) return rc;
  std::unique_ptr<kds_server> s(new kds_server());
  s->P = *params;
  KDS_CK(cudaGetDevice(&s->device));
  int lo = 0, hi = 0;
  KDS_CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  KDS_CK(cudaStreamCreateWithPriority(&s->sA, cudaStreamNonBlocking, hi));
  KDS_CK(cudaStreamCreateWithPriority(&s->sA2, cudaStreamNonBlocking, hi));
  KDS_CK(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming));
  KDS_CK(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming));
  // both build streams at the lowest priority: a build stream above the other made the
  // two passes preempt each other's blocks (two overlapped passes took 35-55 ms instead of
  // 8-13 ms in some steps)
  KDS_CK(cudaStreamCreateWithPriority(&s->sB, cudaStreamNonBlocking, lo));
  KDS_CK(cudaStreamCreateWithPriority(&s->sB2, cudaStreamNonBlocking, lo));
  size_t fr = 0, tot = 0;
  KDS_CK(cudaMemGetInfo(&fr, &tot));
  const int64_t avail = (int64_t)(fr * 0.9);
  s->cap = params->hbm_cap > 0 ? std::min<int64_t>(params->hbm_cap, avail) : avail;
  if (!params->serial) {
    s->S = params->max_slots;
    s->arena[0].init(params->max_tiles);
    s->arena[1].init(params->max_tiles);
    s->h_tiles[0].assign(params->max_tiles, TileDev{params->max_slots, params->max_slots, 0, 0});
    s->h_tiles[1].assign(params->max_tiles, TileDev{params->max_slots, params->max_slots, 0, 0});
    const int S1 = s->S + 1;
    KDS_CK(cudaMalloc(&s->d_jobs, sizeof(JobIn) * S1));
    KDS_CK(cudaMalloc(&s->d_states, sizeof(JobState) * S1));
    KDS_CK(cudaMalloc(&s->d_outs, sizeof(JobOut) * S1));
    KDS_CK(cudaMalloc(&s->d_lins, sizeof(LinDev) * S1));
    KDS_CK(cudaMalloc(&s->d_res, sizeof(SlotResult) * S1));
    KDS_CK(cudaMalloc(&s->d_touched, sizeof(unsigned long long) * S1));
    KDS_CK(cudaMemset(s->d_touched, 0, sizeof(unsigned long long) * S1));
    for (int k = 0; k < 2; ++k) {
      KDS_CK(cudaMalloc(&s->d_tiles[k], sizeof(TileDev) * params->max_tiles));
      KDS_CK(cudaMemcpy(s->d_tiles[k], s->h_tiles[k].data(), sizeof(TileDev) * params->max_tiles,
                        cudaMemcpyHostToDevice));
      KDS_CK(cudaMalloc(&s->d_partials[k], sizeof(double) * kPStride * params->max_tiles));
      KDS_CK(cudaMalloc(&s->d_pairs[k], sizeof(int2) * params->max_tiles));
      KDS_CK(cudaMallocHost(&s->h_stage[k], stage_bytes(s.get())));
      KDS_CK(cudaMallocHost(&s->h_res[k], sizeof(SlotResult) * S1));
      KDS_CK(cudaEventCreateWithFlags(&s->ev_tick[k], cudaEventDisableTiming));
      KDS_CK(cudaEventCreate(&s->ev_lin[k][0]));
      KDS_CK(cudaEventCreate(&s->ev_lin[k][1]));
    }
    KDS_CK(cudaMalloc(&s->d_stage, 2 * stage_bytes(s.get())));
    // every slot starts finished; the sentinel slot S stays finished
    std::vector<JobState> st(S1);
    memset(st.data(), 0, sizeof(JobState) * S1);
    for (auto& x : st) x.done = 1;
    KDS_CK(cudaMemcpy(s->d_states, st.data(), sizeof(JobState) * S1, cudaMemcpyHostToDevice));
    s->slot_req.assign(s->S, nullptr);
    for (int i = s->S - 1; i >= 0; --i) s->free_slots.push_back(i);
    rc = linearize_smem_setup();
    if (rc) return rc;
  }
  *out = s.release();
  return KDS_OK;
}

int kds_server_add_stream(kds_server* s, const float* map_xyz, int64_t n, int64_t max_scan_points,
                          int32_t* stream_id) {
  if (!s || !map_xyz || n <= 0 || max_scan_points <= 0 || !stream_id) {
    set_error("kds_server_add_stream: bad arguments");
    return KDS_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> g(s->mu);
  if (s->started) { set_error("kds_server_add_stream: the server has started"); return KDS_ERR_STATE; }
  StreamState st;
  st.max_scan_points = max_scan_points;
  const int64_t wcap = max_scan_points * s->P.map_every;
  for (int k = 0; k < 2; ++k) KDS_CK(cudaMalloc(&st.win[k], 12 * wcap));
  // map version 0: built here, before the clock starts
  float* dxyz = nullptr;
  KDS_CK(cudaMalloc(&dxyz, 12 * n));
  KDS_CK(cudaMemcpy(dxyz, map_xyz, 12 * n, cudaMemcpyHostToDevice));
  if (s->zero_cap < std::max(n, wcap)) {
    if (s->zero_stamps) cudaFree(s->zero_stamps);
    s->zero_cap = std::max(n, wcap);
    KDS_CK(cudaMalloc(&s->zero_stamps, 8 * s->zero_cap));
    KDS_CK(cudaMemset(s->zero_stamps, 0, 8 * s->zero_cap));
  }
  kds_tree* t = nullptr;
  int rc = kds_tree_build(dxyz, (const double*)s->zero_stamps, n, KDS_MEM_DEVICE, &s->P.tree, s->sA, &t);
  cudaStreamSynchronize(s->sA);
  cudaFree(dxyz);
  if (rc) {
    for (int k = 0; k < 2; ++k) cudaFree(st.win[k]);
    return rc;
  }
  MapVersion mv;
  mv.tree = t;
  st.maps[0] = mv;
  st.installed = 0;
  *stream_id = (int32_t)s->streams.size();
  s->streams.push_back(std::move(st));
  return KDS_OK;
}

int kds_server_submit(kds_server* s, const kds_request* req, int64_t* ticket) {
  if (!s || !req || !ticket || req->n <= 0 || !req->xyz || (req->type != KDS_ICP && req->type != KDS_CTICP)) {
    set_error("kds_server_submit: bad arguments");
    return KDS_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> g(s->mu);
  if (s->thread_error) { set_error("%s", s->thread_error_text); return s->thread_error; }
  if (req->stream < 0 || req->stream >= (int32_t)s->streams.size()) {
    set_error("kds_server_submit: unknown stream %d", req->stream);
    return KDS_ERR_INVALID_ARG;
  }
  StreamState& st = s->streams[req->stream];
  if (req->n > st.max_scan_points) {
    set_error("kds_server_submit: %lld points exceed the stream's max_scan_points %lld", (long long)req->n,
              (long long)st.max_scan_points);
    return KDS_ERR_CAPACITY;
  }
  if (!s->pending.empty() && req->arrival < s->pending.back()->in.arrival) {
    set_error("kds_server_submit: arrivals must be non-decreasing");
    return KDS_ERR_INVALID_ARG;
  }
  std::unique_ptr<Request> r(new Request());
  r->ticket = (int64_t)s->reqs.size();
  r->in = *req;
  r->seq = st.next_seq++;
  r->window = r->seq / s->P.map_every;
  if ((int)st.win_fill.size() <= r->window) {
    st.win_fill.resize(r->window + 1, 0);
    st.win_done.resize(r->window + 1, 0);
    st.win_ranges.resize(r->window + 1);
  }
  r->win_off = st.win_fill[r->window];
  st.win_fill[r->window] += req->n;
  double t0 = 0.0;
  if (req->stamps) {
    cudaPointerAttributes sa;
    bool dev_stamps = false;
    if (cudaPointerGetAttributes(&sa, req->stamps) == cudaSuccess)
      dev_stamps = sa.type == cudaMemoryTypeDevice;
    else
      cudaGetLastError();
    if (dev_stamps) {
      std::vector<double> hs((size_t)req->n);
      KDS_CK(cudaMemcpy(hs.data(), req->stamps, sizeof(double) * req->n, cudaMemcpyDeviceToHost));
      t0 = *std::min_element(hs.begin(), hs.end());
    } else {
      t0 = req->stamps[0];
      for (int64_t i = 1; i < req->n; ++i) t0 = std::min(t0, req->stamps[i]);
    }
  }
  r->ts_start = t0;
  cudaPointerAttributes pa;
  if (cudaPointerGetAttributes(&pa, req->xyz) == cudaSuccess)
    r->host_input = pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged;
  else
    cudaGetLastError();
  memset(&r->res, 0, sizeof(r->res));
  r->res.t_arrival = req->arrival;
  r->res.map_version = r->window;
  *ticket = r->ticket;
  s->pending.push_back(r.get());
  s->reqs.push_back(std::move(r));
  s->cv_build.notify_all();
  return KDS_OK;
}

int kds_server_start(kds_server* s) {
  if (!s) return KDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(s->mu);
  if (s->started) { set_error("kds_server_start: already started"); return KDS_ERR_STATE; }
  s->started = true;
  s->t0 = std::chrono::steady_clock::now();
  if (s->P.serial) {
    s->th_build = std::thread(serial_loop, s);
  } else {
    s->th_build = std::thread(build_loop, s, s->sB, 0);
    if (s->P.build_threads > 1) s->th_build2 = std::thread(build_loop, s, s->sB2, 1);
    s->th_gn = std::thread(gn_loop, s);
  }
  return KDS_OK;
}

int kds_server_drain(kds_server* s, double timeout_s) {
  if (!s) return KDS_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto pred = [&]() { return s->thread_error != KDS_OK || s->completed == (int64_t)s->reqs.size(); };
  if (timeout_s > 0) {
    if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) {
      set_error("kds_server_drain: %lld of %lld requests finished before the timeout", (long long)s->completed,
                (long long)s->reqs.size());
      return KDS_ERR_TIMEOUT;
    }
  } else {
    s->cv_done.wait(lk, pred);
  }
  if (s->thread_error) { set_error("%s", s->thread_error_text); return s->thread_error; }
  return KDS_OK;
}

int kds_server_wait(kds_server* s, int64_t ticket, double timeout_s, kds_result* out) {
  if (!s || !out) return KDS_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  if (ticket < 0 || ticket >= (int64_t)s->reqs.size()) { set_error("kds_server_wait: bad ticket"); return KDS_ERR_INVALID_ARG; }
  Request* r = s->reqs[ticket].get();
  auto pred = [&]() { return s->thread_error != KDS_OK || r->done; };
  if (timeout_s > 0) {
    if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) {
      set_error("kds_server_wait: request %lld not finished before the timeout", (long long)ticket);
      return KDS_ERR_TIMEOUT;
    }
  } else {
    s->cv_done.wait(lk, pred);
  }
  if (!r->done && s->thread_error) { set_error("%s", s->thread_error_text); return s->thread_error; }
  *out = r->res;
  return KDS_OK;
}

int kds_server_get_trace(kds_server* s, double* rows4, int32_t cap, int32_t* n) {
  if (!s || !n || (cap > 0 && !rows4)) return KDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(s->mu);
  *n = (int32_t)s->trace.size();
  const int m = std::min<int>(cap, (int)s->trace.size());
  for (int i = 0; i < m; ++i)
    for (int k = 0; k < 4; ++k) rows4[4 * i + k] = s->trace[i][k];
  return KDS_OK;
}

int kds_server_get_stats(kds_server* s, kds_server_stats* st) {
  if (!s || !st) return KDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(s->mu);
  memset(st, 0, sizeof(*st));
  st->submitted = (int64_t)s->reqs.size();
  st->completed = s->completed;
  st->ticks = s->ticks;
  st->build_passes = s->build_passes;
  st->map_builds = s->map_builds;
  st->built_trees = s->built_trees;
  st->hbm_cap = s->cap;
  st->peak_reserved = s->peak_reserved;
  st->mean_active = s->ticks ? s->sum_active / (double)s->ticks : 0.0;
  st->lin_ms = s->lin_ms;
  st->lin_ticks = s->lin_launches;
  st->leaf_iterations = s->leaf_iterations;
  st->alg_bytes = s->alg_bytes;
  st->h2d_bytes = s->h2d_bytes;
  st->d2h_bytes = s->d2h_bytes;
  st->build_ms = s->build_ms;
  st->build_busy_ms = s->build_busy_ms;
  st->build_released_ahead = s->released_ahead;
  st->build_points = s->build_points;
  st->build_point_levels = s->build_point_levels;
  st->build_global_point_levels = s->build_global_point_levels;
  return KDS_OK;
}

void kds_server_free(kds_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stopping = true;
    s->cv_build.notify_all();
    s->cv_gn.notify_all();
    s->cv_done.notify_all();
  }
  if (s->th_build.joinable()) s->th_build.join();
  if (s->th_build2.joinable()) s->th_build2.join();
  if (s->th_gn.joinable()) s->th_gn.join();
  cudaStreamSynchronize(s->sA);
  cudaStreamSynchronize(s->sB);
  cudaStreamSynchronize(s->sB2);
  for (auto& r : s->reqs) {
    if (r->tree) kds_tree_free(r->tree);
    if (r->batch && r->batch->block) {
      cudaFree(r->batch->block);
      r->batch->block = nullptr;
    }
  }
  for (auto& mt : s->map_tasks) cudaEventDestroy(mt.ready);
  for (auto& st : s->streams) {
    for (auto& kv : st.maps) kds_tree_free(kv.second.tree);
    for (int k = 0; k < 2; ++k) cudaFree(st.win[k]);
  }
  cudaStreamSynchronize(s->sA);
  cudaStreamSynchronize(s->sB);
  cudaStreamSynchronize(s->sB2);
  cudaFree(s->d_jobs);
  cudaFree(s->d_states);
  cudaFree(s->d_outs);
  cudaFree(s->d_lins);
  cudaFree(s->d_res);
  cudaFree(s->d_touched);
  cudaFree(s->d_bitmap);
  cudaFree(s->d_stage);
  cudaFree(s->zero_stamps);
  for (int k = 0; k < 2; ++k) {
    cudaFree(s->d_tiles[k]);
    cudaFree(s->d_pairs[k]);
    cudaFree(s->d_partials[k]);
    if (s->h_stage[k]) cudaFreeHost(s->h_stage[k]);
    if (s->h_res[k]) cudaFreeHost(s->h_res[k]);
    if (s->ev_tick[k]) cudaEventDestroy(s->ev_tick[k]);
    if (s->ev_lin[k][0]) cudaEventDestroy(s->ev_lin[k][0]);
    if (s->ev_lin[k][1]) cudaEventDestroy(s->ev_lin[k][1]);
  }
  cudaStreamSynchronize(s->sA2);
  if (s->ev_fork) cudaEventDestroy(s->ev_fork);
  if (s->ev_join) cudaEventDestroy(s->ev_join);
  cudaStreamDestroy(s->sA);
  cudaStreamDestroy(s->sA2);
  cudaStreamDestroy(s->sB);
  cudaStreamDestroy(s->sB2);
  cudaGetLastError();
  delete s;
}
