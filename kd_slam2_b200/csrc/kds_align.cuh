// Device-side job layout of the fused linearization kernel and its host runner.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "kds_internal.cuh"

namespace kds {

constexpr int kMaxLog = 64;      // per-job stats_log depth
constexpr int kPStride = 200;    // doubles per tile partial: 189 entries (D = 18) + stats
constexpr int kPStats = 192;     // offset of the 7 stats values inside a partial

// Per-iteration float view of the state for one (job, fixed entry) pair: the
// QuadraticTermCache of kd/icp/icp_.h:97-102 plus the velocities.
struct CacheF {
  float Xm[12];
  float Xf[12];
  float Xmf[12];
  float v[6];
  float fv[6];
};

struct ParamsF {
  float kernel_threshold;
  float damping;
  float max_error;
  float min_normal_cos;
  int32_t min_good_measurements;
  int32_t max_iterations;
  float velocity_damping;
  int32_t term_crit;
  float d_pert;
  float d_score;
};

// One fixed entry of a job (the FixedEntry of kd/icp/tree_aligner_base_.h:57-74).
struct LinDev {
  const DNode* fnodes;
  const float* fdts;
  int32_t f_num_nodes;
  int32_t job;
  double Xf[12];
  double fv[6];
  CacheF cache;  // written on the device
};

struct JobIn {
  const float4* m_md;
  const float4* m_nrm;
  int32_t m_num_leaves;
  int32_t kind;  // 0 ICP, 1 CT, 2 CT dual
  int32_t mode;  // KDS_JOB_*
  int32_t stats_mode;
  int32_t lin_begin, lin_count;
  int32_t tile_begin, tile_count;
  ParamsF P;
  int32_t prior_enabled;
  int32_t keep_cache;  // 1: use the caches already in LinDev (explicit-cache linearization)
  double prior_ZXi[12];
  double prior_info[36];
  double X0[12];
  double v0[6];
};

struct JobState {
  double X[12];
  double v[6];
  int32_t iter, done, result, max_iter;
  unsigned int arrive;
  float prev_score;
};

struct JobOut {
  double X[12];
  double v[6];
  int32_t result;
  int32_t iterations;
  kds_stats stats;
  double H[144];
  double b[12];
  double dx[12];
  double H_vel_B[36], b_vel_B[6], H_cross_pose_vel_B[36], H_cross_vel_AB[36];
};

struct TileDev {
  int32_t job;
  int32_t lin;
  int32_t leaf_begin;
  int32_t leaf_end;
};

// Owns the device buffers of a batch of jobs and (optionally) a CUDA graph of its
// launches: k_init_jobs followed by one k_linearize per Gauss-Newton iteration.
struct Runner {
  void* block = nullptr;
  int cap_jobs = 0, cap_lins = 0, cap_tiles = 0;
  JobIn* d_jobs = nullptr;
  JobState* d_states = nullptr;
  JobOut* d_outs = nullptr;
  kds_stats* d_logs = nullptr;
  LinDev* d_lins = nullptr;
  TileDev* d_tiles = nullptr;
  double* d_partials = nullptr;  // scratch: one kPStride partial per tile
  int32_t* d_err = nullptr;      // error bits of the last launch sequence (zeroed by k_init_jobs)
  int32_t* d_ready = nullptr;    // persistent form: per job, the next iteration that may start
  unsigned int* d_queue = nullptr;  // persistent form: [0] next work item, [1] abort
  int2* d_pairs = nullptr;          // two-tile blocks: (tile, tile or -1), grouped by kind
  std::vector<JobIn> h_jobs;
  std::vector<LinDev> h_lins;
  std::vector<TileDev> h_tiles;
  std::vector<int2> h_pairs;
  int kind_pair_begin[3] = {0, 0, 0}, kind_pair_count[3] = {0, 0, 0};
  int num_jobs = 0, num_tiles = 0;
  int kind_begin[3] = {0, 0, 0}, kind_count[3] = {0, 0, 0};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  std::vector<int64_t> graph_key;
  std::vector<int64_t> last_key;  // shape of the previous run
  // number of top fixed-tree nodes each block stages in shared memory (32 B each)
  int stage_nodes = 2047;
  // tiles of larger jobs first (1) or in job order (0); tuned by kds_batch_autotune
  int order_by_size = 0;
  // 1: every iteration of every job in one persistent launch over a device work queue
  // (k_linearize_persistent); 0: one k_linearize launch per iteration and kind
  int persistent = 0;
  // 1: two tiles of one (job, fixed entry) per block, two descents in flight per thread
  // (k_linearize_pair); ignored by the persistent form
  int pair_tiles = 0;
  bool smem_attr_set = false;
  bool persistent_attr_set = false;
  // optional event pair per linearization launch (measurement only)
  bool profiling = false;
  std::vector<cudaEvent_t> prof_ev;
  int prof_launches = 0;
  int ensure_events(int n);
  double profile_mean_ms(int* launches) const;

  int reserve(int nj, int nl, int nt);
  void release();
  void drop_graph();
  int setup(const std::vector<JobIn>& jobs, const std::vector<LinDev>& lins, cudaStream_t s);
  int max_launches() const;
  int enqueue(cudaStream_t s, int32_t* dbg_match, int32_t* dbg_status);
  int run(cudaStream_t s, bool use_graph, int32_t* dbg_match, int32_t* dbg_status);
  int fetch(cudaStream_t s, std::vector<JobOut>& outs, std::vector<kds_stats>* logs);
  ~Runner() { release(); }
};

int count_touched(Runner& R, int kind, int64_t fixed_nodes, int64_t* out, cudaStream_t s);
// KDS_OK for err == 0, else KDS_ERR_TIMEOUT with a message for the error bits of
// k_linearize (1: a tree-top copy wait gave up, results valid; 2: the copy was not seen
// complete at block exit, context suspect).
int timeout_status(int32_t err);
// Polls of the first bounded wait for the tree-top copy, on the current device.
int set_wait_spins(int32_t spins);
// on: 1/0 enables/disables the phase stamps (-1 leaves it); out16 (nullable) receives them
int phase_stamps(int on, unsigned long long* out16);

// Served-loop helpers.  In the served loop a slot index is both the job index and the
// fixed-entry index; the tiles of each kind live in their own arena.
struct SlotResult {
  int32_t done, result, iterations, pad_;
  kds_stats stats;
  double X[12];
  double v[6];
  unsigned long long touched;  // distinct fixed nodes the descents visit at the initial state (profiling)
};
constexpr int kStageNodes = 2047;  // most fixed-tree nodes any launch stages in shared memory
constexpr int kServeStage = 1023;  // nodes the served loop stages (a smaller stage leaves room for more blocks)
constexpr int kTileSurfels = 128;  // moving surfels per tile = threads per k_linearize block
// Copies n admitted job records into their slots and initialises those jobs.
int launch_admit_slots(const int32_t* d_slots, int n, const JobIn* new_jobs, const LinDev* new_lins, JobIn* jobs,
                       JobState* states, JobOut* outs, LinDev* lins, cudaStream_t s);
int launch_linearize(int kind, int ntiles, const JobIn* jobs, JobState* states, JobOut* outs, LinDev* lins,
                     const TileDev* tiles, double* partials, cudaStream_t s);
// Two tiles of one (job, fixed entry) per block (k_linearize_pair): pairs[i] = (tile,
// second tile or -1).
int launch_linearize_pairs(int kind, int npairs, const JobIn* jobs, JobState* states, JobOut* outs, LinDev* lins,
                           const TileDev* tiles, const int2* pairs, double* partials, cudaStream_t s);
int launch_collect(int n, const JobState* states, const JobOut* outs, const unsigned long long* touched,
                   SlotResult* res, cudaStream_t s);
// Counts the distinct fixed nodes that the descents of job `slot` visit at its current
// caches into *count (bitmap: words zeroed 32-bit words of scratch).
int launch_touch(int kind, const JobIn* jobs, const LinDev* lins, int slot, int num_leaves, uint32_t* bitmap,
                 int64_t words, unsigned long long* count, cudaStream_t s);
int linearize_smem_setup();

// One linearization whose scratch is a file-scope device array (no allocation).
// Rejects more than 65,536 moving leaves with KDS_ERR_CAPACITY.
int linearize_static(const TreeDev& fixed, const TreeDev& moving, int32_t type, const kds_aligner_params& P,
                     const double* X, const double* Xf, const double* v, const double* fv, int32_t stats_mode,
                     cudaStream_t s, double* H, double* b, kds_stats* stats);

// Device assembly of multi-view factor blocks from a runner's last outputs (kds_factor.cu).
int batch_assemble(Runner& R, const kds_factor* F, int32_t nf, int32_t nvars, float ratio, cudaStream_t s,
                   int32_t* num_blocks, int32_t* block_rc, double* H_out, double* b_out, int32_t* enabled_out);

}  // namespace kds
