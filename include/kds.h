/*
 * kds.h -- C ABI of the B200-native KD-SLAM registration path (libkds.so).
 *
 * This library replaces, for one CUDA device, the reference's registration hot path:
 * surfel KD-tree build, greedy nearest-surfel descent, symmetric surfel-to-surfel ICP,
 * continuous-time CT-ICP with per-leaf deskew, and the Gauss-Newton H,b reduction and
 * solve.  Each entry point names the reference interface it stands in for (paths are
 * relative to the reference project, kd/ = kd_slam2/src/lib/kd_slam/).
 *
 * Conventions
 *  - Every function returns an int status (KDS_OK = 0, negative on error); none exits
 *    the process (the reference's CUDA_CHECK calls exit(), kd/cuda/cuda_common.h:30-35).
 *  - Poses are 3x4 row-major [R | t] (12 doubles), world <- body, as Eigen::Isometry3.
 *  - Velocities are [v_x v_y v_z w_x w_y w_z] (decoupled body velocity, kd/cticp/cticp_.h:135-138).
 *  - `stream` arguments take a cudaStream_t; NULL selects the per-thread default stream.
 *  - Handles are not thread-safe; distinct handles may be used from distinct threads.
 *  - The caller owns trees; aligners hold non-owning references to them
 *    (kd/icp/tree_aligner_base_.h:49-50) and own their device workspaces.
 */
#ifndef KDS_H
#define KDS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  KDS_OK = 0,
  KDS_ERR_INVALID_ARG = -1,
  KDS_ERR_CUDA = -2,
  KDS_ERR_OOM = -3,
  KDS_ERR_TREE_REJECTED = -4, /* makeTree returned nullptr: too few points or good leaves */
  KDS_ERR_RANGE = -5,         /* coordinate or timestamp outside the supported range */
  KDS_ERR_BAD_TREE = -6,      /* malformed node array */
  KDS_ERR_STATE = -7,         /* aligner used without fixed/moving tree */
  KDS_ERR_TIMEOUT = -8,       /* a bounded device-side wait gave up */
  KDS_ERR_ADMISSION = -9,     /* server refused a request (memory budget) */
  KDS_ERR_NO_DEVICE = -10,
  KDS_ERR_CAPACITY = -11,     /* a fixed-size buffer is too small for the request */
  KDS_ERR_DIVERGED = -12      /* the tracker's aligned pose is not finite */
};

enum { KDS_ICP = 0, KDS_CTICP = 1 };
enum { KDS_MEM_HOST = 0, KDS_MEM_DEVICE = 1 };

typedef struct kds_tree kds_tree;
typedef struct kds_aligner kds_aligner;

/* Human-readable text of the last error on the calling thread. */
const char* kds_last_error(void);

/* Number of CUDA kernels libkds has launched in this process (launch accounting; no
 * reference counterpart).  Launches replayed from a CUDA graph count once per replay. */
int64_t kds_launch_count(void);

/* Replaces lib/kd_slam_cuda_init.cu:3-6 (cudaSetDeviceFlags in a .so constructor):
 * selects the device and, if blocking_sync != 0, sets cudaDeviceScheduleBlockingSync
 * before the context exists.  Optional; first use of any entry point initialises. */
int kds_init(int32_t device, int32_t blocking_sync);

/* ------------------------------------------------------------------------------
 * Tree
 * ------------------------------------------------------------------------------ */

/* TreeGenerator_ PARAMs (kd/tree/tree_generator_.h:18-25), same names and defaults. */
typedef struct {
  int32_t propagate_normal;         /* false */
  int32_t tree_min_good_leaves;     /* 10 */
  int32_t leaf_min_points;          /* 5 */
  int32_t leaf_max_points;          /* 30 */
  float leaf_density;               /* 100 */
  float leaf_min_normal_incidence;  /* 0.1 */
  float leaf_eigenvalue_threshold;  /* 1e-3 (read but unused, as in the reference) */
  float leaf_normal_eigenratio;     /* 0.1 */
  float prune_min_normal_incidence; /* 0.1: IsGoodLeafPredicate_ default, kd/tree/tree_predicates_.h:15 */
  int32_t max_level;                /* 48: depth cap (the reference has none) */
} kds_tree_params;

void kds_tree_params_default(kds_tree_params* p);

typedef struct {
  int64_t num_nodes;
  int64_t num_leaves;
  int64_t num_points;
  int64_t num_unpruned;
  double ts_start; /* Tree_::_ts_start */
  int32_t accepted;
  int32_t depth;
  int32_t global_levels; /* levels the build ran level by level; the levels below, in subtrees of at
                            most 1,024 points, were finished in shared memory (== depth if none) */
  int32_t pad_;
} kds_tree_info;

/* Replaces TreeGenerator_::makeTree (kd/tree/tree_generator_impl_.h:7-19) and the
 * TreeCPU_ build + prune + BFS relabel it runs (kd/tree/tree_cpu_.h:61-90,172-207),
 * built on the GPU.  xyz: n*3 floats, stamps: n doubles or NULL (all zero).
 * mem: KDS_MEM_HOST (copied to the device inside) or KDS_MEM_DEVICE.
 * Returns KDS_ERR_TREE_REJECTED (and *out = NULL) where makeTree returns nullptr. */
int kds_tree_build(const float* xyz, const double* stamps, int64_t n, int32_t mem, const kds_tree_params* p,
                   void* stream, kds_tree** out);

/* Batched form of kds_tree_build: num_trees clouds stored back to back (cloud r is
 * points [offsets[r], offsets[r+1]) of xyz/stamps; offsets[0] = 0) built in one
 * level-synchronous pass.  out[r] / status[r] per cloud (KDS_OK or
 * KDS_ERR_TREE_REJECTED); the return value reports failures of the whole call. */
int kds_tree_build_batch(const float* xyz, const double* stamps, const int64_t* offsets, int32_t num_trees,
                         int32_t mem, const kds_tree_params* p, void* stream, kds_tree** out, int32_t* status);
/* kds_tree_build_batch over clouds in separate host arrays: cloud r is counts[r] points
 * at xyz[r] (stamps[r], or zeros when stamps or stamps[r] is NULL), copied one by one
 * into place on the device, so the caller need not pack them into one array first. */
int kds_tree_build_batch_gather(const float* const* xyz, const double* const* stamps, const int64_t* counts,
                                int32_t num_trees, const kds_tree_params* p, void* stream, kds_tree** out,
                                int32_t* status);

/* Replaces Tree_CUDAfromCPU_ (kd/tree/tree_cuda_impl_.h:197-222): uploads a node
 * array in the Node_ field order (kd/tree/node_.h:33-43), BFS numbered, node 0 the
 * root.  dts_mean/dts_cov/start/end may be NULL.  Leaves = nodes with no children. */
int kds_tree_import(const float* mean, const float* dir, const double* dts_mean, const double* dts_cov,
                    const int64_t* idx_start, const int64_t* idx_end, const int32_t* left, const int32_t* right,
                    int64_t num_nodes, double ts_start, kds_tree** out);

int kds_tree_get_info(const kds_tree* t, kds_tree_info* info);

/* Tree_::root_mean / root_eigenvalues / root_eigenvectors (kd/tree/tree_.h:35-37) as
 * TreeCPU_'s constructor sets them (kd/tree/tree_cpu_.h:72-86): the root's mean, its
 * covariance eigenvalues ascending and eigenvectors column-major (columns 0 and 2
 * reoriented towards the origin, column 0 negated if the determinant is negative).
 * Built trees carry their own; trees from kds_tree_from_msg carry the message's; trees
 * from kds_tree_import carry zeros.  Any pointer may be NULL. */
int kds_tree_get_root(const kds_tree* t, float mean[3], float eigenvalues[3], float eigenvectors[9]);

/* ------------------------------------------------------------------------------
 * Scan input: toPointsVector + Voxelizer_::voxelize, on the device
 * ------------------------------------------------------------------------------ */

/* Voxelizer_ PARAMs (kd/utils/voxelizer_.h:37-41), same names and defaults. */
typedef struct {
  float range_min;      /* 0: min lidar range [m] */
  float range_max;      /* 100: max lidar range [m] */
  float space_res;      /* 0: spatial voxel resolution [m]; 0 = no voxel grid */
  float time_res;       /* 0: temporal voxel resolution [s]; 0 = disabled */
  int32_t use_boundary; /* 0: conservative boundary clipping */
} kds_voxel_params;

void kds_voxel_params_default(kds_voxel_params* p);

/* Replaces toPointsVector (lib/kd_io/scan_utils_impl_.h:9-33) followed by
 * Voxelizer_::voxelize (kd/utils/voxelizer_impl_.h:111-145): stamps are the per-point
 * stamps when given, else msg_t + (atan2(y, x) + pi) / (2 pi) * scan_duration when
 * scan_duration > 0, else msg_t.  Without a voxel grid the points within
 * [range_min, range_max] are kept in input order; with one, each occupied voxel gives
 * the mean of its points (float sums in input order, stamps in double, as the
 * reference's Accumulator) if that mean is within range -- voxels in ascending order of
 * their integer index (x, y, z, t) where the reference emits its hash map's order.
 * Inputs and outputs are in the memory that mem names; out_xyz (3n floats) and
 * out_stamps (n doubles, may be NULL) have room for n points; *out_n receives the
 * count.  The output feeds kds_tree_build directly. */
int kds_points_voxelize(const float* xyz, const double* stamps, int64_t n, int32_t mem, double msg_t,
                        double scan_duration, const kds_voxel_params* p, void* stream, float* out_xyz,
                        double* out_stamps, int64_t* out_n);

/* ------------------------------------------------------------------------------
 * Tree wire format: kd_slam2_msgs/msg/KDTree3f with KDNode3f nodes (no points)
 * ------------------------------------------------------------------------------ */

/* kd_slam2_msgs/msg/KDNode3f (kd_slam2_msgs/msg/KDNode3f.msg), field for field, in the
 * layout of its generated C++ struct (56 bytes). */
typedef struct {
  float mean[3];
  float direction[3];
  uint32_t idx_start;
  uint32_t idx_end;
  int32_t idx_left;
  int32_t idx_right;
  double dts_mean;
  double dts_covariance;
} kds_kdnode3f;

/* The tree fields of kd_slam2_msgs/msg/KDTree3f (kd_slam2_msgs/msg/KDTree3f.msg; the
 * header and src_topic stay with the caller).  nodes: host memory, num_nodes records. */
typedef struct {
  double ts_start;
  float root_mean[3];
  float root_eigenvalues[3];
  float root_eigenvectors[9]; /* column-major, as in the message */
  int64_t num_nodes;
  kds_kdnode3f* nodes;
} kds_kdtree3f;

/* Replaces TreeLoader_::fromTreeMsg (lib/kd_io/tree_loader_impl_.h:59-70) with the
 * bag reader's KDTree3f -> Tree_ conversion (lib/kd_io/rosbag2_message_reader.cpp:159-191):
 * uploads the node records (one copy of the raw records, unpacked on the device) as a
 * device tree without points.  The nodes must be BFS numbered (children after their
 * parent), as the reference's pruned trees are; otherwise KDS_ERR_BAD_TREE. */
int kds_tree_from_msg(const kds_kdtree3f* msg, kds_tree** out);

/* Replaces toMessage / makeKDTreeMessage (lib/kd_io/slam_messages.h:47-80) and the bag
 * writer's Tree_ -> KDTree3f conversion (lib/kd_io/rosbag2_message_writer.cpp:258-290):
 * fills the tree fields of msg.  On entry msg->num_nodes is the capacity of msg->nodes
 * (may be 0 with nodes NULL to query the count); on return it is the tree's node count,
 * and KDS_ERR_CAPACITY is returned if the records did not fit. */
int kds_tree_to_msg(const kds_tree* t, kds_kdtree3f* msg);

/* Device-to-host copy of the tree (any pointer may be NULL).  leaves: num_leaves node
 * indices (Tree_::_leaves_indices_ptr); perm: num_points input indices in final order. */
int kds_tree_export(const kds_tree* t, float* mean, float* dir, double* dts_mean, double* dts_cov, int64_t* idx_start,
                    int64_t* idx_end, int32_t* left, int32_t* right, int32_t* level, int64_t* leaves, int64_t* perm);

/* Replaces TreeCUDA_::applyVelocitiesInPlace / applyIsometryInPlace
 * (kd/tree/tree_cuda_impl_.h:132-173): per-node morph mean <- R(w dts) mean + v dts,
 * dir <- R dir, or a rigid transform of every node. */
int kds_tree_apply_velocities(kds_tree* t, const float v[6], int32_t skip_leaves, void* stream);
int kds_tree_apply_isometry(kds_tree* t, const float X[12], void* stream);

/* Replaces TreeCUDA_::extractCompressedLeaves (kd/tree/tree_cuda_impl_.h:42-112):
 * writes [mean, dir] per leaf (6 floats), optionally morphed by v (may be NULL). */
int kds_tree_extract_compressed_leaves(const kds_tree* t, const float* v6, float* out, void* stream);
/* The same gather into a device buffer of the caller (num_leaves * 6 floats): no
 * allocation and no copy, asynchronous on `stream` -- a headless stand-in for the
 * viewer's leaf events, where the reference allocates, copies and frees per call
 * (kd/tree/tree_cuda_impl_.h:97-112). */
int kds_tree_extract_compressed_leaves_device(const kds_tree* t, const float* v6, float* out_device, void* stream);

/* Releases the tree's device memory to the stream-ordered pool on the stream it was
 * built on.  As with TreeCUDA_'s destructor, no work using the tree may be pending on
 * other streams. */
void kds_tree_free(kds_tree* t);

/* ------------------------------------------------------------------------------
 * Aligners: ICPB2003D / CTICPB2003D (in place of ICPCUDA3D / CTICPCUDA3D)
 * ------------------------------------------------------------------------------ */

/* TreeAlignerBase_ PARAMs (kd/icp/tree_aligner_base_.h:39-47), CTICP_ velocity_damping
 * (kd/cticp/cticp_.h:61) and ICPTerminationCriteriaScore_ (kd/icp/icp_stats_.h:84-102). */
typedef struct {
  float kernel_threshold;        /* 0.1 */
  float damping;                 /* 1 */
  float max_error;               /* 1 */
  float min_normal_cos;          /* cos(25 deg) */
  int32_t min_good_measurements; /* 10 */
  int32_t max_iterations;        /* 20 */
  float velocity_damping;        /* 100 (CT only) */
  int32_t term_crit;             /* 0: none (nullptr), 1: ICPTerminationCriteriaScore */
  float d_pert;                  /* 1e-3 */
  float d_score;                 /* 1e-3 */
} kds_aligner_params;

void kds_aligner_params_default(kds_aligner_params* p);

/* ICPStats_ (kd/icp/icp_stats_.h:10-21), same field order. */
typedef struct {
  int32_t num_inliers, num_outliers, num_bad, num_err_normal, num_err_fn;
  float chi2, chi2_kernelized, pert_pose_norm, pert_vel_norm;
} kds_stats;

int kds_aligner_create(int32_t type, const kds_aligner_params* p, kds_aligner** out);
int kds_aligner_set_params(kds_aligner* a, const kds_aligner_params* p);
int kds_aligner_set_stream(kds_aligner* a, void* stream);
/* setFixed / setMoving (kd/icp/tree_aligner_base_.h:52-53): non-owning. */
int kds_aligner_set_fixed(kds_aligner* a, const kds_tree* fixed);
int kds_aligner_set_moving(kds_aligner* a, const kds_tree* moving);
/* setX/getX/setFixedX (:87-89), setVelocities/velocities/resetMovingState (:93-95). */
int kds_aligner_set_x(kds_aligner* a, const double X[12]);
int kds_aligner_get_x(const kds_aligner* a, double X[12]);
int kds_aligner_set_fixed_x(kds_aligner* a, const double X[12]);
int kds_aligner_set_velocities(kds_aligner* a, const double v[6]);
int kds_aligner_get_velocities(const kds_aligner* a, double v[6]);
int kds_aligner_set_fixed_velocities(kds_aligner* a, const double v[6]);
int kds_aligner_reset_moving_state(kds_aligner* a);
/* setPosePrior (:127-133); info all-zero disables the prior. */
int kds_aligner_set_pose_prior(kds_aligner* a, const double X_ref[12], const double Z[12], const double info[36]);
/* _fixed_forest / makeFixedEntry (:57-76,136): with entries present, oneRound sums
 * H,b,stats over them (kd/icp/icp_impl_.h:55-71). */
int kds_aligner_add_fixed_entry(kds_aligner* a, const kds_tree* fixed, const double X[12]);
int kds_aligner_clear_fixed_forest(kds_aligner* a);

/* compute (kd/icp/tree_aligner_base_.h:100-115): the whole Gauss-Newton loop runs on
 * the device (one kernel per iteration, one host sync at the end).  *result is the
 * reference's return value: -i on a failed round i, i on early termination, else
 * max_iterations. */
int kds_aligner_compute(kds_aligner* a, int32_t stats_mode, int32_t* result);
/* oneRound (kd/icp/icp_impl_.h:52-90, kd/cticp/cticp_impl_.h:47-92); *ok = 0/1. */
int kds_aligner_one_round(kds_aligner* a, int32_t stats_mode, int32_t* ok);
/* buildQuadraticForm (kd/icp/icp_impl_.h:23-27) and, for CT, buildQuadraticFormDual
 * (kd/cticp/cticp_impl_.h:41-45): H, b and stats at the current state, no update. */
int kds_aligner_build_quadratic_form(kds_aligner* a, int32_t stats_mode);
int kds_aligner_build_quadratic_form_dual(kds_aligner* a, int32_t stats_mode);
/* Public fields H, b, dx (D = 6 for ICP, 12 for CT; row-major D*D). */
int kds_aligner_get_hb(const kds_aligner* a, double* H, double* b, double* dx);
/* H_dual_vel_B, b_dual_vel_B, H_dual_cross_pose_vel_B, H_dual_cross_vel_AB
 * (kd/cticp/cticp_.h:183-186), row-major 6x6 / 6. */
int kds_aligner_get_dual(const kds_aligner* a, double H_vel_B[36], double b_vel_B[6], double H_cross_pose_vel_B[36],
                         double H_cross_vel_AB[36]);
/* getPoseHessian (ICP: H; CT: Schur complement, kd/cticp/cticp_.h:169-177). */
int kds_aligner_get_pose_hessian(const kds_aligner* a, double H6[36]);
int kds_aligner_get_stats(const kds_aligner* a, kds_stats* s);
/* stats_log of the last compute (kd/icp/tree_aligner_base_.h:135). */
int kds_aligner_get_stats_log(const kds_aligner* a, kds_stats* log, int32_t cap, int32_t* n);
/* One linearization at explicit float caches (Xm, Xf, Xmf: 3x 12 floats) and
 * velocities: per-leaf fixed-leaf index (-1 when the descent ends at a pruned child)
 * and status (0 inlier, 1 outlier, 2 bad, 3 err_normal, 4 err_fn), plus H, b, stats.
 * Exposes quadraticTerm's correspondences for parity checks. */
int kds_aligner_linearize_debug(kds_aligner* a, const float caches[36], const float v[6], const float fixed_v[6],
                                int32_t kind, int32_t stats_mode, int32_t* match, int32_t* status, double* H,
                                double* b, kds_stats* stats);
/* Measurement hooks (no reference counterpart).  With profiling on, compute() records a
 * CUDA event pair around every linearization launch on the aligner's stream, inside the
 * graph when one is used; get_profile returns the mean launch duration of the last
 * compute in milliseconds.  count_touched_nodes returns the number of distinct
 * fixed-tree nodes that the descents of the moving leaves visit at the current state
 * (the fixed-tree term of the algorithmic-bytes model). */
int kds_aligner_set_profiling(kds_aligner* a, int32_t on);
int kds_aligner_get_profile(const kds_aligner* a, double* mean_ms, int32_t* launches);
int kds_aligner_count_touched_nodes(kds_aligner* a, int64_t* count);
/* SM-clock stamps of the last profiled linearization launch: [0..3] first block
 * (entry, fixed-tree top staged, tile done, partial published), [8..15] the block that
 * ran the Gauss-Newton step (entry, partials summed, state staged, factorization start,
 * factorized, solved, pose updated, done).  Measurement hook only. */
int kds_phase_stamps(uint64_t out[16]);
/* Diagnostics hook (no reference counterpart): the number of polls of the bounded wait
 * with which each linearization block waits for its TMA copy of the fixed tree's top
 * nodes into shared memory, on the current device (default 1,048,576).  When that wait
 * gives up, the block reads the whole tree from global memory instead -- the results are
 * the same -- and the call returns KDS_ERR_TIMEOUT with its outputs written.  Before
 * exiting, a block waits again (up to 1,048,576 polls, whatever this setting) so that no
 * copy outlives it; if even that wait gives up, the error text says so and the CUDA
 * context should not be used further.  Tests set 0 to exercise the fallback path. */
int kds_set_tma_wait_limit(int32_t polls);
void kds_aligner_free(kds_aligner* a);

/* ------------------------------------------------------------------------------
 * Batched alignment: many independent (moving, fixed) pairs in one launch per
 * Gauss-Newton iteration -- the multi-view bundle-adjustment linearisations
 * (MultiViewICPFactor_::compute, kd/map/multiview_icp_factor_impl_.h:10-62) and
 * whole alignments of uneven sizes.
 * ------------------------------------------------------------------------------ */
enum { KDS_JOB_COMPUTE = 0, KDS_JOB_LINEARIZE = 1, KDS_JOB_LINEARIZE_DUAL = 2 };

typedef struct {
  int32_t type;   /* KDS_ICP / KDS_CTICP */
  int32_t mode;   /* KDS_JOB_* */
  int32_t stats_mode;
  int32_t pad_;
  const kds_tree* fixed;
  const kds_tree* moving;
  kds_aligner_params params;
  double X[12];        /* in: initial guess; out: estimate */
  double fixed_X[12];
  double v[6];         /* in/out (CT) */
  double fixed_v[6];
  /* outputs */
  int32_t result;
  int32_t iterations;
  kds_stats stats;
  double H[144];       /* D*D, D = 6 or 12 */
  double b[12];
  double H_vel_B[36], b_vel_B[6], H_cross_pose_vel_B[36], H_cross_vel_AB[36]; /* dual */
} kds_job;

typedef struct kds_batch kds_batch;
int kds_batch_create(kds_batch** out);
/* Runs all jobs; with use_graph != 0, a job-set shape that runs a second time in a
 * row is captured into a CUDA graph, which is replayed while the shape stays. */
int kds_batch_run(kds_batch* b, kds_job* jobs, int32_t num_jobs, int32_t use_graph, void* stream);
/* Launch-shape autotuner for a job set (no reference counterpart): times the batched
 * launches for each candidate configuration -- tree-top nodes staged in shared memory
 * per block (0, 1023, 2047) x tiles of the larger jobs first or in job order x the
 * form: (0) one linearization launch per iteration and kind (graph-captured), one tile
 * of 128 moving surfels per block; (1) one persistent launch that runs every iteration
 * of every job from a device work queue; (2) as (0) with two tiles of a job per block,
 * each thread keeping two descents in flight -- keeps the fastest in the batch handle
 * for the following kds_batch_run calls, and reports its index (config = stage index +
 * 3 * order + 6 * form) and the mean milliseconds of all eighteen (ms_out: 18 doubles,
 * may be NULL).  The jobs are read, not modified; results do not depend on the
 * configuration. */
int kds_batch_autotune(kds_batch* b, kds_job* jobs, int32_t num_jobs, void* stream, int32_t* chosen,
                       double* ms_out);
/* Sets the batch's launch configuration directly (an index as kds_batch_autotune reports
 * it, 0..17); KDS_ERR_INVALID_ARG otherwise. */
int kds_batch_configure(kds_batch* b, int32_t config);

/* One multi-view bundle-adjustment factor over a job of the last kds_batch_run.
 * ICP (a KDS_ICP job): var[0] = fixed pose, var[1] = moving pose (MultiViewICPFactor_).
 * CT-ICP (a KDS_CTICP job run as KDS_JOB_LINEARIZE_DUAL): var = pose_A, vel_A, pose_B,
 * vel_B (MultiViewCTICPFactor_).  Variables are 6-dimensional, numbered by the caller. */
typedef struct {
  int32_t job;
  int32_t var[4];
} kds_factor;

/* Replaces the block updates of MultiViewICPFactor_::compute and
 * MultiViewCTICPFactor_::compute (kd/map/multiview_icp_factor_impl_.h:30-62,
 * kd/map/multiview_cticp_factor_impl_.h:33-83) for all factors at once, on the device,
 * from the H, b of the last kds_batch_run: a factor counts when
 * inlierRatio() > disable_inlier_ratio (enabled[f], may be NULL); the sum of the counted
 * factors' blocks is returned as the upper block triangle (row variable <= column
 * variable): block k is variables (block_rc[2k], block_rc[2k+1]), 36 doubles row-major
 * in H_blocks, sorted by (row, column); b: 6 doubles per variable (may be NULL).
 * Contributions are summed in FP64 in factor order.  On entry *num_blocks is the
 * capacity (0 with NULL block_rc / H_blocks queries the count); on return the count,
 * with KDS_ERR_CAPACITY if the blocks did not fit. */
int kds_batch_assemble(kds_batch* b, const kds_factor* factors, int32_t num_factors, int32_t num_vars,
                       float disable_inlier_ratio, void* stream, int32_t* num_blocks, int32_t* block_rc,
                       double* H_blocks, double* b_vec, int32_t* enabled);
void kds_batch_free(kds_batch* b);

/* ------------------------------------------------------------------------------
 * Tracker step: the odometry of TrackerProc_::addFrame
 * (kd/tracker/tracker_proc_frame_impl_.h:33-115) with its motion model
 * (ZeroVelMotionModel_ / ConstVelMotionModel_, kd/motion_model/zero_vel_motion_model_.h,
 * kd/motion_model/const_vel_motion_model_.h) and the keyframe switch of
 * SLAMProc_::addFrame / addKeyframe (kd/slam/slam_proc_frame_impl_.h:8-49, 73-138) with
 * relocalisation, loop search and the pose graph left out: a frame that fails
 * shouldSwitchKeyframe (kd/tracker/tracker_proc_frame_impl_.h:118-123) becomes the
 * keyframe.  Each step morphs the frame tree by the predicted velocity
 * (Frame::applyVelocity, kd/map/map_.h:103-110), aligns it to the keyframe tree from
 * pose_in_kf * prediction, updates the motion model with the relative motion and, for
 * CT-ICP, morphs the tree again by the estimated residual velocities.
 * ------------------------------------------------------------------------------ */
typedef struct kds_tracker kds_tracker;

enum { KDS_MOTION_ZERO_VEL = 0, KDS_MOTION_CONST_VEL = 1 };
/* KDStatus (kd/map/map_common.h:74-83): values the tracker reports. */
enum { KDS_STATUS_INIT = 0, KDS_STATUS_TRACKING = 1 };

typedef struct {
  int32_t aligner_type;       /* odom_aligner: KDS_ICP / KDS_CTICP (KDS_CTICP) */
  kds_aligner_params aligner; /* its PARAMs (kds_aligner_params_default; CT damping 100) */
  int32_t motion_model;       /* KDS_MOTION_ZERO_VEL (the reference's default) / KDS_MOTION_CONST_VEL */
  float motion_model_alpha;   /* ConstVelMotionModel_ low-pass factor (0.9) */
  float min_inlier_frac;      /* TrackerProc_ PARAMs (kd/tracker/tracker_proc_.h:55-57): 0.6 */
  float max_kf_trans;         /* 3.0 m */
  float max_kf_rot_deg;       /* 360 deg */
} kds_tracker_params;

void kds_tracker_params_default(kds_tracker_params* p);

typedef struct {
  int32_t status;            /* KDS_STATUS_INIT on the first frame, else KDS_STATUS_TRACKING */
  int32_t result;            /* the aligner's compute() return (-1 on the first frame) */
  int32_t new_keyframe;      /* 1 when this frame became the keyframe */
  int32_t frame_idx;         /* _frame_idx before the step */
  int32_t keyframe_count;    /* keyframes made so far, this one included */
  int32_t pad_;
  double frame_duration;     /* ts - previous ts (0 on the first frame) */
  double pose_in_kf[12];     /* after the step, before a keyframe switch resets it */
  double pose_in_world[12];  /* the frame's pose_in_world */
  double velocity[6];        /* velocity applied before the alignment (velocityLog / frame_duration) */
  double ct_velocity[6];     /* CT-ICP: the residual velocities applied after it (else 0) */
  kds_stats stats;           /* the aligner's stats (zero on the first frame) */
} kds_tracker_result;

/* Creates a tracker with its own aligner.  All work runs on `stream` (NULL: the
 * calling thread's default stream). */
int kds_tracker_create(const kds_tracker_params* p, void* stream, kds_tracker** out);
/* One addFrame.  The frame tree is transformed in place, by T_base_lidar first when it
 * is not NULL (TrackerProc_::makeFrame, tracker_proc_frame_impl_.h:15-16), then by the
 * velocity morphs, as the reference's frame tree is.  A frame that becomes the
 * keyframe is copied into the tracker, so the caller keeps ownership of every tree it
 * passes.  A non-finite aligned pose returns KDS_ERR_DIVERGED and leaves the tracker's
 * pose and motion model as they were before the step (the reference throws).  The call
 * returns with its device work done (the morphed tree and the keyframe copy are final). */
int kds_tracker_add_frame(kds_tracker* t, kds_tree* frame, double ts, const double T_base_lidar[12],
                          kds_tracker_result* out);
/* The same step for n independent trackers at once (many sensor streams, no reference
 * counterpart): every tracker's morphs and keyframe copies run on `stream`, and the n
 * alignments run as one batch (kds_batch_run, COMPUTE jobs, graph-captured when the job
 * set's shape repeats) instead of n aligner calls.  Each tracker's result is what
 * kds_tracker_add_frame gives it.  codes[i] (may be NULL) is KDS_OK or that tracker's
 * error (KDS_ERR_DIVERGED leaves only that tracker as it was); the return value is
 * KDS_OK or the first error.  The trackers must be distinct, and their own streams idle. */
int kds_tracker_add_frames(kds_tracker* const* trackers, kds_tree* const* frames, const double* ts,
                           const double* T_base_lidar, int32_t n, kds_batch* batch, void* stream,
                           kds_tracker_result* out, int32_t* codes);
/* Pose of the last frame in the world (TrackerProc_::poseGlobal) and relative to its keyframe. */
int kds_tracker_get_pose(const kds_tracker* t, double pose_global[12], double pose_in_kf[12]);
/* The keyframe tree the next frame is aligned to (owned by the tracker; NULL before the first frame). */
int kds_tracker_get_keyframe(const kds_tracker* t, const kds_tree** kf, double pose_in_world[12]);
/* Checkpoint / resume of a tracker (no reference counterpart: the reference saves its map
 * as a bag of keyframe trees plus the factor graph, lib/kd_io/kd_map_io_.h:19-186).  The
 * state is plain data; the keyframe travels separately as a tree (kds_tree_to_msg /
 * kds_tree_from_msg carry everything the alignment reads).  A tracker restored with
 * set_state and that keyframe continues exactly as the saved one would. */
typedef struct {
  kds_tracker_params params;
  double last_ts, frame_duration;   /* ZeroVelMotionModel_ state */
  double T_delta_log[6];            /* ConstVelMotionModel_ state */
  double kf_pose_in_world[12], pose_in_kf[12], pose_global[12];
  int32_t frame_idx, keyframe_count;
  int32_t has_keyframe, pad_;
} kds_tracker_state;
int kds_tracker_get_state(const kds_tracker* t, kds_tracker_state* st);
/* keyframe: required when st->has_keyframe (copied into the tracker).  st->params must
 * match the tracker's aligner type, motion model and every aligner parameter (compared
 * field by field); otherwise the call changes nothing and returns KDS_ERR_INVALID_ARG
 * naming the first field that differs.  The motion model's alpha and the keyframe
 * thresholds are taken from the state. */
int kds_tracker_set_state(kds_tracker* t, const kds_tracker_state* st, const kds_tree* keyframe);
/* Motion model reset (ZeroVelMotionModel_::reset / ConstVelMotionModel_::reset), keyframe dropped. */
int kds_tracker_reset(kds_tracker* t);
void kds_tracker_free(kds_tracker* t);

/* ------------------------------------------------------------------------------
 * Served registration (no reference counterpart: the reference runs one tracker
 * thread with one aligner per role, kd/tracker/tracker_proc_.h:82).  Many sensor
 * streams submit scan-to-map ICP / CT-ICP registrations; each stream's local surfel
 * map stays on the device and is rebuilt from the stream's last map_every
 * registered scans (world frame, deskewed with the estimated velocities); requests
 * are admitted by device memory and run with continuous batching.  Every
 * registration computes exactly what kds_tree_build + kds_aligner_compute compute
 * (CT: TreeAlignerBase_::compute, kd/icp/tree_aligner_base_.h:100-115).
 * ------------------------------------------------------------------------------ */
typedef struct kds_server kds_server;

typedef struct {
  int32_t max_slots;        /* registrations on the device at once (512) */
  int32_t map_every;        /* map rebuilt from the last map_every scans of a stream (5) */
  int32_t max_build_trees;  /* trees per build pass (128) */
  int32_t serial;           /* 1: plain drop-in, one request at a time via the per-call API (0) */
  int32_t profile;          /* 1: time the linearization launches of every tick and count the
                               fixed nodes each registration touches (0; adds work) */
  int32_t max_tiles;        /* tile arena per aligner kind, 128 moving surfels per tile (32768) */
  int32_t iters_per_tick;   /* Gauss-Newton iterations queued per tick (3) */
  int64_t hbm_cap;          /* admission cap in bytes; 0: 90% of the free memory at create */
  int64_t max_build_points; /* points per build pass (16 Mi) */
  kds_tree_params tree;     /* scans and maps */
  kds_aligner_params icp;   /* KDS_ICP requests */
  kds_aligner_params ct;    /* KDS_CTICP requests */
  int32_t build_threads;    /* build threads, each with its own stream: 1 or 2 (1).  With 2, one
                               builds the map rebuilds and the requests whose map is installed,
                               the other the requests whose map is not there yet (while the
                               reservations stay under a quarter of the cap): typical steps
                               are shorter, but while the two passes overlap some steps
                               stall for tens to hundreds of milliseconds */
  int32_t pad_;
} kds_server_params;

typedef struct {
  int32_t stream;        /* from kds_server_add_stream */
  int32_t type;          /* KDS_ICP / KDS_CTICP */
  int64_t n;             /* points */
  const float* xyz;      /* n*3, host or device memory; must stay valid until the request has finished */
  const double* stamps;  /* n, host or device memory, or NULL */
  double X0[12];         /* initial guess (3x4 row-major) */
  double v0[6];          /* initial velocities (CT) */
  double arrival;        /* seconds after kds_server_start at which the request arrives */
} kds_request;

typedef struct {
  int32_t status;        /* KDS_OK, KDS_ERR_TREE_REJECTED, KDS_ERR_ADMISSION */
  int32_t result;        /* compute()'s return value */
  int32_t iterations;
  int32_t map_version;
  kds_stats stats;
  double X[12];
  double v[6];
  double t_arrival, t_admit, t_built, t_done; /* seconds after kds_server_start */
} kds_result;

typedef struct {
  int64_t submitted, completed, ticks, build_passes, map_builds, built_trees;
  int64_t hbm_cap, peak_reserved;
  double mean_active;      /* registrations per tick */
  double lin_ms;           /* device time of the linearization launches (profile = 1) */
  int64_t lin_ticks;       /* ticks timed */
  int64_t leaf_iterations; /* moving surfels linearized, summed over ticks */
  double alg_bytes;        /* profile = 1: algorithmic bytes of the linearizations (32 B per moving
                              surfel + 32 B per distinct fixed node touched + tile partials, per iteration) */
  int64_t h2d_bytes;       /* request points copied from host memory */
  int64_t d2h_bytes;       /* results read back to the host */
  double build_ms;         /* wall time of the tree-build passes (requests and map rebuilds) */
  int64_t build_points;    /* points those passes built */
  double build_point_levels; /* sum over the passes of points x levels */
  double build_global_point_levels; /* sum over the passes of points x levels built level by level
                                       (the levels below ran in shared-memory subtrees) */
  double build_busy_ms;     /* wall time during which at least one build pass ran (passes of the
                               two build threads overlap) */
  int64_t build_released_ahead; /* trees built ahead of their map and released to make room
                                   under the cap (rebuilt later; two build threads only) */
} kds_server_stats;

void kds_server_params_default(kds_server_params* p);
int kds_server_create(const kds_server_params* p, kds_server** out);
/* Adds a stream with its initial map (world-frame points, host) before start;
 * max_scan_points bounds the scans it will submit. */
int kds_server_add_stream(kds_server* s, const float* map_xyz, int64_t n, int64_t max_scan_points,
                          int32_t* stream_id);
/* Queues a request (arrivals non-decreasing); the ticket identifies its result. */
int kds_server_submit(kds_server* s, const kds_request* r, int64_t* ticket);
int kds_server_start(kds_server* s);
/* Waits for every submitted request (timeout_s <= 0: no limit). */
int kds_server_drain(kds_server* s, double timeout_s);
int kds_server_wait(kds_server* s, int64_t ticket, double timeout_s, kds_result* out);
int kds_server_get_stats(kds_server* s, kds_server_stats* st);
/* Timeline of the served loop for diagnosis: rows of 4 doubles (kind, count, begin,
 * end); kind 0 = a tree-build pass (count = points), kind 1 = a Gauss-Newton tick from
 * its launch to the host reading its results (count = registrations in the tick);
 * times in seconds after kds_server_start.  *n = rows recorded (may exceed cap). */
int kds_server_get_trace(kds_server* s, double* rows4, int32_t cap, int32_t* n);
void kds_server_free(kds_server* s);

/* One linearization that allocates no memory.  This entry point has no counterpart in
 * the reference; it serves callers that cannot allocate device memory while they run
 * (real-time loops that reserve all memory at start-up, code that must not call
 * cudaMalloc/cudaFree because those can block on the device or on allocator locks).
 *
 * It computes what kds_aligner_build_quadratic_form computes for a single fixed tree
 * (D = 6 for KDS_ICP, 12 for KDS_CTICP): H (row-major D*D), b (D) and stats at pose X,
 * velocities v (CT only, NULL = zero), fixed pose fixed_X and fixed velocities fixed_v
 * (NULL = zero).  Its scratch (about 0.8 MB) is one static device array of the library,
 * held by every GPU that loads the library until the process exits; the trees and the
 * outputs are the caller's.  At most 65,536 moving leaves per call: larger moving trees
 * return KDS_ERR_CAPACITY.
 *
 * The first call on each device resolves the array's address and sets kernel
 * attributes; make that first call before any stream capture.  All calls share the
 * array, so calls that overlap on the GPU (other streams, other threads) race on it.
 * The call blocks until its results have reached the host.  H, b, stats may be NULL.
 * The call has its own error slot inside the array (read back with the outputs in one
 * copy on `stream`), so it never reports another call's device error.  On
 * KDS_ERR_TIMEOUT (kds_set_tma_wait_limit) H, b and stats are written and valid. */
int kds_linearize_static(const kds_tree* fixed, const kds_tree* moving, int32_t type,
                         const kds_aligner_params* params, const double X[12], const double fixed_X[12],
                         const double v[6], const double fixed_v[6], int32_t stats_mode, void* stream, double* H,
                         double* b, kds_stats* stats);

#ifdef __cplusplus
}
#endif
#endif /* KDS_H */
