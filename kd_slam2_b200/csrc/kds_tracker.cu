// Tracker step: TrackerProc_::addFrame (kd/tracker/tracker_proc_frame_impl_.h:33-115)
// with ZeroVelMotionModel_ / ConstVelMotionModel_ (kd/motion_model/) and the keyframe
// switch of SLAMProc_ (kd/slam/slam_proc_frame_impl_.h:8-49, 73-138) without
// relocalisation, loop search or the pose graph.
//
// One step is host bookkeeping around three device operations of this library:
//   1. the pre-deskew morph of the frame tree by velocityLog / frame_duration
//      (Frame::applyVelocity, kd/map/map_.h:103-110) -- one k_apply_velocities launch
//      plus the leaf gather;
//   2. the alignment of the frame to the keyframe tree from pose_in_kf * prediction
//      (alignFrames, kd/map/map_align_utils_.h:10-31) -- the aligner's graph-captured
//      Gauss-Newton loop;
//   3. for CT-ICP, the morph by the estimated residual velocities.
// A keyframe switch copies the (deskewed) frame tree on the device.  The motion-model
// and pose arithmetic is FP64 on the host, as the aligner's pose math is.
#include <cmath>
#include <cstring>
#include <vector>

#include "kds_internal.cuh"

using namespace kds;

namespace {

// 3x4 row-major isometries [R | t] in double.
struct Iso {
  double m[12];
};

Iso iso_identity() {
  Iso X;
  for (int i = 0; i < 12; ++i) X.m[i] = 0.0;
  X.m[0] = X.m[5] = X.m[10] = 1.0;
  return X;
}

// A * B: R = Ra Rb, t = Ra tb + ta (each row summed left to right)
Iso iso_mul(const Iso& A, const Iso& B) {
  Iso C;
  for (int r = 0; r < 3; ++r) {
    const double* a = A.m + 4 * r;
    for (int c = 0; c < 4; ++c) {
      double s = a[0] * B.m[c] + a[1] * B.m[4 + c] + a[2] * B.m[8 + c];
      C.m[4 * r + c] = (c == 3) ? s + a[3] : s;
    }
  }
  return C;
}

// [R^T | -R^T t]
Iso iso_inv(const Iso& A) {
  Iso C;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) C.m[4 * r + c] = A.m[4 * c + r];
  for (int r = 0; r < 3; ++r)
    C.m[4 * r + 3] = -(C.m[4 * r] * A.m[3] + C.m[4 * r + 1] * A.m[7] + C.m[4 * r + 2] * A.m[11]);
  return C;
}

// rodrigues(w) (kd/utils/geometry_3d_impl_.h:37-46): identity below 1e-9, else
// I + sin(a) S + (1 - cos(a)) S^2 with S = skew(w / a), evaluated element-wise.
void rodrigues(const double* w, double* R) {
  const double angle = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1.0 : 0.0;
  if (angle < 1e-9) return;
  const double inv = 1.0 / angle;
  const double n[3] = {w[0] * inv, w[1] * inv, w[2] * inv};
  const double S[9] = {0.0, -n[2], n[1], n[2], 0.0, -n[0], -n[1], n[0], 0.0};
  double S2[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) S2[3 * i + j] = S[3 * i] * S[j] + S[3 * i + 1] * S[3 + j] + S[3 * i + 2] * S[6 + j];
  const double s = std::sin(angle), omc = 1.0 - std::cos(angle);
  for (int i = 0; i < 9; ++i) R[i] = (R[i] + s * S[i]) + omc * S2[i];
}

// expmap (geometry_3d_impl_.h:176-184): t = v[0:3], R = rodrigues(v[3:6])
Iso expmap(const double* v) {
  Iso X;
  double R[9];
  rodrigues(v + 3, R);
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) X.m[4 * r + c] = R[3 * r + c];
    X.m[4 * r + 3] = v[r];
  }
  return X;
}

// logmap = [t, logSO3(R)] (geometry_3d_impl_.h:48-59, 186-192)
void logmap(const Iso& X, double* v) {
  const double* m = X.m;
  double cos_a = 0.5 * (((m[0] + m[5]) + m[10]) - 1.0);
  cos_a = std::max(-1.0, std::min(1.0, cos_a));
  const double angle = std::acos(cos_a);
  const double ax[3] = {m[9] - m[6], m[2] - m[8], m[4] - m[1]};
  const double f = angle < 1e-7 ? 0.5 : angle / (2.0 * std::sin(angle));
  for (int i = 0; i < 3; ++i) {
    v[i] = m[4 * i + 3];
    v[3 + i] = ax[i] * f;
  }
}

// GeometryTraits_<3>::getAngle = Eigen::AngleAxis(R).angle() (kd/utils/geometry_3d_.h:83-85):
// the rotation's unit quaternion by Shepperd's method (branch on the trace, else on
// the largest diagonal entry), then 2 atan2(|q.xyz|, |q.w|), in [0, pi].
double rotation_angle(const Iso& X) {
  const double* m = X.m;
  auto M = [&](int i, int j) { return m[4 * i + j]; };
  double q[4];  // x, y, z, w
  const double tr = (M(0, 0) + M(1, 1)) + M(2, 2);
  if (tr > 0.0) {
    double t = std::sqrt(tr + 1.0);
    q[3] = 0.5 * t;
    t = 0.5 / t;
    q[0] = (M(2, 1) - M(1, 2)) * t;
    q[1] = (M(0, 2) - M(2, 0)) * t;
    q[2] = (M(1, 0) - M(0, 1)) * t;
  } else {
    int i = 0;
    if (M(1, 1) > M(0, 0)) i = 1;
    if (M(2, 2) > M(i, i)) i = 2;
    const int j = (i + 1) % 3, k = (j + 1) % 3;
    double t = std::sqrt(((M(i, i) - M(j, j)) - M(k, k)) + 1.0);
    q[i] = 0.5 * t;
    t = 0.5 / t;
    q[3] = (M(k, j) - M(j, k)) * t;
    q[j] = (M(j, i) + M(i, j)) * t;
    q[k] = (M(k, i) + M(i, k)) * t;
  }
  const double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
  if (n == 0.0) return 0.0;
  return 2.0 * std::atan2(n, std::fabs(q[3]));
}

bool iso_finite(const Iso& X) {
  for (double x : X.m)
    if (!std::isfinite(x)) return false;
  return true;
}

}  // namespace

struct kds_tracker {
  kds_tracker_params P;
  cudaStream_t stream = nullptr;
  kds_aligner* aligner = nullptr;
  kds_tree* keyframe = nullptr;  // device copy owned by the tracker
  Iso kf_pose_in_world = iso_identity();
  Iso pose_in_kf = iso_identity();
  Iso pose_global = iso_identity();  // the last frame's pose_in_world
  // ZeroVelMotionModel_ state (zero_vel_motion_model_.h:23-35) and ConstVel's _T_delta_log
  double last_ts = -1.0;
  double frame_duration = 0.0;
  double T_delta_log[6] = {0, 0, 0, 0, 0, 0};
  int32_t frame_idx = 0;
  int32_t keyframe_count = 0;
};

namespace {

void motion_reset(kds_tracker* t) {
  t->last_ts = -1.0;
  t->frame_duration = 0.0;
  for (double& x : t->T_delta_log) x = 0.0;
}

// doPredict (zero_vel_motion_model_.h:23-30)
void motion_predict(kds_tracker* t, double ts) {
  t->frame_duration = t->last_ts < 0 ? 0.0 : ts - t->last_ts;
  t->last_ts = ts;
}

// velocityLog(): ConstVel's filtered log of the per-frame motion, zero for ZeroVel
void velocity_log(const kds_tracker* t, double* v) {
  for (int i = 0; i < 6; ++i) v[i] = t->P.motion_model == KDS_MOTION_CONST_VEL ? t->T_delta_log[i] : 0.0;
}

// prediction(): expmap(_T_delta_log) for ConstVel, identity for ZeroVel
Iso motion_prediction(const kds_tracker* t) {
  if (t->P.motion_model != KDS_MOTION_CONST_VEL) return iso_identity();
  return expmap(t->T_delta_log);
}

// ConstVelMotionModel_::doUpdate (const_vel_motion_model_.h:24-31):
// T_delta_log = alpha T_delta_log + (1 - alpha) logmap(delta)
void motion_update(kds_tracker* t, const Iso& delta) {
  if (t->P.motion_model != KDS_MOTION_CONST_VEL) return;
  const double alpha = (double)t->P.motion_model_alpha;
  double dv[6];
  logmap(delta, dv);
  for (int i = 0; i < 6; ++i) t->T_delta_log[i] = alpha * t->T_delta_log[i] + (1.0 - alpha) * dv[i];
}

// Frame::applyVelocity: morph only when the velocity is not zero
int apply_velocity(kds_tree* tree, const double* v, cudaStream_t s) {
  bool zero = true;
  for (int i = 0; i < 6; ++i) zero = zero && v[i] == 0.0;
  if (zero) return KDS_OK;
  float vf[6];
  for (int i = 0; i < 6; ++i) vf[i] = (float)v[i];
  return tree_apply_velocities(tree, vf, 0, s);
}

// TrackerProc_::shouldSwitchKeyframe (tracker_proc_frame_impl_.h:118-123); inlierRatio()
// in float as ICPStats_ computes it (kd/icp/icp_stats_.h:28-31)
bool should_switch(const kds_tracker* t, const Iso& X, const kds_stats& st) {
  const int leaves = st.num_inliers + st.num_outliers + st.num_bad + st.num_err_normal + st.num_err_fn;
  const float ratio = leaves ? (float)st.num_inliers / (float)leaves : 0.f;
  const double tn = std::sqrt(X.m[3] * X.m[3] + X.m[7] * X.m[7] + X.m[11] * X.m[11]);
  const float max_rot_rad = t->P.max_kf_rot_deg * float(M_PI / 180.);
  return ratio < t->P.min_inlier_frac || tn > (double)t->P.max_kf_trans ||
         std::fabs(rotation_angle(X)) > (double)max_rot_rad;
}

// SLAMProc_::addKeyframe (slam_proc_frame_impl_.h:73-138), tracker part: the frame
// becomes the keyframe; ZeroVel/ConstVel onKeyframe and onOriginReset are no-ops.
int make_keyframe(kds_tracker* t, const kds_tree* frame, const Iso& pose_in_world, cudaStream_t s) {
  kds_tree* copy = nullptr;
  int rc = tree_clone(frame, s, &copy);
  if (rc != KDS_OK) return rc;
  if (t->keyframe) {
    tree_release(t->keyframe->d);
    delete t->keyframe;
  }
  t->keyframe = copy;
  t->kf_pose_in_world = pose_in_world;
  t->pose_in_kf = iso_identity();
  ++t->keyframe_count;
  return KDS_OK;
}

// What a step must restore when it fails.
struct Saved {
  Iso pose_in_kf_prev;
  double last_ts, frame_duration;
};

int restore(kds_tracker* t, const Saved& sv, int code) {
  t->last_ts = sv.last_ts;
  t->frame_duration = sv.frame_duration;
  return code;
}

// The step up to the alignment: makeFrame's T_base_lidar, doPredict, the pre-deskew
// morph, and the first frame (which becomes the keyframe: *done = true).  Otherwise
// *X0 = pose_in_kf * prediction for the alignment.
int pre_step(kds_tracker* t, kds_tree* frame, double ts, const double* T_base_lidar, cudaStream_t s,
             kds_tracker_result* out, Saved* sv, bool* done, Iso* X0) {
  *done = false;
  if (!std::isfinite(ts)) { set_error("kds_tracker_add_frame: timestamp is not finite"); return KDS_ERR_INVALID_ARG; }
  memset(out, 0, sizeof(*out));
  out->result = -1;
  out->frame_idx = t->frame_idx;
  int rc = KDS_OK;
  if (T_base_lidar) {
    float Xf[12];
    for (int i = 0; i < 12; ++i) Xf[i] = (float)T_base_lidar[i];
    if ((rc = tree_apply_isometry(frame, Xf, s)) != KDS_OK) return rc;
  }
  sv->pose_in_kf_prev = t->pose_in_kf;
  sv->last_ts = t->last_ts;
  sv->frame_duration = t->frame_duration;
  motion_predict(t, ts);
  out->frame_duration = t->frame_duration;
  double vel[6] = {0, 0, 0, 0, 0, 0};
  if (t->frame_duration > 0) {
    double vl[6];
    velocity_log(t, vl);
    for (int i = 0; i < 6; ++i) vel[i] = vl[i] / t->frame_duration;
    if ((rc = apply_velocity(frame, vel, s)) != KDS_OK) return restore(t, *sv, rc);
  }
  memcpy(out->velocity, vel, sizeof(vel));
  if (!t->keyframe) {
    // first frame: Init, and SLAMProc_ makes it the keyframe at the origin
    const Iso I = iso_identity();
    if ((rc = make_keyframe(t, frame, I, s)) != KDS_OK) return restore(t, *sv, rc);
    t->pose_global = I;
    out->status = KDS_STATUS_INIT;
    out->new_keyframe = 1;
    out->keyframe_count = t->keyframe_count;
    memcpy(out->pose_in_kf, I.m, sizeof(I.m));
    memcpy(out->pose_in_world, I.m, sizeof(I.m));
    ++t->frame_idx;
    *done = true;
    return KDS_OK;
  }
  *X0 = iso_mul(t->pose_in_kf, motion_prediction(t));
  return KDS_OK;
}

// The step after the alignment (X, stats, result, CT velocities cv): the divergence
// check, doUpdate, the CT morph and the keyframe test.
int post_step(kds_tracker* t, kds_tree* frame, const Iso& X, const kds_stats& st, int32_t result, const double* cv,
              cudaStream_t s, const Saved& sv, kds_tracker_result* out) {
  out->result = result;
  out->stats = st;
  if (!iso_finite(X)) {
    set_error("kds_tracker_add_frame: solver diverged at frame %d", t->frame_idx);
    return restore(t, sv, KDS_ERR_DIVERGED);
  }
  t->pose_in_kf = X;
  const Iso pose_in_world = iso_mul(t->kf_pose_in_world, X);
  motion_update(t, iso_mul(iso_inv(sv.pose_in_kf_prev), X));
  int rc = KDS_OK;
  if (t->P.aligner_type == KDS_CTICP) {
    if ((rc = apply_velocity(frame, cv, s)) != KDS_OK) return rc;
    memcpy(out->ct_velocity, cv, sizeof(double) * 6);
  }
  t->pose_global = pose_in_world;
  out->status = KDS_STATUS_TRACKING;
  memcpy(out->pose_in_kf, X.m, sizeof(X.m));
  memcpy(out->pose_in_world, pose_in_world.m, sizeof(X.m));
  if (should_switch(t, X, st)) {
    if ((rc = make_keyframe(t, frame, pose_in_world, s)) != KDS_OK) return rc;
    out->new_keyframe = 1;
  }
  out->keyframe_count = t->keyframe_count;
  ++t->frame_idx;
  return KDS_OK;
}

// A step returns with its device work done: the frame tree's morphs and the keyframe
// copy are final when the call returns, whichever stream the caller uses next.
int finish(cudaStream_t s, int rc) {
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess && rc == KDS_OK) return cuda_status(e, "tracker step", __FILE__, __LINE__);
  return rc;
}

}  // namespace

extern "C" {

void kds_tracker_params_default(kds_tracker_params* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->aligner_type = KDS_CTICP;
  kds_aligner_params_default(&p->aligner);
  p->motion_model = KDS_MOTION_ZERO_VEL;
  p->motion_model_alpha = 0.9f;
  p->min_inlier_frac = 0.6f;
  p->max_kf_trans = 3.0f;
  p->max_kf_rot_deg = 360.f;
}

int kds_tracker_create(const kds_tracker_params* p, void* stream, kds_tracker** out) {
  if (!p || !out) { set_error("kds_tracker_create: NULL argument"); return KDS_ERR_INVALID_ARG; }
  *out = nullptr;
  if ((p->aligner_type != KDS_ICP && p->aligner_type != KDS_CTICP) ||
      (p->motion_model != KDS_MOTION_ZERO_VEL && p->motion_model != KDS_MOTION_CONST_VEL) ||
      !(p->motion_model_alpha >= 0.f && p->motion_model_alpha <= 1.f)) {
    set_error("kds_tracker_create: aligner_type, motion_model or motion_model_alpha out of range");
    return KDS_ERR_INVALID_ARG;
  }
  kds_tracker* t = new kds_tracker();
  t->P = *p;
  t->stream = as_stream(stream);
  int rc = kds_aligner_create(p->aligner_type, &p->aligner, &t->aligner);
  if (rc == KDS_OK) rc = kds_aligner_set_stream(t->aligner, t->stream);
  if (rc != KDS_OK) {
    if (t->aligner) kds_aligner_free(t->aligner);
    delete t;
    return rc;
  }
  *out = t;
  return KDS_OK;
}

int kds_tracker_add_frame(kds_tracker* t, kds_tree* frame, double ts, const double T_base_lidar[12],
                          kds_tracker_result* out) {
  if (!t || !frame || !out) { set_error("kds_tracker_add_frame: NULL argument"); return KDS_ERR_INVALID_ARG; }
  Saved sv;
  bool done = false;
  Iso X0;
  int rc = pre_step(t, frame, ts, T_base_lidar, t->stream, out, &sv, &done, &X0);
  if (rc != KDS_OK || done) return finish(t->stream, rc);
  // alignFrames: fixed = keyframe, moving = frame, fixed X = I, X = X0, zero velocities
  const Iso I = iso_identity();
  const double zero6[6] = {0, 0, 0, 0, 0, 0};
  int32_t result = 0;
  if ((rc = kds_aligner_set_fixed(t->aligner, t->keyframe)) != KDS_OK ||
      (rc = kds_aligner_set_moving(t->aligner, frame)) != KDS_OK ||
      (rc = kds_aligner_set_fixed_x(t->aligner, I.m)) != KDS_OK ||
      (rc = kds_aligner_set_x(t->aligner, X0.m)) != KDS_OK ||
      (rc = kds_aligner_set_velocities(t->aligner, zero6)) != KDS_OK ||
      (rc = kds_aligner_compute(t->aligner, 0, &result)) != KDS_OK)
    return restore(t, sv, rc);
  Iso X;
  kds_stats st;
  double cv[6] = {0, 0, 0, 0, 0, 0};
  kds_aligner_get_x(t->aligner, X.m);
  kds_aligner_get_stats(t->aligner, &st);
  if (t->P.aligner_type == KDS_CTICP) kds_aligner_get_velocities(t->aligner, cv);
  rc = post_step(t, frame, X, st, result, cv, t->stream, sv, out);
  return finish(t->stream, rc);
}

int kds_tracker_add_frames(kds_tracker* const* trackers, kds_tree* const* frames, const double* ts,
                           const double* T_base_lidar, int32_t n, kds_batch* batch, void* stream,
                           kds_tracker_result* out, int32_t* codes) {
  if (n < 0 || (n > 0 && (!trackers || !frames || !ts || !batch || !out))) {
    set_error("kds_tracker_add_frames: NULL argument or negative count");
    return KDS_ERR_INVALID_ARG;
  }
  if (n == 0) return KDS_OK;
  for (int32_t i = 0; i < n; ++i) {
    if (!trackers[i] || !frames[i]) { set_error("kds_tracker_add_frames: NULL tracker or frame %d", i); return KDS_ERR_INVALID_ARG; }
    for (int32_t j = 0; j < i; ++j)
      if (trackers[j] == trackers[i]) { set_error("kds_tracker_add_frames: tracker %d repeated", i); return KDS_ERR_INVALID_ARG; }
  }
  cudaStream_t s = as_stream(stream);
  std::vector<Saved> sv((size_t)n);
  std::vector<int32_t> rcs((size_t)n, KDS_OK), job_of((size_t)n, -1);
  std::vector<kds_job> jobs;
  jobs.reserve((size_t)n);
  const Iso I = iso_identity();
  for (int32_t i = 0; i < n; ++i) {
    bool done = false;
    Iso X0;
    rcs[i] = pre_step(trackers[i], frames[i], ts[i], T_base_lidar ? T_base_lidar + 12 * (size_t)i : nullptr, s,
                      &out[i], &sv[i], &done, &X0);
    if (rcs[i] != KDS_OK || done) continue;
    kds_job j;
    memset(&j, 0, sizeof(j));
    j.type = trackers[i]->P.aligner_type;
    j.mode = KDS_JOB_COMPUTE;
    j.fixed = trackers[i]->keyframe;
    j.moving = frames[i];
    j.params = trackers[i]->P.aligner;
    memcpy(j.X, X0.m, sizeof(j.X));
    memcpy(j.fixed_X, I.m, sizeof(j.fixed_X));
    job_of[i] = (int32_t)jobs.size();
    jobs.push_back(j);
  }
  if (!jobs.empty()) {
    int rc = kds_batch_run(batch, jobs.data(), (int32_t)jobs.size(), 1, s);
    if (rc != KDS_OK) {
      for (int32_t i = 0; i < n; ++i)
        if (job_of[i] >= 0) rcs[i] = restore(trackers[i], sv[i], rc);
      job_of.assign((size_t)n, -1);
    }
  }
  for (int32_t i = 0; i < n; ++i) {
    if (job_of[i] < 0) continue;
    const kds_job& j = jobs[(size_t)job_of[i]];
    Iso X;
    memcpy(X.m, j.X, sizeof(X.m));
    double cv[6] = {0, 0, 0, 0, 0, 0};
    if (j.type == KDS_CTICP) memcpy(cv, j.v, sizeof(cv));
    rcs[i] = post_step(trackers[i], frames[i], X, j.stats, j.result, cv, s, sv[i], &out[i]);
  }
  int first = KDS_OK;
  for (int32_t i = 0; i < n; ++i) {
    if (codes) codes[i] = rcs[i];
    if (first == KDS_OK && rcs[i] != KDS_OK) first = rcs[i];
  }
  return finish(s, first);
}

int kds_tracker_get_pose(const kds_tracker* t, double pose_global[12], double pose_in_kf[12]) {
  if (!t) { set_error("kds_tracker_get_pose: NULL tracker"); return KDS_ERR_INVALID_ARG; }
  if (pose_global) memcpy(pose_global, t->pose_global.m, sizeof(double) * 12);
  if (pose_in_kf) memcpy(pose_in_kf, t->pose_in_kf.m, sizeof(double) * 12);
  return KDS_OK;
}

int kds_tracker_get_keyframe(const kds_tracker* t, const kds_tree** kf, double pose_in_world[12]) {
  if (!t) { set_error("kds_tracker_get_keyframe: NULL tracker"); return KDS_ERR_INVALID_ARG; }
  if (kf) *kf = t->keyframe;
  if (pose_in_world) memcpy(pose_in_world, t->kf_pose_in_world.m, sizeof(double) * 12);
  return KDS_OK;
}

int kds_tracker_get_state(const kds_tracker* t, kds_tracker_state* st) {
  if (!t || !st) { set_error("kds_tracker_get_state: NULL argument"); return KDS_ERR_INVALID_ARG; }
  memset(st, 0, sizeof(*st));
  st->params = t->P;
  st->last_ts = t->last_ts;
  st->frame_duration = t->frame_duration;
  memcpy(st->T_delta_log, t->T_delta_log, sizeof(st->T_delta_log));
  memcpy(st->kf_pose_in_world, t->kf_pose_in_world.m, sizeof(double) * 12);
  memcpy(st->pose_in_kf, t->pose_in_kf.m, sizeof(double) * 12);
  memcpy(st->pose_global, t->pose_global.m, sizeof(double) * 12);
  st->frame_idx = t->frame_idx;
  st->keyframe_count = t->keyframe_count;
  st->has_keyframe = t->keyframe ? 1 : 0;
  return KDS_OK;
}

int kds_tracker_set_state(kds_tracker* t, const kds_tracker_state* st, const kds_tree* keyframe) {
  if (!t || !st) { set_error("kds_tracker_set_state: NULL argument"); return KDS_ERR_INVALID_ARG; }
  if (st->params.aligner_type != t->P.aligner_type || st->params.motion_model != t->P.motion_model) {
    set_error("kds_tracker_set_state: the state's aligner type or motion model differs from the tracker's");
    return KDS_ERR_INVALID_ARG;
  }
  {  // the aligner settings decide every later pose: a state saved under others is refused
    const kds_aligner_params& a = st->params.aligner;
    const kds_aligner_params& b = t->P.aligner;
    const char* diff = nullptr;
    if (a.kernel_threshold != b.kernel_threshold) diff = "kernel_threshold";
    else if (a.damping != b.damping) diff = "damping";
    else if (a.max_error != b.max_error) diff = "max_error";
    else if (a.min_normal_cos != b.min_normal_cos) diff = "min_normal_cos";
    else if (a.min_good_measurements != b.min_good_measurements) diff = "min_good_measurements";
    else if (a.max_iterations != b.max_iterations) diff = "max_iterations";
    else if (a.velocity_damping != b.velocity_damping) diff = "velocity_damping";
    else if (a.term_crit != b.term_crit) diff = "term_crit";
    else if (a.d_pert != b.d_pert) diff = "d_pert";
    else if (a.d_score != b.d_score) diff = "d_score";
    if (diff) {
      set_error("kds_tracker_set_state: the state's aligner parameter %s differs from the tracker's", diff);
      return KDS_ERR_INVALID_ARG;
    }
  }
  if (st->has_keyframe && !keyframe) { set_error("kds_tracker_set_state: the state needs its keyframe tree"); return KDS_ERR_INVALID_ARG; }
  kds_tree* copy = nullptr;
  if (st->has_keyframe) {
    int rc = tree_clone(keyframe, t->stream, &copy);
    if (rc != KDS_OK) return rc;
    cudaError_t e = cudaStreamSynchronize(t->stream);
    if (e != cudaSuccess) {
      tree_release(copy->d);
      delete copy;
      return cuda_status(e, "kds_tracker_set_state", __FILE__, __LINE__);
    }
  }
  if (t->keyframe) {
    tree_release(t->keyframe->d);
    delete t->keyframe;
  }
  t->keyframe = copy;
  t->P.motion_model_alpha = st->params.motion_model_alpha;
  t->P.min_inlier_frac = st->params.min_inlier_frac;
  t->P.max_kf_trans = st->params.max_kf_trans;
  t->P.max_kf_rot_deg = st->params.max_kf_rot_deg;
  t->last_ts = st->last_ts;
  t->frame_duration = st->frame_duration;
  memcpy(t->T_delta_log, st->T_delta_log, sizeof(t->T_delta_log));
  memcpy(t->kf_pose_in_world.m, st->kf_pose_in_world, sizeof(double) * 12);
  memcpy(t->pose_in_kf.m, st->pose_in_kf, sizeof(double) * 12);
  memcpy(t->pose_global.m, st->pose_global, sizeof(double) * 12);
  t->frame_idx = st->frame_idx;
  t->keyframe_count = st->keyframe_count;
  return KDS_OK;
}

int kds_tracker_reset(kds_tracker* t) {
  if (!t) { set_error("kds_tracker_reset: NULL tracker"); return KDS_ERR_INVALID_ARG; }
  motion_reset(t);
  if (t->keyframe) {
    tree_release(t->keyframe->d);
    delete t->keyframe;
    t->keyframe = nullptr;
  }
  t->kf_pose_in_world = t->pose_in_kf = t->pose_global = iso_identity();
  t->frame_idx = 0;
  t->keyframe_count = 0;
  return KDS_OK;
}

void kds_tracker_free(kds_tracker* t) {
  if (!t) return;
  if (t->keyframe) {
    tree_release(t->keyframe->d);
    delete t->keyframe;
  }
  if (t->aligner) kds_aligner_free(t->aligner);
  delete t;
}

}  // extern "C"
