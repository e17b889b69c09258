// C++ adapter over the C ABI in kds.h with the method names of the reference's
// aligner and tree-generator types, so that call sites written against
// TreeAlignerBase_ (kd/icp/tree_aligner_base_.h:52-137) and TreeGenerator_
// (kd/tree/tree_generator_.h:18-41) keep their shape.  Errors are rethrown as
// std::runtime_error, as the reference does; compute() keeps its int return value.
//
// Poses are 3x4 row-major [R | t] in double (12 values); velocities are
// [v_x v_y v_z w_x w_y w_z].  A caller holding Eigen types converts at the call site
// (Isometry3f::matrix().topRows<3>() in row-major order).
//
// Header-only; link with libkds.so.
#pragma once

#include <array>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "kds.h"

namespace kds_b200 {

using Pose = std::array<double, 12>;
using Vector6 = std::array<double, 6>;
using Stats = kds_stats;

inline Pose identity() { return Pose{1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0}; }

inline void check(int rc, const char* where) {
  if (rc != KDS_OK) {
    std::string msg = std::string(where) + ": status " + std::to_string(rc) + ": " + kds_last_error();
    throw std::runtime_error(msg);
  }
}

// Parameter setters by the reference's PARAM names (kd/tree/tree_generator_.h:18-25,
// kd/icp/tree_aligner_base_.h:39-47, kd/cticp/cticp_.h:61, kd/icp/icp_stats_.h:89-90).
// They return false for a name the type does not have.
inline bool set_tree_param(kds_tree_params& p, const std::string& k, double v) {
  if (k == "propagate_normal") p.propagate_normal = v != 0.0;
  else if (k == "tree_min_good_leaves") p.tree_min_good_leaves = (int32_t)v;
  else if (k == "leaf_min_points") p.leaf_min_points = (int32_t)v;
  else if (k == "leaf_max_points") p.leaf_max_points = (int32_t)v;
  else if (k == "leaf_density") p.leaf_density = (float)v;
  else if (k == "leaf_min_normal_incidence") p.leaf_min_normal_incidence = (float)v;
  else if (k == "leaf_eigenvalue_threshold") p.leaf_eigenvalue_threshold = (float)v;
  else if (k == "leaf_normal_eigenratio") p.leaf_normal_eigenratio = (float)v;
  else return false;
  return true;
}

inline bool set_aligner_param(kds_aligner_params& p, int32_t type, const std::string& k, double v) {
  if (k == "kernel_threshold") p.kernel_threshold = (float)v;
  else if (k == "damping") p.damping = (float)v;
  else if (k == "max_error") p.max_error = (float)v;
  else if (k == "min_normal_cos") p.min_normal_cos = (float)v;
  else if (k == "min_good_measurements") p.min_good_measurements = (int32_t)v;
  else if (k == "max_iterations") p.max_iterations = (int32_t)v;
  else if (k == "velocity_damping" && type == KDS_CTICP) p.velocity_damping = (float)v;
  else if (k == "d_pert") { p.d_pert = (float)v; p.term_crit = 1; }
  else if (k == "d_score") { p.d_score = (float)v; p.term_crit = 1; }
  else return false;
  return true;
}

// ---------------------------------------------------------------------------
// Trees.  Owns its device memory (as TreeCUDA_ does, kd/tree/tree_cuda_impl_.h:30-40).
class Tree {
 public:
  explicit Tree(kds_tree* t) : _t(t) {}
  ~Tree() {
    if (_t) kds_tree_free(_t);
  }
  Tree(const Tree&) = delete;
  Tree& operator=(const Tree&) = delete;

  kds_tree* handle() const { return _t; }
  kds_tree_info info() const {
    kds_tree_info i;
    check(kds_tree_get_info(_t, &i), "kds_tree_get_info");
    return i;
  }
  int64_t numNodes() const { return info().num_nodes; }
  int64_t numLeaves() const { return info().num_leaves; }
  double tsStart() const { return info().ts_start; }
  bool isGPU() const { return true; }
  // Tree_::applyVelocitiesInPlace / applyIsometryInPlace (kd/tree/tree_.h:15-56)
  void applyVelocitiesInPlace(const Vector6& v, bool skip_leaves = false) {
    float vf[6];
    for (int i = 0; i < 6; ++i) vf[i] = (float)v[i];
    check(kds_tree_apply_velocities(_t, vf, skip_leaves ? 1 : 0, nullptr), "kds_tree_apply_velocities");
  }
  void applyIsometryInPlace(const Pose& X) {
    float xf[12];
    for (int i = 0; i < 12; ++i) xf[i] = (float)X[i];
    check(kds_tree_apply_isometry(_t, xf, nullptr), "kds_tree_apply_isometry");
  }
  // extractCompressedLeaves: [mean, dir] per leaf
  std::vector<float> extractCompressedLeaves() const {
    std::vector<float> out((size_t)numLeaves() * 6);
    check(kds_tree_extract_compressed_leaves(_t, nullptr, out.data(), nullptr), "kds_tree_extract_compressed_leaves");
    return out;
  }
  // toMessage (lib/kd_io/slam_messages.h:47-80): the tree fields of a KDTree3f message;
  // the node records are written to `nodes`, which the returned struct points into.
  kds_kdtree3f toMessage(std::vector<kds_kdnode3f>& nodes) const {
    kds_kdtree3f m{};
    check(kds_tree_to_msg(_t, &m), "kds_tree_to_msg");  // node count
    nodes.resize((size_t)m.num_nodes);
    m.nodes = nodes.data();
    check(kds_tree_to_msg(_t, &m), "kds_tree_to_msg");
    return m;
  }
  // TreeLoader_::fromTreeMsg (lib/kd_io/tree_loader_impl_.h:59-70): a device tree without points
  static std::shared_ptr<Tree> fromTreeMsg(const kds_kdtree3f& m) {
    kds_tree* t = nullptr;
    check(kds_tree_from_msg(&m, &t), "kds_tree_from_msg");
    return std::make_shared<Tree>(t);
  }

 private:
  kds_tree* _t;
};
using TreePtr = std::shared_ptr<Tree>;

// TreeGenerator_ with the reference's PARAM names and defaults.
class TreeGeneratorB2003D {
 public:
  TreeGeneratorB2003D() { kds_tree_params_default(&_p); }
  kds_tree_params& params() { return _p; }
  const kds_tree_params& params() const { return _p; }

  // Sets a PARAM by its reference name; returns false for a name this type lacks.
  bool setParam(const std::string& k, double v) { return set_tree_param(_p, k, v); }
  void setParams(const kds_tree_params& p) { _p = p; }

  // makeTree (kd/tree/tree_generator_impl_.h:7-19): nullptr where the reference
  // rejects the cloud.  xyz: n*3 floats on the host; stamps: n doubles or nullptr.
  TreePtr makeTree(const float* xyz, const double* stamps, int64_t n, void* stream = nullptr) const {
    kds_tree* t = nullptr;
    int rc = kds_tree_build(xyz, stamps, n, KDS_MEM_HOST, &_p, stream, &t);
    if (rc == KDS_ERR_TREE_REJECTED) return nullptr;
    check(rc, "kds_tree_build");
    return std::make_shared<Tree>(t);
  }

 private:
  kds_tree_params _p;
};

// ---------------------------------------------------------------------------
// Aligners.  Hold non-owning tree pointers (kd/icp/tree_aligner_base_.h:49-50).
class AlignerB200 {
 public:
  AlignerB200(const AlignerB200&) = delete;
  AlignerB200& operator=(const AlignerB200&) = delete;
  virtual ~AlignerB200() {
    if (_a) kds_aligner_free(_a);
  }
  kds_aligner* handle() const { return _a; }
  kds_aligner_params& params() { return _p; }
  const kds_aligner_params& params() const { return _p; }
  int dim() const { return _type == KDS_ICP ? 6 : 12; }
  bool isGPU() const { return true; }

  // Sets a PARAM by its reference name and pushes it to the aligner.
  bool setParam(const std::string& k, double v) {
    if (!set_aligner_param(_p, _type, k, v)) return false;
    check(kds_aligner_set_params(_a, &_p), "kds_aligner_set_params");
    return true;
  }
  void setParams(const kds_aligner_params& p) {
    _p = p;
    check(kds_aligner_set_params(_a, &_p), "kds_aligner_set_params");
  }
  int32_t alignerType() const { return _type; }
  // term_crit: nullptr (none) or ICPTerminationCriteriaScore{d_pert, d_score}
  void setTerminationCriteria(bool on, double d_pert = 1e-3, double d_score = 1e-3) {
    _p.term_crit = on ? 1 : 0;
    _p.d_pert = (float)d_pert;
    _p.d_score = (float)d_score;
    check(kds_aligner_set_params(_a, &_p), "kds_aligner_set_params");
  }
  void setStream(void* s) { check(kds_aligner_set_stream(_a, s), "kds_aligner_set_stream"); }

  void setFixed(const Tree& t) { check(kds_aligner_set_fixed(_a, t.handle()), "kds_aligner_set_fixed"); }
  void setMoving(const Tree& t) { check(kds_aligner_set_moving(_a, t.handle()), "kds_aligner_set_moving"); }
  void setX(const Pose& X) { check(kds_aligner_set_x(_a, X.data()), "kds_aligner_set_x"); }
  Pose getX() const {
    Pose X;
    check(kds_aligner_get_x(_a, X.data()), "kds_aligner_get_x");
    return X;
  }
  void setFixedX(const Pose& X) { check(kds_aligner_set_fixed_x(_a, X.data()), "kds_aligner_set_fixed_x"); }
  void resetMovingState() { check(kds_aligner_reset_moving_state(_a), "kds_aligner_reset_moving_state"); }
  void setPosePrior(const Pose& X_ref, const Pose& Z, const std::array<double, 36>& omega) {
    check(kds_aligner_set_pose_prior(_a, X_ref.data(), Z.data(), omega.data()), "kds_aligner_set_pose_prior");
  }
  // _fixed_forest / makeFixedEntry
  void addFixedEntry(const Tree& t, const Pose& X) {
    check(kds_aligner_add_fixed_entry(_a, t.handle(), X.data()), "kds_aligner_add_fixed_entry");
  }
  void clearFixedForest() { check(kds_aligner_clear_fixed_forest(_a), "kds_aligner_clear_fixed_forest"); }

  // compute: -i on a failed round i, i on early termination, else max_iterations
  int compute(bool stats_mode = false) {
    int32_t r = 0;
    check(kds_aligner_compute(_a, stats_mode ? 1 : 0, &r), "kds_aligner_compute");
    return r;
  }
  bool oneRound(bool stats_mode = false) {
    int32_t ok = 0;
    check(kds_aligner_one_round(_a, stats_mode ? 1 : 0, &ok), "kds_aligner_one_round");
    return ok != 0;
  }
  void buildQuadraticForm(bool stats_mode = false) {
    check(kds_aligner_build_quadratic_form(_a, stats_mode ? 1 : 0), "kds_aligner_build_quadratic_form");
  }
  // public fields H, b, dx (row-major, D = dim())
  std::vector<double> H() const { return hb(0); }
  std::vector<double> b() const { return hb(1); }
  std::vector<double> dx() const { return hb(2); }
  std::array<double, 36> getPoseHessian() const {
    std::array<double, 36> H6;
    check(kds_aligner_get_pose_hessian(_a, H6.data()), "kds_aligner_get_pose_hessian");
    return H6;
  }
  Stats stats() const {
    Stats s;
    check(kds_aligner_get_stats(_a, &s), "kds_aligner_get_stats");
    return s;
  }
  std::vector<Stats> statsLog() const {
    std::vector<Stats> log(256);
    int32_t n = 0;
    check(kds_aligner_get_stats_log(_a, log.data(), (int32_t)log.size(), &n), "kds_aligner_get_stats_log");
    log.resize((size_t)n);
    return log;
  }

 protected:
  explicit AlignerB200(int32_t type) : _type(type) {
    kds_aligner_params_default(&_p);
    check(kds_aligner_create(type, &_p, &_a), "kds_aligner_create");
  }
  std::vector<double> hb(int which) const {
    const int D = dim();
    std::vector<double> H((size_t)D * D), b((size_t)D), dx((size_t)D);
    check(kds_aligner_get_hb(_a, H.data(), b.data(), dx.data()), "kds_aligner_get_hb");
    return which == 0 ? H : (which == 1 ? b : dx);
  }
  int32_t _type;
  kds_aligner_params _p;
  kds_aligner* _a = nullptr;
};

// In place of ICPCPU3D / ICPCUDA3D.
class ICPB2003D : public AlignerB200 {
 public:
  ICPB2003D() : AlignerB200(KDS_ICP) {}
};

// In place of CTICPCPU3D / CTICPCUDA3D.
class CTICPB2003D : public AlignerB200 {
 public:
  CTICPB2003D() : AlignerB200(KDS_CTICP) {}
  void setVelocities(const Vector6& v) { check(kds_aligner_set_velocities(_a, v.data()), "kds_aligner_set_velocities"); }
  Vector6 velocities() const {
    Vector6 v;
    check(kds_aligner_get_velocities(_a, v.data()), "kds_aligner_get_velocities");
    return v;
  }
  void setFixedVelocities(const Vector6& v) {
    check(kds_aligner_set_fixed_velocities(_a, v.data()), "kds_aligner_set_fixed_velocities");
  }
  void buildQuadraticFormDual(bool stats_mode = false) {
    check(kds_aligner_build_quadratic_form_dual(_a, stats_mode ? 1 : 0), "kds_aligner_build_quadratic_form_dual");
  }
};

// ---------------------------------------------------------------------------
// Tracker step: the odometry of TrackerProc_::addFrame with its motion model and
// SLAMProc_'s keyframe switch (kd/tracker/tracker_proc_frame_impl_.h:33-123).
// Takes the aligner's type and PARAMs; the keyframe is a device copy it owns.
class TrackerB200 {
 public:
  using Result = kds_tracker_result;
  // PARAM names: min_inlier_frac, max_kf_trans, max_kf_rot_deg (kd/tracker/tracker_proc_.h:55-57),
  // motion_model_alpha (kd/motion_model/const_vel_motion_model_.h:19)
  static bool setParam(kds_tracker_params& p, const std::string& k, double v) {
    if (k == "min_inlier_frac") p.min_inlier_frac = (float)v;
    else if (k == "max_kf_trans") p.max_kf_trans = (float)v;
    else if (k == "max_kf_rot_deg") p.max_kf_rot_deg = (float)v;
    else if (k == "motion_model_alpha") p.motion_model_alpha = (float)v;
    else return false;
    return true;
  }
  TrackerB200(const AlignerB200& odom_aligner, bool const_vel, kds_tracker_params p = defaults(),
              void* stream = nullptr) {
    p.aligner_type = odom_aligner.alignerType();
    p.aligner = odom_aligner.params();
    p.motion_model = const_vel ? KDS_MOTION_CONST_VEL : KDS_MOTION_ZERO_VEL;
    check(kds_tracker_create(&p, stream, &_t), "kds_tracker_create");
  }
  ~TrackerB200() {
    if (_t) kds_tracker_free(_t);
  }
  TrackerB200(const TrackerB200&) = delete;
  TrackerB200& operator=(const TrackerB200&) = delete;

  static kds_tracker_params defaults() {
    kds_tracker_params p;
    kds_tracker_params_default(&p);
    return p;
  }
  // addFrame: frame is transformed in place (T_base_lidar, then the velocity morphs)
  Result addFrame(Tree& frame, double ts, const Pose* T_base_lidar = nullptr) {
    Result r;
    check(kds_tracker_add_frame(_t, frame.handle(), ts, T_base_lidar ? T_base_lidar->data() : nullptr, &r),
          "kds_tracker_add_frame");
    return r;
  }
  Pose poseGlobal() const {
    Pose X;
    check(kds_tracker_get_pose(_t, X.data(), nullptr), "kds_tracker_get_pose");
    return X;
  }
  Pose poseInKeyframe() const {
    Pose X;
    check(kds_tracker_get_pose(_t, nullptr, X.data()), "kds_tracker_get_pose");
    return X;
  }
  void reset() { check(kds_tracker_reset(_t), "kds_tracker_reset"); }
  kds_tracker* handle() const { return _t; }

 private:
  kds_tracker* _t = nullptr;
};

// ---------------------------------------------------------------------------
// Reader for the blocks of a BOSS .conf file: a sequence of `"Type" : { ... }`
// objects with `//` comments, an integer "#id", scalar and string fields, and nested
// `{ "#pointer" : id }` references.  Enough to take the PARAM values of the
// aligner and tree-generator blocks from the reference's configuration files.
struct ConfObject {
  std::string type;
  int id = -1;
  std::map<std::string, std::string> fields;   // scalar/string values, as written
  std::map<std::string, int> pointers;         // field -> referenced #id
};

class ConfReader {
 public:
  static std::vector<ConfObject> parse(const std::string& text) {
    ConfReader r(strip_comments(text));
    std::vector<ConfObject> out;
    for (;;) {
      r.ws();
      if (r.eof()) break;
      ConfObject o;
      o.type = r.string_lit();
      r.expect(':');
      r.object(o);
      out.push_back(std::move(o));
    }
    return out;
  }
  static std::vector<ConfObject> load(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return parse(ss.str());
  }
  static const ConfObject* find_id(const std::vector<ConfObject>& objs, int id) {
    for (auto& o : objs)
      if (o.id == id) return &o;
    return nullptr;
  }
  // The parameters of an aligner block of the given type (KDS_ICP / KDS_CTICP), starting
  // from the defaults and following term_crit to its ICPTerminationCriteriaScore block
  // (a missing or negative #pointer means no criterion).  Non-numeric fields such as
  // name and log_file are skipped.
  static kds_aligner_params aligner_params(int32_t type, const ConfObject& o, const std::vector<ConfObject>& all) {
    kds_aligner_params p;
    kds_aligner_params_default(&p);
    for (auto& kv : o.fields) {
      double v;
      if (numeric(kv.second, &v)) set_aligner_param(p, type, kv.first, v);
    }
    p.term_crit = 0;
    auto tc = o.pointers.find("term_crit");
    if (tc != o.pointers.end() && tc->second >= 0) {
      const ConfObject* t = find_id(all, tc->second);
      if (!t) throw std::runtime_error("term_crit points to a missing #id");
      double v;
      p.term_crit = 1;
      p.d_pert = t->fields.count("d_pert") && numeric(t->fields.at("d_pert"), &v) ? (float)v : 1e-3f;
      p.d_score = t->fields.count("d_score") && numeric(t->fields.at("d_score"), &v) ? (float)v : 1e-3f;
    }
    return p;
  }
  static kds_tree_params tree_params(const ConfObject& o) {
    kds_tree_params p;
    kds_tree_params_default(&p);
    for (auto& kv : o.fields) {
      double v;
      if (numeric(kv.second, &v)) set_tree_param(p, kv.first, v);
    }
    return p;
  }
  static void configure(AlignerB200& a, const ConfObject& o, const std::vector<ConfObject>& all) {
    a.setParams(aligner_params(a.alignerType(), o, all));
  }
  static void configure(TreeGeneratorB2003D& g, const ConfObject& o) { g.setParams(tree_params(o)); }

 private:
  explicit ConfReader(std::string s) : _s(std::move(s)) {}
  static std::string strip_comments(const std::string& t) {
    std::string o;
    bool in_str = false;
    for (size_t i = 0; i < t.size(); ++i) {
      char c = t[i];
      if (in_str) {
        o += c;
        if (c == '\\' && i + 1 < t.size()) o += t[++i];
        else if (c == '"') in_str = false;
      } else if (c == '"') {
        in_str = true;
        o += c;
      } else if (c == '/' && i + 1 < t.size() && t[i + 1] == '/') {
        while (i < t.size() && t[i] != '\n') ++i;
        o += '\n';
      } else {
        o += c;
      }
    }
    return o;
  }
  static bool numeric(const std::string& s, double* v) {
    if (s.empty()) return false;
    char* end = nullptr;
    *v = std::strtod(s.c_str(), &end);
    return end && *end == '\0';
  }
  bool eof() const { return _i >= _s.size(); }
  void ws() {
    while (!eof() && std::isspace((unsigned char)_s[_i])) ++_i;
  }
  void expect(char c) {
    ws();
    if (eof() || _s[_i] != c) throw std::runtime_error(std::string("conf: expected '") + c + "'");
    ++_i;
  }
  std::string string_lit() {
    ws();
    if (eof() || _s[_i] != '"') throw std::runtime_error("conf: expected a string");
    std::string r;
    for (++_i; !eof() && _s[_i] != '"'; ++_i) {
      if (_s[_i] == '\\' && _i + 1 < _s.size()) ++_i;
      r += _s[_i];
    }
    if (eof()) throw std::runtime_error("conf: unterminated string");
    ++_i;
    return r;
  }
  std::string scalar() {
    ws();
    size_t b = _i;
    while (!eof() && _s[_i] != ',' && _s[_i] != '}' && _s[_i] != ']' && !std::isspace((unsigned char)_s[_i])) ++_i;
    return _s.substr(b, _i - b);
  }
  void skip_value() {
    ws();
    if (eof()) return;
    char c = _s[_i];
    if (c == '"') { string_lit(); return; }
    if (c == '{' || c == '[') {
      char close = c == '{' ? '}' : ']';
      int depth = 0;
      for (; !eof(); ++_i) {
        if (_s[_i] == '"') { string_lit(); --_i; continue; }
        if (_s[_i] == c) ++depth;
        else if (_s[_i] == close && --depth == 0) { ++_i; return; }
      }
      return;
    }
    scalar();
  }
  void object(ConfObject& o) {
    expect('{');
    for (;;) {
      ws();
      if (!eof() && _s[_i] == '}') { ++_i; return; }
      std::string key = string_lit();
      expect(':');
      ws();
      if (!eof() && _s[_i] == '"') {
        o.fields[key] = string_lit();
      } else if (!eof() && _s[_i] == '{') {
        // nested object: a pointer reference or an inline value
        size_t save = _i;
        ++_i;
        ws();
        bool is_ptr = false;
        if (!eof() && _s[_i] == '"') {
          std::string k2 = string_lit();
          if (k2 == "#pointer") {
            expect(':');
            o.pointers[key] = std::atoi(scalar().c_str());
            expect('}');
            is_ptr = true;
          }
        }
        if (!is_ptr) {
          _i = save;
          skip_value();
        }
      } else if (!eof() && _s[_i] == '[') {
        skip_value();
      } else {
        std::string v = scalar();
        if (key == "#id") o.id = std::atoi(v.c_str());
        else o.fields[key] = v;
      }
      ws();
      if (!eof() && _s[_i] == ',') ++_i;
    }
  }
  std::string _s;
  size_t _i = 0;
};

}  // namespace kds_b200
