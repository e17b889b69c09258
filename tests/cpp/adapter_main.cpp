// Test driver for include/kds.hpp.
//   adapter_main conf <file.conf>
//       prints the parameters that the conf blocks configure (no device needed)
//   adapter_main align <file.conf> <fixed.bin> <moving.bin> <x0.bin> <v0.bin> <out.bin>
//       builds both trees with the conf's TreeGeneratorB2003D, runs the conf's
//       CTICPB2003D and writes [result, X(12), v(6)] as doubles
//   adapter_main track <file.conf> <out.bin> <frame0.bin> <frame1.bin> ...
//       tracks the frames (stamps of frame i start at 0.1 i; ts = 0.1 i) with the
//       conf's CTICPB2003D and a constant-velocity TrackerB200 (max_kf_trans 0.5,
//       min_inlier_frac 0.3) and writes [new_keyframe, result, pose_in_world(12)] per frame
// A cloud file is int64 n, then n*3 float32 xyz, then n float64 stamps.
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "kds.hpp"

using namespace kds_b200;

static void read_cloud(const std::string& path, std::vector<float>& xyz, std::vector<double>& st) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open " + path);
  int64_t n = 0;
  f.read(reinterpret_cast<char*>(&n), sizeof(n));
  xyz.resize((size_t)n * 3);
  st.resize((size_t)n);
  f.read(reinterpret_cast<char*>(xyz.data()), (std::streamsize)(xyz.size() * sizeof(float)));
  f.read(reinterpret_cast<char*>(st.data()), (std::streamsize)(st.size() * sizeof(double)));
  if (!f) throw std::runtime_error("short read " + path);
}

template <size_t N>
static std::array<double, N> read_vec(const std::string& path) {
  std::array<double, N> v;
  std::ifstream f(path, std::ios::binary);
  f.read(reinterpret_cast<char*>(v.data()), sizeof(double) * N);
  if (!f) throw std::runtime_error("short read " + path);
  return v;
}

static const ConfObject* find_type(const std::vector<ConfObject>& objs, const char* type) {
  for (auto& o : objs)
    if (o.type == type) return &o;
  throw std::runtime_error(std::string("no block of type ") + type);
}

static int conf_mode(const std::string& path) {
  auto objs = ConfReader::load(path);
  TreeGeneratorB2003D gen;
  ConfReader::configure(gen, *find_type(objs, "TreeGeneratorB2003D"));
  const kds_tree_params& t = gen.params();
  std::printf("tree %d %d %d %d %.9g %.9g %.9g %.9g\n", t.propagate_normal, t.tree_min_good_leaves, t.leaf_min_points,
              t.leaf_max_points, t.leaf_density, t.leaf_min_normal_incidence, t.leaf_eigenvalue_threshold,
              t.leaf_normal_eigenratio);
  const char* types[2] = {"CTICPB2003D", "ICPB2003D"};
  for (const char* ty : types) {
    const int32_t type = std::string(ty) == "CTICPB2003D" ? KDS_CTICP : KDS_ICP;
    kds_aligner_params p = ConfReader::aligner_params(type, *find_type(objs, ty), objs);
    std::printf("%s %.9g %.9g %.9g %.9g %d %d %.9g %d %.9g %.9g\n", ty, p.kernel_threshold, p.damping, p.max_error,
                p.min_normal_cos, p.min_good_measurements, p.max_iterations, p.velocity_damping, p.term_crit, p.d_pert,
                p.d_score);
  }
  return 0;
}

static int align_mode(char** argv) {
  auto objs = ConfReader::load(argv[2]);
  TreeGeneratorB2003D gen;
  ConfReader::configure(gen, *find_type(objs, "TreeGeneratorB2003D"));
  std::vector<float> xf, xm;
  std::vector<double> sf, sm;
  read_cloud(argv[3], xf, sf);
  read_cloud(argv[4], xm, sm);
  TreePtr fixed = gen.makeTree(xf.data(), sf.data(), (int64_t)sf.size());
  TreePtr built = gen.makeTree(xm.data(), sm.data(), (int64_t)sm.size());
  if (!fixed || !built) throw std::runtime_error("tree rejected");
  // the moving tree goes through the tree wire format (toMessage / fromTreeMsg): the
  // alignment must not change
  std::vector<kds_kdnode3f> records;
  const kds_kdtree3f msg = built->toMessage(records);
  TreePtr moving = Tree::fromTreeMsg(msg);
  CTICPB2003D a;
  ConfReader::configure(a, *find_type(objs, "CTICPB2003D"), objs);
  a.setFixed(*fixed);
  a.setMoving(*moving);
  a.setX(read_vec<12>(argv[5]));
  a.setVelocities(read_vec<6>(argv[6]));
  int r = a.compute();
  Pose X = a.getX();
  Vector6 v = a.velocities();
  std::vector<double> out;
  out.push_back((double)r);
  out.insert(out.end(), X.begin(), X.end());
  out.insert(out.end(), v.begin(), v.end());
  std::ofstream f(argv[7], std::ios::binary);
  f.write(reinterpret_cast<const char*>(out.data()), (std::streamsize)(out.size() * sizeof(double)));
  std::printf("result %d inliers %d\n", r, a.stats().num_inliers);
  return 0;
}

static int track_mode(int argc, char** argv) {
  auto objs = ConfReader::load(argv[2]);
  TreeGeneratorB2003D gen;
  ConfReader::configure(gen, *find_type(objs, "TreeGeneratorB2003D"));
  CTICPB2003D odom;
  ConfReader::configure(odom, *find_type(objs, "CTICPB2003D"), objs);
  kds_tracker_params tp = TrackerB200::defaults();
  TrackerB200::setParam(tp, "max_kf_trans", 0.5);
  TrackerB200::setParam(tp, "min_inlier_frac", 0.3);
  TrackerB200 tracker(odom, true, tp);
  std::vector<double> out;
  for (int i = 4; i < argc; ++i) {
    std::vector<float> xyz;
    std::vector<double> st;
    read_cloud(argv[i], xyz, st);
    TreePtr t = gen.makeTree(xyz.data(), st.data(), (int64_t)st.size());
    if (!t) throw std::runtime_error("tree rejected");
    TrackerB200::Result r = tracker.addFrame(*t, 0.1 * (i - 4));
    out.push_back((double)r.new_keyframe);
    out.push_back((double)r.result);
    out.insert(out.end(), r.pose_in_world, r.pose_in_world + 12);
  }
  std::ofstream f(argv[3], std::ios::binary);
  f.write(reinterpret_cast<const char*>(out.data()), (std::streamsize)(out.size() * sizeof(double)));
  const Pose g = tracker.poseGlobal();
  std::printf("frames %d x %.6f\n", argc - 4, g[3]);
  return 0;
}

int main(int argc, char** argv) {
  try {
    if (argc >= 3 && std::string(argv[1]) == "conf") return conf_mode(argv[2]);
    if (argc >= 8 && std::string(argv[1]) == "align") return align_mode(argv);
    if (argc >= 5 && std::string(argv[1]) == "track") return track_mode(argc, argv);
    std::fprintf(stderr,
                 "usage: adapter_main conf <file> | align <conf> <fixed> <moving> <x0> <v0> <out> |"
                 " track <conf> <out> <frames...>\n");
    return 2;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
