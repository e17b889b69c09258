// Seeded synthetic LiDAR input for tests and benchmarks (not part of the hot path).
//
// Scene: ground plane z = 0 plus axis-aligned boxes.  Scanner: a spinning LiDAR
// with `beams` elevation rows and `cols` azimuth columns; column i is fired at
// t_i = t_start + i * scan_time / cols, the timing model of the reference scanner
// (kd/d3/scanner.cpp:15,41-42).  The sensor pose at time t is X_start * M(t) with
// M(t) = [rodrigues(w t) | v t], the decoupled constant-velocity model the CT-ICP
// aligner estimates (kd/d3/cticp_impl_.h:75-85).  Each point is returned in the
// sensor frame at its own firing time, so a moving sensor yields a skewed scan.
// Rays are intersected analytically with the plane and the boxes (slab test).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

struct Rng {  // splitmix64 -> uniform / gaussian; identical on every platform
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uni() { return (double)(next() >> 11) * 0x1p-53; }
  double uni(double a, double b) { return a + (b - a) * uni(); }
  double gauss() {
    double u1 = uni(), u2 = uni();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

struct Box {
  double lo[3], hi[3];
};

struct Scene {
  std::vector<Box> boxes;
};

inline void rodrigues(const double w[3], double R[9]) {
  double a = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  if (a < 1e-12) {
    for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1.0 : 0.0;
    return;
  }
  double n[3] = {w[0] / a, w[1] / a, w[2] / a};
  double s = std::sin(a), c = 1.0 - std::cos(a);
  double K[9] = {0, -n[2], n[1], n[2], 0, -n[0], -n[1], n[0], 0};
  double K2[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double acc = 0;
      for (int k = 0; k < 3; ++k) acc += K[i * 3 + k] * K[k * 3 + j];
      K2[i * 3 + j] = acc;
    }
  for (int i = 0; i < 9; ++i) R[i] = ((i % 4 == 0) ? 1.0 : 0.0) + s * K[i] + c * K2[i];
}

// pose as R (row-major 3x3) + t
struct Pose {
  double R[9];
  double t[3];
};

inline Pose compose(const Pose& A, const Pose& B) {
  Pose C;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      double acc = 0;
      for (int k = 0; k < 3; ++k) acc += A.R[i * 3 + k] * B.R[k * 3 + j];
      C.R[i * 3 + j] = acc;
    }
    double acc = A.t[i];
    for (int k = 0; k < 3; ++k) acc += A.R[i * 3 + k] * B.t[k];
    C.t[i] = acc;
  }
  return C;
}

inline Pose motion_at(const double v[6], double t) {
  Pose M;
  double w[3] = {v[3] * t, v[4] * t, v[5] * t};
  rodrigues(w, M.R);
  for (int i = 0; i < 3; ++i) M.t[i] = v[i] * t;
  return M;
}

inline double cast(const Scene& S, const double o[3], const double d[3], double tmax) {
  double best = tmax;
  if (d[2] < -1e-12) {
    double t = -o[2] / d[2];
    if (t > 0 && t < best) best = t;
  }
  for (const Box& b : S.boxes) {
    double t0 = 0.0, t1 = best;
    bool hit = true;
    for (int k = 0; k < 3 && hit; ++k) {
      if (std::fabs(d[k]) < 1e-15) {
        if (o[k] < b.lo[k] || o[k] > b.hi[k]) hit = false;
      } else {
        double inv = 1.0 / d[k];
        double ta = (b.lo[k] - o[k]) * inv, tb = (b.hi[k] - o[k]) * inv;
        if (ta > tb) std::swap(ta, tb);
        t0 = std::max(t0, ta);
        t1 = std::min(t1, tb);
        if (t0 > t1) hit = false;
      }
    }
    if (hit && t0 > 1e-9 && t0 < best) best = t0;
  }
  return best;
}

}  // namespace

extern "C" {

// Scene with a ground plane and `num_boxes` boxes (footprint sides U[1,8] m, height
// U[2,15] m) whose centres lie within `radius` m of the origin, keeping a 4 m wide
// corridor along +x free for the sensor trajectory.  Writes 6 doubles per box.
int32_t kds_synth_scene(uint64_t seed, int32_t num_boxes, double radius, double* boxes_out) {
  Rng rng(seed);
  int made = 0, guard = 0;
  while (made < num_boxes && guard < 100000) {
    ++guard;
    double r = radius * std::sqrt(rng.uni());
    double th = rng.uni(0, 6.283185307179586);
    double cx = r * std::cos(th), cy = r * std::sin(th);
    double sx = rng.uni(1.0, 8.0), sy = rng.uni(1.0, 8.0), h = rng.uni(2.0, 15.0);
    double lo[3] = {cx - sx / 2, cy - sy / 2, 0.0}, hi[3] = {cx + sx / 2, cy + sy / 2, h};
    if (hi[1] > -4.0 && lo[1] < 4.0 && hi[0] > -40.0) continue;  // corridor
    if (std::hypot(cx, cy) < 5.0) continue;
    for (int k = 0; k < 3; ++k) { boxes_out[6 * made + k] = lo[k]; boxes_out[6 * made + 3 + k] = hi[k]; }
    ++made;
  }
  return made;
}

// Casts one sweep.  start_pose12: sensor pose at t_start (3x4 row-major, world <- sensor).
// vel6: [v; w] body velocity (decoupled motion).  Beam elevations are uniform in
// [elev_min, elev_max] degrees, columns uniform in azimuth [0, 2pi).  Returns the
// number of points written (<= beams*cols); xyz in the sensor frame at firing time.
int64_t kds_synth_scan(const double* boxes, int32_t num_boxes, const double* start_pose12, const double* vel6,
                       int32_t beams, int32_t cols, double elev_min_deg, double elev_max_deg, double scan_time,
                       double t_start, double r_min, double r_max, double noise_sigma, uint64_t seed,
                       int32_t num_threads, float* xyz_out, double* stamps_out) {
  Scene S;
  for (int i = 0; i < num_boxes; ++i) {
    Box b;
    for (int k = 0; k < 3; ++k) { b.lo[k] = boxes[6 * i + k]; b.hi[k] = boxes[6 * i + 3 + k]; }
    S.boxes.push_back(b);
  }
  Pose X0;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) X0.R[i * 3 + j] = start_pose12[i * 4 + j];
    X0.t[i] = start_pose12[i * 4 + 3];
  }
  double v[6];
  for (int i = 0; i < 6; ++i) v[i] = vel6 ? vel6[i] : 0.0;
  const double deg = 3.141592653589793 / 180.0;
  int nt = std::max(1, std::min(num_threads, 64));
  std::vector<std::vector<float>> pts(nt);
  std::vector<std::vector<double>> sts(nt);
  auto work = [&](int tid) {
    for (int c = tid; c < cols; c += nt) {
      Rng rng(seed * 1000003ull + (uint64_t)c);
      double tc = scan_time * (double)c / (double)cols;
      Pose W = compose(X0, motion_at(v, tc));
      double az = 6.283185307179586 * (double)c / (double)cols;
      for (int b = 0; b < beams; ++b) {
        double el = (beams > 1) ? (elev_min_deg + (elev_max_deg - elev_min_deg) * (double)b / (double)(beams - 1))
                                : elev_min_deg;
        el *= deg;
        double dl[3] = {std::cos(el) * std::cos(az), std::cos(el) * std::sin(az), std::sin(el)};
        double dw[3];
        for (int i = 0; i < 3; ++i) dw[i] = W.R[i * 3] * dl[0] + W.R[i * 3 + 1] * dl[1] + W.R[i * 3 + 2] * dl[2];
        double t = cast(S, W.t, dw, r_max + 1.0);
        double noise = noise_sigma * rng.gauss();
        if (!(t >= r_min && t <= r_max)) continue;
        double rr = t + noise;
        if (rr < r_min || rr > r_max) continue;
        pts[tid].push_back((float)(dl[0] * rr));
        pts[tid].push_back((float)(dl[1] * rr));
        pts[tid].push_back((float)(dl[2] * rr));
        sts[tid].push_back(t_start + tc);
      }
    }
  };
  std::vector<std::thread> th;
  for (int i = 0; i < nt; ++i) th.emplace_back(work, i);
  for (auto& t : th) t.join();
  // deterministic interleave: column c was produced by thread c % nt in column order
  std::vector<size_t> pos(nt, 0);
  int64_t k = 0;
  std::vector<size_t> ps(nt, 0);
  for (int c = 0; c < cols; ++c) {
    int tid = c % nt;
    // points of column c are the next run in pts[tid] with stamp == t_start + tc
    double tc = t_start + scan_time * (double)c / (double)cols;
    while (ps[tid] < sts[tid].size() && sts[tid][ps[tid]] == tc) {
      size_t q = ps[tid];
      xyz_out[3 * k] = pts[tid][3 * q];
      xyz_out[3 * k + 1] = pts[tid][3 * q + 1];
      xyz_out[3 * k + 2] = pts[tid][3 * q + 2];
      stamps_out[k] = sts[tid][q];
      ++k;
      ++ps[tid];
    }
  }
  return k;
}

// Applies a pose (3x4) to points in place, in double: p <- R p + t.
void kds_synth_transform(float* xyz, int64_t n, const double* pose12) {
  for (int64_t i = 0; i < n; ++i) {
    double p[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    for (int r = 0; r < 3; ++r)
      xyz[3 * i + r] = (float)(pose12[r * 4] * p[0] + pose12[r * 4 + 1] * p[1] + pose12[r * 4 + 2] * p[2] + pose12[r * 4 + 3]);
  }
}

}  // extern "C"
