// CPU oracle for the KD-SLAM registration hot path -- TEST INFRASTRUCTURE ONLY.
//
// This is a restatement of the reference's CPU path in plain C++17 (no Eigen), used
// by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg as the
// checker.  Nothing in the product library links or calls it.
//
// Parity status: the reference cannot be compiled in this environment (Eigen3,
// srrg2_core/srrg2_solver and ROS2 are absent), so no reference outputs exist.  The
// per-leaf Jacobian math is pinned by the reference's own known-answer tests
// (apps/tests/jacobians/motion_jacobian_3d_test.cpp, pose_error_jacobian_3d_test.cpp),
// re-run against this file's functions.  Tree build and solve are "parity unpinned":
// their arithmetic is fixed canonically here (see orc_tree.cpp) and the CUDA product
// is checked against that canonical definition bit-for-bit.
//
// Compile with -ffp-contract=off: every float expression below is evaluated in the
// written order with separate multiply and add roundings, which the CUDA kernels
// reproduce with __fmul_rn/__fadd_rn.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

namespace orc {

template <class T> struct V3 {
  T v[3];
  T& operator[](int i) { return v[i]; }
  const T& operator[](int i) const { return v[i]; }
};
template <class T> struct M3 {
  T a[3][3];  // row-major
};
template <class T> struct Iso {
  M3<T> R;
  V3<T> t;
};

template <class T> inline V3<T> v3(T x, T y, T z) { V3<T> r; r[0] = x; r[1] = y; r[2] = z; return r; }
template <class T> inline V3<T> vzero() { return v3<T>(0, 0, 0); }
template <class T> inline M3<T> mzero() { M3<T> m; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) m.a[i][j] = T(0); return m; }
template <class T> inline M3<T> meye() { M3<T> m = mzero<T>(); m.a[0][0] = m.a[1][1] = m.a[2][2] = T(1); return m; }

// 3-term dot product in Eigen's unrolled reduction order for fixed size 3:
// x0 + (x1 + x2)  (kd/tree/node_.h:55 and every .dot() on the path).
template <class T> inline T dot3(const V3<T>& a, const V3<T>& b) {
  T p0 = a[0] * b[0];
  T p1 = a[1] * b[1];
  T p2 = a[2] * b[2];
  return p0 + (p1 + p2);
}
template <class T> inline V3<T> vadd(const V3<T>& a, const V3<T>& b) { return v3<T>(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
template <class T> inline V3<T> vsub(const V3<T>& a, const V3<T>& b) { return v3<T>(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
template <class T> inline V3<T> vscale(const V3<T>& a, T s) { return v3<T>(a[0] * s, a[1] * s, a[2] * s); }
template <class T> inline V3<T> vneg(const V3<T>& a) { return v3<T>(-a[0], -a[1], -a[2]); }
template <class T> inline V3<T> cross(const V3<T>& a, const V3<T>& b) {
  return v3<T>(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
template <class T> inline V3<T> mrow(const M3<T>& m, int i) { return v3<T>(m.a[i][0], m.a[i][1], m.a[i][2]); }
template <class T> inline V3<T> mcol(const M3<T>& m, int j) { return v3<T>(m.a[0][j], m.a[1][j], m.a[2][j]); }

// Matrix * vector and matrix * matrix in coefficient order (each output = dot3).
template <class T> inline V3<T> mat_vec(const M3<T>& m, const V3<T>& p) {
  return v3<T>(dot3(mrow(m, 0), p), dot3(mrow(m, 1), p), dot3(mrow(m, 2), p));
}
template <class T> inline M3<T> mat_mul(const M3<T>& A, const M3<T>& B) {
  M3<T> C;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) C.a[i][j] = dot3(mrow(A, i), mcol(B, j));
  return C;
}
template <class T> inline M3<T> transpose(const M3<T>& A) {
  M3<T> C;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) C.a[i][j] = A.a[j][i];
  return C;
}
template <class T> inline M3<T> skew(const V3<T>& v) {
  M3<T> m;
  m.a[0][0] = 0;     m.a[0][1] = -v[2]; m.a[0][2] = v[1];
  m.a[1][0] = v[2];  m.a[1][1] = 0;     m.a[1][2] = -v[0];
  m.a[2][0] = -v[1]; m.a[2][1] = v[0];  m.a[2][2] = 0;
  return m;
}

// applyIsometry_ / applyRotation_ (kd/utils/geometry_.h:11-37): explicit row loop
// returned(r) = ((t_r + X_r0 p0) + X_r1 p1) + X_r2 p2, with t = 0 for rotations.
template <class T> inline V3<T> apply_iso(const Iso<T>& X, const V3<T>& p) {
  V3<T> r;
  for (int i = 0; i < 3; ++i) {
    T acc = X.t[i];
    for (int c = 0; c < 3; ++c) acc = acc + X.R.a[i][c] * p[c];
    r[i] = acc;
  }
  return r;
}
template <class T> inline V3<T> apply_rot(const Iso<T>& X, const V3<T>& p) {
  V3<T> r;
  for (int i = 0; i < 3; ++i) {
    T acc = T(0);
    for (int c = 0; c < 3; ++c) acc = acc + X.R.a[i][c] * p[c];
    r[i] = acc;
  }
  return r;
}

template <class T> inline Iso<T> iso_identity() { Iso<T> X; X.R = meye<T>(); X.t = vzero<T>(); return X; }
// Isometry inverse and product as Eigen's Transform does them (linear block first).
template <class T> inline Iso<T> iso_inverse(const Iso<T>& X) {
  Iso<T> r;
  r.R = transpose(X.R);
  r.t = vneg(mat_vec(r.R, X.t));
  return r;
}
template <class T> inline Iso<T> iso_mul(const Iso<T>& A, const Iso<T>& B) {
  Iso<T> r;
  r.R = mat_mul(A.R, B.R);
  r.t = vadd(mat_vec(A.R, B.t), A.t);
  return r;
}
template <class Tout, class Tin> inline Iso<Tout> iso_cast(const Iso<Tin>& X) {
  Iso<Tout> r;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) r.R.a[i][j] = (Tout)X.R.a[i][j];
    r.t[i] = (Tout)X.t[i];
  }
  return r;
}
// 3x4 row-major packing [R | t] used across the C ABI.
template <class T, class S> inline Iso<T> iso_from12(const S* m) {
  Iso<T> r;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) r.R.a[i][j] = (T)m[i * 4 + j];
    r.t[i] = (T)m[i * 4 + 3];
  }
  return r;
}
template <class T, class S> inline void iso_to12(const Iso<T>& X, S* m) {
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) m[i * 4 + j] = (S)X.R.a[i][j];
    m[i * 4 + 3] = (S)X.t[i];
  }
}

// ---------------------------------------------------------------------------
// Canonical single-precision sine/cosine.  The reference calls sinf/cosf
// (kd/utils/geometry_3d_impl_.h:26) whose last bit differs between libm builds;
// the CT warp feeds the tree descent, so CPU and GPU use this one definition:
// Cody-Waite reduction by pi/2 with a three-part constant (Cody & Waite 1980,
// "Software Manual for the Elementary Functions"), then Taylor polynomials on
// [-pi/4, pi/4] evaluated in Horner form.  Accuracy <= 2 ulp for |x| < 400.
inline void sincos_canon(float x, float* s_out, float* c_out) {
  const float two_over_pi = 0.636619772367581343f;
  float q = std::nearbyint(x * two_over_pi);
  int j = (int)q;
  float r = x - q * 1.5703125f;
  r = r - q * 4.837512969970703125e-4f;
  r = r - q * 7.54978995489188216e-8f;
  float r2 = r * r;
  float t = r2 * 2.75573192e-6f;
  t = -1.98412698e-4f + t;
  t = r2 * t;
  t = 8.33333333e-3f + t;
  t = r2 * t;
  t = -1.66666667e-1f + t;
  t = r2 * t;
  float sn = r + r * t;
  float u = r2 * -2.75573192e-7f;
  u = 2.48015873e-5f + u;
  u = r2 * u;
  u = -1.38888889e-3f + u;
  u = r2 * u;
  u = 4.16666667e-2f + u;
  u = r2 * u;
  u = -0.5f + u;
  u = r2 * u;
  float cs = 1.0f + u;
  switch (j & 3) {
    case 0: *s_out = sn; *c_out = cs; break;
    case 1: *s_out = cs; *c_out = -sn; break;
    case 2: *s_out = -sn; *c_out = -cs; break;
    default: *s_out = -cs; *c_out = sn; break;
  }
}
inline void sincos_t(float x, float* s, float* c) { sincos_canon(x, s, c); }
inline void sincos_t(double x, double* s, double* c) { *s = std::sin(x); *c = std::cos(x); }

// Canonical double-precision sine/cosine of the product's FP64 pose update
// (kd_slam2_b200/csrc/kds_align.cu, sincos_canon_d), restated so that MODE_MIXED's
// expmap is bit-identical to the GPU's: Cody-Waite reduction by pi/2 with a three-part
// constant of 33 + 33 + 53 bits, then the Taylor series of sin to r^17 and of cos to
// r^18 in Horner form.  Within 2 ulp of libm (tests/test_oracle_pins.py).
inline void sincos_canon_d(double x, double* s_out, double* c_out) {
  const double q = std::nearbyint(x * 0x1.45f306dc9c883p-1);
  const long long j = (long long)q;
  double r = x - q * 0x1.921fb54400000p+0;
  r = r - q * 0x1.0b4611a600000p-34;
  r = r - q * 0x1.3198a2e037073p-69;
  const double r2 = r * r;
  double t = 0x1.952c77030ad4ap-49;
  t = -0x1.ae7f3e733b81fp-41 + r2 * t;
  t = 0x1.6124613a86d09p-33 + r2 * t;
  t = -0x1.ae64567f544e4p-26 + r2 * t;
  t = 0x1.71de3a556c734p-19 + r2 * t;
  t = -0x1.a01a01a01a01ap-13 + r2 * t;
  t = 0x1.1111111111111p-7 + r2 * t;
  t = -0x1.5555555555555p-3 + r2 * t;
  const double sn = r + r * (r2 * t);
  double u = -0x1.6827863b97d97p-53;
  u = 0x1.ae7f3e733b81fp-45 + r2 * u;
  u = -0x1.93974a8c07c9dp-37 + r2 * u;
  u = 0x1.1eed8eff8d898p-29 + r2 * u;
  u = -0x1.27e4fb7789f5cp-22 + r2 * u;
  u = 0x1.a01a01a01a01ap-16 + r2 * u;
  u = -0x1.6c16c16c16c17p-10 + r2 * u;
  u = 0x1.5555555555555p-5 + r2 * u;
  u = -0.5 + r2 * u;
  const double cs = 1.0 + r2 * u;
  switch ((int)(j & 3)) {
    case 0: *s_out = sn; *c_out = cs; break;
    case 1: *s_out = cs; *c_out = -sn; break;
    case 2: *s_out = -sn; *c_out = -cs; break;
    default: *s_out = -cs; *c_out = sn; break;
  }
}

// ---------------------------------------------------------------------------
// GeometryTraits_<3> restated (kd/utils/geometry_3d_impl_.h).
template <class T> inline M3<T> rodrigues_angle(T s, T c, const M3<T>& S, const M3<T>& S2) {
  // Identity() + sin(a)*S + (1-cos(a))*S2, evaluated element-wise left to right.
  M3<T> R;
  T omc = T(1) - c;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      T id = (i == j) ? T(1) : T(0);
      R.a[i][j] = (id + s * S.a[i][j]) + omc * S2.a[i][j];
    }
  return R;
}
// rodrigues(w), geometry_3d_impl_.h:37-46
template <class T> inline M3<T> rodrigues(const V3<T>& w) {
  T angle = std::sqrt(dot3(w, w));
  if (angle < T(1e-9)) return meye<T>();
  T inv = T(1) / angle;
  V3<T> n = vscale(w, inv);
  M3<T> S = skew(n);
  M3<T> S2 = mat_mul(S, S);
  T s, c;
  sincos_t(angle, &s, &c);
  return rodrigues_angle(s, c, S, S2);
}
// dRxp(ur, dR, w, u), geometry_3d_impl_.h:143-174 (Gallego & Yezzi 2014)
template <class T> inline void dRxp(V3<T>& ur, M3<T>& dR, const V3<T>& w, const V3<T>& u) {
  T angle = std::sqrt(dot3(w, w));
  if (angle < T(1e-9)) {
    ur = u;
    M3<T> su = skew(u);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) dR.a[i][j] = -su.a[i][j];
    return;
  }
  T inv = T(1) / angle;
  V3<T> n = vscale(w, inv);
  M3<T> S = skew(n);
  M3<T> S2 = mat_mul(S, S);
  T s, c;
  sincos_t(angle, &s, &c);
  M3<T> R = rodrigues_angle(s, c, S, S2);
  ur = mat_vec(R, u);
  // -R * skew(u) * (n n^T + (R^T - I) * S * (1/angle))
  M3<T> nnT;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) nnT.a[i][j] = n[i] * n[j];
  M3<T> RtmI = transpose(R);
  for (int i = 0; i < 3; ++i) RtmI.a[i][i] = RtmI.a[i][i] - T(1);
  M3<T> A = mat_mul(RtmI, S);
  M3<T> inner;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) inner.a[i][j] = nnT.a[i][j] + A.a[i][j] * inv;
  M3<T> su = skew(u);
  M3<T> Rs = mat_mul(R, su);
  M3<T> P = mat_mul(Rs, inner);
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) dR.a[i][j] = -P.a[i][j];
}
// expmap (geometry_3d_impl_.h:176-184): decoupled, t = v[0:3], R = rodrigues(v[3:6])
template <class T> inline Iso<T> expmap(const T* v) {
  Iso<T> X;
  X.t = v3<T>(v[0], v[1], v[2]);
  X.R = rodrigues(v3<T>(v[3], v[4], v[5]));
  return X;
}
// The same in FP64 with the canonical sine/cosine (MODE_MIXED: the product's pose update).
inline Iso<double> expmap_canon(const double* v) {
  Iso<double> X;
  X.t = v3<double>(v[0], v[1], v[2]);
  V3<double> w = v3<double>(v[3], v[4], v[5]);
  double angle = std::sqrt(dot3(w, w));
  if (angle < 1e-9) {
    X.R = meye<double>();
    return X;
  }
  double inv = 1.0 / angle;
  M3<double> S = skew(vscale(w, inv));
  M3<double> S2 = mat_mul(S, S);
  double s, c;
  sincos_canon_d(angle, &s, &c);
  X.R = rodrigues_angle(s, c, S, S2);
  return X;
}

// The product's FP64 solve (kd_slam2_b200/csrc/kds_align.cu, tail_warp): Cholesky of
// the lower triangle of A (n <= 12) by column sweeps -- per pivot one square root and one
// reciprocal, the column scaled by it, the trailing triangle updated -- then L y = rhs
// and L^T x = y by column sweeps.  Returns false (x = 0) when a pivot is not positive.
inline bool chol_solve_cols(int n, const double* A_in, const double* rhs, double* x) {
  double A[12][12], inv[12], y[12];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) A[i][j] = A_in[i * n + j];
  bool ok = true;
  for (int k = 0; k < n; ++k) {
    double d = A[k][k];
    ok = ok && (d > 0.0);
    double lkk = std::sqrt(std::fmax(d, 1e-300));
    double iv = 1.0 / lkk;
    for (int i = k + 1; i < n; ++i) A[i][k] = A[i][k] * iv;
    A[k][k] = lkk;
    inv[k] = iv;
    for (int i = k + 1; i < n; ++i)
      for (int j = k + 1; j <= i; ++j) A[i][j] = A[i][j] - A[i][k] * A[j][k];
  }
  for (int i = 0; i < n; ++i) y[i] = rhs[i];
  for (int k = 0; k < n; ++k) {
    const double yk = y[k] * inv[k];
    y[k] = yk;
    for (int i = k + 1; i < n; ++i) y[i] = y[i] - A[i][k] * yk;
  }
  for (int k = n - 1; k >= 0; --k) {
    const double xk = y[k] * inv[k];
    y[k] = xk;
    for (int i = 0; i < k; ++i) y[i] = y[i] - A[k][i] * xk;
  }
  for (int i = 0; i < n; ++i) x[i] = ok ? y[i] : 0.0;
  return ok;
}
// logSO3 (geometry_3d_impl_.h:48-59)
template <class T> inline V3<T> logSO3(const M3<T>& R) {
  T tr = R.a[0][0] + R.a[1][1] + R.a[2][2];
  T cos_a = T(0.5) * (tr - T(1));
  cos_a = std::max(T(-1), std::min(T(1), cos_a));
  T angle = std::acos(cos_a);
  V3<T> ax = v3<T>(R.a[2][1] - R.a[1][2], R.a[0][2] - R.a[2][0], R.a[1][0] - R.a[0][1]);
  if (angle < T(1e-7)) return vscale(ax, T(0.5));
  return vscale(ax, angle / (T(2) * std::sin(angle)));
}
template <class T> inline void logmap(const Iso<T>& X, T* out6) {
  V3<T> w = logSO3(X.R);
  for (int i = 0; i < 3; ++i) { out6[i] = X.t[i]; out6[3 + i] = w[i]; }
}
// dlogSO3 (geometry_3d_impl_.h:75-105), 3x9, column-major coefficient order of R
template <class T> inline void dlogSO3(const M3<T>& R, T J[3][9]) {
  V3<T> ax = v3<T>(R.a[2][1] - R.a[1][2], R.a[0][2] - R.a[2][0], R.a[1][0] - R.a[0][1]);
  T tr = R.a[0][0] + R.a[1][1] + R.a[2][2];
  T cos_a = T(0.5) * (tr - T(1));
  cos_a = std::max(T(-1), std::min(T(1), cos_a));
  T angle = std::acos(cos_a);
  bool small = angle < T(1e-7);
  T f = small ? T(0.5) : angle / (T(2) * std::sin(angle));
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 9; ++j) J[i][j] = T(0);
  J[0][5] = f;  J[0][7] = -f;
  J[1][6] = f;  J[1][2] = -f;
  J[2][1] = f;  J[2][3] = -f;
  if (!small) {
    T s = std::sin(angle);
    T c = (s - angle * std::cos(angle)) / (T(4) * s * s * s);
    for (int k = 0; k < 3; ++k) {
      J[k][0] -= c * ax[k];
      J[k][4] -= c * ax[k];
      J[k][8] -= c * ax[k];
    }
  }
}
// poseToPoseError / dPoseToPoseError (geometry_3d_impl_.h:117-140)
template <class T> inline void pose_to_pose_error(const Iso<T>& ZXi, const Iso<T>& Xm, T* e6) {
  logmap(iso_mul(ZXi, Xm), e6);
}
template <class T> inline void dpose_to_pose_error(const Iso<T>& ZXi, const Iso<T>& Xm, T Jout[6][6]) {
  Iso<T> P = iso_mul(ZXi, Xm);
  const M3<T>& R = ZXi.R;
  const V3<T>& t = Xm.t;
  T B[12][6];
  for (int i = 0; i < 12; ++i) for (int j = 0; j < 6; ++j) B[i][j] = T(0);
  M3<T> Rst = mat_mul(R, skew(t));
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) { B[i][j] = R.a[i][j]; B[i][3 + j] = -Rst.a[i][j]; }
  for (int k = 0; k < 3; ++k) {
    M3<T> Rsk = mat_mul(R, skew(mcol(Xm.R, k)));
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) B[3 + 3 * k + i][3 + j] = -Rsk.a[i][j];
  }
  // dlogmap(P) (6x12) * B
  T Dl[6][12];
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 12; ++j) Dl[i][j] = T(0);
  for (int i = 0; i < 3; ++i) Dl[i][i] = T(1);
  T Js[3][9];
  dlogSO3(P.R, Js);
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 9; ++j) Dl[3 + i][3 + j] = Js[i][j];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      T acc = T(0);
      for (int k = 0; k < 12; ++k) acc += Dl[i][k] * B[k][j];
      Jout[i][j] = acc;
    }
}

// ---------------------------------------------------------------------------
// Symmetric LDL^T with diagonal pivoting (Golub & Van Loan, "Matrix Computations",
// symmetric pivoting by largest remaining diagonal).  Solves (A) x = rhs for n <= 18.
template <class T> inline bool ldlt_solve(int n, const T* A_in, const T* rhs, T* x) {
  T A[18][18];
  int perm[18];
  for (int i = 0; i < n; ++i) {
    perm[i] = i;
    for (int j = 0; j < n; ++j) A[i][j] = A_in[i * n + j];
  }
  T L[18][18];
  T D[18];
  for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) L[i][j] = (i == j) ? T(1) : T(0);
  for (int k = 0; k < n; ++k) {
    int p = k;
    T best = std::fabs(A[k][k]);
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(A[i][i]) > best) { best = std::fabs(A[i][i]); p = i; }
    if (p != k) {
      for (int j = 0; j < n; ++j) { T tmp = A[k][j]; A[k][j] = A[p][j]; A[p][j] = tmp; }
      for (int i = 0; i < n; ++i) { T tmp = A[i][k]; A[i][k] = A[i][p]; A[i][p] = tmp; }
      for (int j = 0; j < k; ++j) { T tmp = L[k][j]; L[k][j] = L[p][j]; L[p][j] = tmp; }
      int tp = perm[k]; perm[k] = perm[p]; perm[p] = tp;
    }
    T d = A[k][k];
    D[k] = d;
    if (d == T(0)) return false;
    for (int i = k + 1; i < n; ++i) L[i][k] = A[i][k] / d;
    for (int i = k + 1; i < n; ++i)
      for (int j = k + 1; j <= i; ++j) {
        A[i][j] = A[i][j] - L[i][k] * d * L[j][k];
        A[j][i] = A[i][j];
      }
  }
  T y[18];
  for (int i = 0; i < n; ++i) y[i] = rhs[perm[i]];
  for (int i = 0; i < n; ++i) {
    T acc = y[i];
    for (int j = 0; j < i; ++j) acc -= L[i][j] * y[j];
    y[i] = acc;
  }
  for (int i = 0; i < n; ++i) y[i] = y[i] / D[i];
  for (int i = n - 1; i >= 0; --i) {
    T acc = y[i];
    for (int j = i + 1; j < n; ++j) acc -= L[j][i] * y[j];
    y[i] = acc;
  }
  for (int i = 0; i < n; ++i) x[perm[i]] = y[i];
  return true;
}

}  // namespace orc
