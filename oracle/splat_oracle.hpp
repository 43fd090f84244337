// CPU oracle for the splatrs render-and-train hot path. TEST INFRASTRUCTURE ONLY: the
// product never links or calls this code; tests, the smoke check and the CPU-baseline
// leg of the benchmark use it as the checker.
//
// This is a restatement, in C++17, of the reference implementation's Rust code
// (harryprayiv/splatrs). Every function keeps the reference's operation order so that,
// with -ffp-contract=off, the float instantiation reproduces the reference's f32 results
// and the double instantiation reproduces its `--features f64` build (the FP64 gradient
// check oracle). Each function cites the reference file:line it follows.
//
// Transcendentals: the reference calls the platform libm through Rust's f32::exp / f32::ln
// (glibc expf/logf on Linux). `Math::cr` switches the float instantiation to the correctly
// rounded exp/log that the CUDA kernels use; the default (false) is the faithful libm path.
//
// Parity status: the reference ships no golden vectors and cannot be built here (no Rust
// toolchain), so this oracle is pinned by replaying the reference's own tests against it:
// the finite-difference gradient checks, the tiled-versus-naive compositing equivalence,
// the unit tests with exact answers and the training-improvement tests.
#pragma once
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <thread>
#include <utility>
#include <vector>

#include "../splatrs_b200/csrc/crmath.h"

namespace ora {

// ---------------------------------------------------------------------------------------
// Thread pool: a stand-in for rayon's global pool (reference src/main.rs:122-127).
// ---------------------------------------------------------------------------------------
int num_threads();
void set_num_threads(int n);
// Run f(i) for i in [0, n) on the pool, in chunks of `grain` claimed dynamically.
void parallel_for(int64_t n, int64_t grain, const std::function<void(int64_t, int64_t)>& f);

// ---------------------------------------------------------------------------------------
// Scalars and literals. A literal is written as the float literal in the f32 build and
// the double literal in the f64 build, exactly as Rust parses `0.3` for each `Real`.
// ---------------------------------------------------------------------------------------
#define ORA_L(x) ((Real)(sizeof(Real) == 4 ? (double)(x##f) : (double)(x)))

struct Math {
  static bool cr;  // use the correctly rounded exp/log in the f32 build
};

inline float rexp(float x) { return Math::cr ? crm::expf_cr(x) : std::exp(x); }
inline double rexp(double x) { return std::exp(x); }
inline float rln(float x) { return Math::cr ? crm::logf_cr(x) : std::log(x); }
inline double rln(double x) { return std::log(x); }

// Rust's float max/min (NaN operand yields the other operand), clamp (NaN propagates)
// and the saturating `as u32` cast (NaN and negatives to 0).
template <class R> inline R rmax(R a, R b) { return std::fmax(a, b); }
template <class R> inline R rmin(R a, R b) { return std::fmin(a, b); }
template <class R> inline R rclamp(R v, R lo, R hi) {
  if (v != v) return v;
  return v < lo ? lo : (v > hi ? hi : v);
}
template <class R> inline uint32_t as_u32(R v) {
  if (!(v > (R)0)) return 0;
  if (v >= (R)4294967295.0) return 0xffffffffu;
  return (uint32_t)v;
}
inline uint32_t f32_bits(float f) {
  uint32_t b;
  std::memcpy(&b, &f, 4);
  return b;
}

// ---------------------------------------------------------------------------------------
// src/math.rs: V3, M3 (row major), Quat (w, x, y, z).
// ---------------------------------------------------------------------------------------
template <class Real> struct V3 {
  Real x, y, z;
  V3() : x(0), y(0), z(0) {}
  V3(Real a, Real b, Real c) : x(a), y(b), z(c) {}
  Real dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }  // math.rs:105
  V3 cross(const V3& o) const {                                           // math.rs:110
    return V3(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x);
  }
  Real norm2() const { return dot(*this); }
  Real norm() const { return std::sqrt(norm2()); }
  V3 normalized() const {                                                 // math.rs:129
    Real n = norm();
    if (n > (Real)0) return (*this) * ((Real)1 / n);
    return *this;
  }
  V3 exp() const { return V3(rexp(x), rexp(y), rexp(z)); }
  Real max_elem() const { return rmax(rmax(x, y), z); }                  // math.rs:149
  Real get(int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
  V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
  V3 operator*(Real s) const { return V3(x * s, y * s, z * s); }
  V3 operator-() const { return V3(-x, -y, -z); }
  V3& operator+=(const V3& o) {
    x += o.x;
    y += o.y;
    z += o.z;
    return *this;
  }
};

template <class Real> struct M3 {
  Real m[3][3];
  M3() { std::memset(m, 0, sizeof(m)); }
  static M3 from_rows(const V3<Real>& r0, const V3<Real>& r1, const V3<Real>& r2) {
    M3 r;
    const V3<Real>* rows[3] = {&r0, &r1, &r2};
    for (int i = 0; i < 3; i++) {
      r.m[i][0] = rows[i]->x;
      r.m[i][1] = rows[i]->y;
      r.m[i][2] = rows[i]->z;
    }
    return r;
  }
  V3<Real> row(int i) const { return V3<Real>(m[i][0], m[i][1], m[i][2]); }
  V3<Real> col(int j) const { return V3<Real>(m[0][j], m[1][j], m[2][j]); }
  V3<Real> mul_v(const V3<Real>& v) const {                               // math.rs:233
    return V3<Real>(row(0).dot(v), row(1).dot(v), row(2).dot(v));
  }
  M3 mul_m(const M3& o) const {                                          // math.rs:238
    M3 r;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        Real s = 0;
        for (int k = 0; k < 3; k++) s += m[i][k] * o.m[k][j];
        r.m[i][j] = s;
      }
    return r;
  }
  M3 transpose() const {
    M3 r;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) r.m[i][j] = m[j][i];
    return r;
  }
  M3 scale_cols(const V3<Real>& s) const {                                // math.rs:264
    M3 r = *this;
    for (int i = 0; i < 3; i++) {
      r.m[i][0] *= s.x;
      r.m[i][1] *= s.y;
      r.m[i][2] *= s.z;
    }
    return r;
  }
  M3 scaled(Real s) const {
    M3 r = *this;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) r.m[i][j] *= s;
    return r;
  }
  Real frob_dot(const M3& o) const {                                     // math.rs:286
    Real s = 0;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) s += m[i][j] * o.m[i][j];
    return s;
  }
};

template <class Real> struct Quat {
  Real w, x, y, z;
  Real norm() const { return std::sqrt(w * w + x * x + y * y + z * z); }  // math.rs:348
  Quat normalized() const {                                               // math.rs:353
    Real n = norm();
    if (n > (Real)0) return Quat{w / n, x / n, y / n, z / n};
    return Quat{1, 0, 0, 0};
  }
  M3<Real> to_mat() const {                                               // math.rs:368-389
    M3<Real> r;
    const Real one = 1, two = 2;
    r.m[0][0] = one - two * (y * y + z * z);
    r.m[0][1] = two * (x * y - w * z);
    r.m[0][2] = two * (x * z + w * y);
    r.m[1][0] = two * (x * y + w * z);
    r.m[1][1] = one - two * (x * x + z * z);
    r.m[1][2] = two * (y * z - w * x);
    r.m[2][0] = two * (x * z - w * y);
    r.m[2][1] = two * (y * z + w * x);
    r.m[2][2] = one - two * (x * x + y * y);
    return r;
  }
};

// math.rs:395-431
template <class Real>
void quat_to_mat_backward(const Quat<Real>& q, const M3<Real>& dr, Real out[4]) {
  const Real w = q.w, x = q.x, y = q.y, z = q.z;
  const Real t2 = 2, t4 = 4;
  M3<Real> a, b, c, d;
  a.m[0][0] = 0;        a.m[0][1] = -t2 * z;  a.m[0][2] = t2 * y;
  a.m[1][0] = t2 * z;   a.m[1][1] = 0;        a.m[1][2] = -t2 * x;
  a.m[2][0] = -t2 * y;  a.m[2][1] = t2 * x;   a.m[2][2] = 0;
  b.m[0][0] = 0;        b.m[0][1] = t2 * y;   b.m[0][2] = t2 * z;
  b.m[1][0] = t2 * y;   b.m[1][1] = -t4 * x;  b.m[1][2] = -t2 * w;
  b.m[2][0] = t2 * z;   b.m[2][1] = t2 * w;   b.m[2][2] = -t4 * x;
  c.m[0][0] = -t4 * y;  c.m[0][1] = t2 * x;   c.m[0][2] = t2 * w;
  c.m[1][0] = t2 * x;   c.m[1][1] = 0;        c.m[1][2] = t2 * z;
  c.m[2][0] = -t2 * w;  c.m[2][1] = t2 * z;   c.m[2][2] = -t4 * y;
  d.m[0][0] = -t4 * z;  d.m[0][1] = -t2 * w;  d.m[0][2] = t2 * x;
  d.m[1][0] = t2 * w;   d.m[1][1] = -t4 * z;  d.m[1][2] = t2 * y;
  d.m[2][0] = t2 * x;   d.m[2][1] = t2 * y;   d.m[2][2] = 0;
  out[0] = dr.frob_dot(a);
  out[1] = dr.frob_dot(b);
  out[2] = dr.frob_dot(c);
  out[3] = dr.frob_dot(d);
}

// math.rs:434-446
template <class Real>
void normalize_backward(const Real raw[4], const Real d_unit[4], Real out[4]) {
  Real n = std::sqrt(raw[0] * raw[0] + raw[1] * raw[1] + raw[2] * raw[2] + raw[3] * raw[3]);
  if (n <= (Real)0) {
    for (int i = 0; i < 4; i++) out[i] = 0;
    return;
  }
  Real u[4] = {raw[0] / n, raw[1] / n, raw[2] / n, raw[3] / n};
  Real dot = u[0] * d_unit[0] + u[1] * d_unit[1] + u[2] * d_unit[2] + u[3] * d_unit[3];
  for (int i = 0; i < 4; i++) out[i] = (d_unit[i] - u[i] * dot) / n;
}

template <class Real> Real sigmoid(Real x) { return (Real)1 / ((Real)1 + rexp(-x)); }  // math.rs:449
template <class Real> Real inverse_sigmoid(Real x) { return rln(x / ((Real)1 - x)); }    // math.rs:454

// ---------------------------------------------------------------------------------------
// src/sh.rs: real spherical harmonics to degree 3.
// ---------------------------------------------------------------------------------------
constexpr int MAX_COEFFS = 16;
constexpr int MAX_DEGREE = 3;
inline int num_coeffs(int degree) { return (degree + 1) * (degree + 1); }

template <class Real> struct SH {
  // sh.rs:16-33: f64 literals rounded to Real.
  static constexpr Real C0 = (Real)0.28209479177387814;
  static constexpr Real C1 = (Real)0.4886025119029199;
  static constexpr Real C2[5] = {(Real)1.0925484305920792, (Real)-1.0925484305920792,
                                 (Real)0.31539156525252005, (Real)-1.0925484305920792,
                                 (Real)0.5462742152960396};
  static constexpr Real C3[7] = {(Real)-0.5900435899266435, (Real)2.890611442640554,
                                 (Real)-0.4570457994644658, (Real)0.3731763325901154,
                                 (Real)-0.4570457994644658, (Real)1.445305721320277,
                                 (Real)-0.5900435899266435};
};

template <class Real> Real rgb_to_sh(Real c) { return (c - ORA_L(0.5)) / SH<Real>::C0; }  // sh.rs:41

// sh.rs:47-75
template <class Real> void sh_basis(int degree, const V3<Real>& dir, Real b[MAX_COEFFS]) {
  for (int i = 0; i < MAX_COEFFS; i++) b[i] = 0;
  const Real x = dir.x, y = dir.y, z = dir.z;
  typedef SH<Real> S;
  b[0] = S::C0;
  if (degree >= 1) {
    b[1] = -S::C1 * y;
    b[2] = S::C1 * z;
    b[3] = -S::C1 * x;
  }
  if (degree >= 2) {
    const Real xx = x * x, yy = y * y, zz = z * z;
    const Real xy = x * y, yz = y * z, xz = x * z;
    const Real two = 2, three = 3, four = 4;
    b[4] = S::C2[0] * xy;
    b[5] = S::C2[1] * yz;
    b[6] = S::C2[2] * (two * zz - xx - yy);
    b[7] = S::C2[3] * xz;
    b[8] = S::C2[4] * (xx - yy);
    if (degree >= 3) {
      b[9] = S::C3[0] * y * (three * xx - yy);
      b[10] = S::C3[1] * xy * z;
      b[11] = S::C3[2] * y * (four * zz - xx - yy);
      b[12] = S::C3[3] * z * (two * zz - three * xx - three * yy);
      b[13] = S::C3[4] * x * (four * zz - xx - yy);
      b[14] = S::C3[5] * z * (xx - yy);
      b[15] = S::C3[6] * x * (xx - three * yy);
    }
  }
}

// sh.rs:80-130
template <class Real> void sh_basis_grad(int degree, const V3<Real>& dir, V3<Real> g[MAX_COEFFS]) {
  for (int i = 0; i < MAX_COEFFS; i++) g[i] = V3<Real>();
  const Real x = dir.x, y = dir.y, z = dir.z;
  typedef SH<Real> S;
  typedef V3<Real> V;
  const Real two = 2, three = 3, four = 4, six = 6, eight = 8;
  if (degree >= 1) {
    g[1] = V(0, -S::C1, 0);
    g[2] = V(0, 0, S::C1);
    g[3] = V(-S::C1, 0, 0);
  }
  if (degree >= 2) {
    const Real xx = x * x, yy = y * y, zz = z * z;
    g[4] = V(S::C2[0] * y, S::C2[0] * x, 0);
    g[5] = V(0, S::C2[1] * z, S::C2[1] * y);
    g[6] = V(-two * S::C2[2] * x, -two * S::C2[2] * y, four * S::C2[2] * z);
    g[7] = V(S::C2[3] * z, 0, S::C2[3] * x);
    g[8] = V(two * S::C2[4] * x, -two * S::C2[4] * y, 0);
    if (degree >= 3) {
      g[9] = V(S::C3[0] * six * x * y, S::C3[0] * (three * xx - three * yy), 0);
      g[10] = V(S::C3[1] * y * z, S::C3[1] * x * z, S::C3[1] * x * y);
      g[11] = V(S::C3[2] * (-two * x * y), S::C3[2] * (four * zz - xx - three * yy),
                S::C3[2] * eight * y * z);
      g[12] = V(S::C3[3] * (-six * x * z), S::C3[3] * (-six * y * z),
                S::C3[3] * (six * zz - three * xx - three * yy));
      g[13] = V(S::C3[4] * (four * zz - three * xx - yy), S::C3[4] * (-two * x * y),
                S::C3[4] * eight * x * z);
      g[14] = V(S::C3[5] * two * x * z, -S::C3[5] * two * y * z, S::C3[5] * (xx - yy));
      g[15] = V(S::C3[6] * (three * xx - three * yy), S::C3[6] * (-six * x * y), 0);
    }
  }
}

// ---------------------------------------------------------------------------------------
// src/camera.rs
// ---------------------------------------------------------------------------------------
template <class Real> struct Camera {
  uint32_t width = 0, height = 0;
  Real fx = 0, fy = 0, cx = 0, cy = 0;
  M3<Real> rot;
  V3<Real> trans;
  V3<Real> world_to_cam(const V3<Real>& p) const { return rot.mul_v(p) + trans; }  // camera.rs:36
  V3<Real> center() const { return -(rot.transpose().mul_v(trans)); }            // camera.rs:41
  // camera.rs:66-93
  static Camera look_at(uint32_t w, uint32_t h, Real fx, Real fy, V3<Real> eye, V3<Real> target,
                        V3<Real> up) {
    V3<Real> forward = (target - eye).normalized();
    V3<Real> right = forward.cross(up).normalized();
    V3<Real> down = forward.cross(right);
    Camera c;
    c.width = w;
    c.height = h;
    c.fx = fx;
    c.fy = fy;
    c.cx = (Real)w / (Real)2;
    c.cy = (Real)h / (Real)2;
    c.rot = M3<Real>::from_rows(right, down, forward);
    c.trans = -(c.rot.mul_v(eye));
    return c;
  }
};

// camera.rs:99-118
template <class Real> Real scene_extent(const std::vector<Camera<Real>>& cams) {
  if (cams.empty()) return 1;
  V3<Real> center;
  for (const auto& c : cams) center += c.center();
  center = center * ((Real)1 / (Real)cams.size());
  Real radius = 0;
  for (const auto& c : cams) radius = rmax(radius, (c.center() - center).norm());
  Real extent = radius * ORA_L(1.1);
  return extent > (Real)0 ? extent : (Real)1;
}

// ---------------------------------------------------------------------------------------
// src/model.rs: the 59-scalar parameter record.
// ---------------------------------------------------------------------------------------
constexpr int NUM_PARAMS = 59;
template <class Real> struct Gaussian {
  Real mean[3];
  Real log_scale[3];
  Real quat[4];
  Real opacity;
  Real sh[MAX_COEFFS][3];
  V3<Real> mean_v() const { return V3<Real>(mean[0], mean[1], mean[2]); }
  V3<Real> scales() const { return V3<Real>(log_scale[0], log_scale[1], log_scale[2]).exp(); }
  Quat<Real> rotation() const { return Quat<Real>{quat[0], quat[1], quat[2], quat[3]}.normalized(); }
  Real alpha() const { return sigmoid(opacity); }
};
static_assert(sizeof(Gaussian<float>) == 59 * 4, "Gaussian record must be 59 packed scalars");
static_assert(sizeof(Gaussian<double>) == 59 * 8, "Gaussian record must be 59 packed scalars");

template <class Real> inline Gaussian<Real> zero_gaussian() {
  Gaussian<Real> g;
  std::memset(&g, 0, sizeof(g));
  return g;
}

// model.rs:113-121
template <class T> void retain_by_mask(std::vector<T>& v, const std::vector<char>& keep) {
  size_t j = 0;
  for (size_t i = 0; i < v.size(); i++)
    if (keep[i]) v[j++] = v[i];
  v.resize(j);
}

// ---------------------------------------------------------------------------------------
// src/project.rs
// ---------------------------------------------------------------------------------------
constexpr uint32_t TILE = 16;  // project.rs:18

template <class Real> struct ProjOpts {  // project.rs:22-43
  Real near_ = ORA_L(0.2);
  Real eps2d = ORA_L(0.3);
  bool antialias = false;
  int sh_degree = 3;
};

template <class Real> struct Proj {  // project.rs:47-64
  Real mean2d[2] = {0, 0};
  Real conic[3] = {0, 0, 0};
  Real depth = 0;
  uint32_t radius = 0;
  Real opacity = 0;
  Real color[3] = {0, 0, 0};
  uint32_t tile_min[2] = {0, 0};
  uint32_t tile_max[2] = {0, 0};
  bool visible() const { return radius > 0; }
  uint32_t num_tiles() const {
    if (radius == 0) return 0;
    return (tile_max[0] - tile_min[0]) * (tile_max[1] - tile_min[1]);
  }
};

template <class Real> struct ProjGrad {  // project.rs:84-93
  Real mean2d[2] = {0, 0};
  Real conic[3] = {0, 0, 0};
  Real opacity = 0;
  Real color[3] = {0, 0, 0};
};

template <class Real> struct Core {  // project.rs:96-125
  V3<Real> t;
  Real txc, tyc;
  bool clamped_x, clamped_y;
  V3<Real> s;
  Quat<Real> q;
  M3<Real> rq, m, sigma;
  Real tmat[2][3];
  Real a0, b0, c0, det0, a, b, c, det;
  Real conic[3];
  Real comp;
  Real mean2d[2];
  Real radius;
  Real o_raw;
  V3<Real> dir;
  Real dist;
  Real basis[MAX_COEFFS];
  Real color_raw[3];
};

template <class Real> inline Real clamp_flag(Real v, Real lo, Real hi, bool* flag) {  // project.rs:127
  if (v < lo) {
    *flag = true;
    return lo;
  }
  if (v > hi) {
    *flag = true;
    return hi;
  }
  *flag = false;
  return v;
}

// project.rs:137-269. Returns false when the Gaussian is culled.
template <class Real>
bool core(const Gaussian<Real>& g, const Camera<Real>& cam, const ProjOpts<Real>& opts, Core<Real>& k) {
  V3<Real> p = g.mean_v();
  V3<Real> t = cam.world_to_cam(p);
  if (t.z != t.z || t.z <= opts.near_) return false;
  V3<Real> s = g.scales();
  Quat<Real> q = g.rotation();
  M3<Real> rq = q.to_mat();
  M3<Real> m = rq.scale_cols(s);
  M3<Real> sigma = m.mul_m(m.transpose());

  const Real W = (Real)cam.width, H = (Real)cam.height;
  Real tan_x = ORA_L(0.5) * W / cam.fx;
  Real tan_y = ORA_L(0.5) * H / cam.fy;
  Real lim_x_pos = (W - cam.cx) / cam.fx + ORA_L(0.3) * tan_x;
  Real lim_x_neg = cam.cx / cam.fx + ORA_L(0.3) * tan_x;
  Real lim_y_pos = (H - cam.cy) / cam.fy + ORA_L(0.3) * tan_y;
  Real lim_y_neg = cam.cy / cam.fy + ORA_L(0.3) * tan_y;
  Real rz = (Real)1 / t.z;
  Real rx = t.x * rz;
  Real ry = t.y * rz;
  bool cx_flag, cy_flag;
  Real rxc = clamp_flag(rx, -lim_x_neg, lim_x_pos, &cx_flag);
  Real ryc = clamp_flag(ry, -lim_y_neg, lim_y_pos, &cy_flag);
  Real txc = rxc * t.z;
  Real tyc = ryc * t.z;
  Real rz2 = rz * rz;
  Real j[2][3] = {{cam.fx * rz, 0, -cam.fx * txc * rz2}, {0, cam.fy * rz, -cam.fy * tyc * rz2}};

  Real tmat[2][3];
  for (int r = 0; r < 2; r++)
    for (int c = 0; c < 3; c++) {
      Real acc = 0;
      for (int kk = 0; kk < 3; kk++) acc += j[r][kk] * cam.rot.m[kk][c];
      tmat[r][c] = acc;
    }
  Real ts[2][3];
  for (int r = 0; r < 2; r++)
    for (int c = 0; c < 3; c++) {
      Real acc = 0;
      for (int kk = 0; kk < 3; kk++) acc += tmat[r][kk] * sigma.m[kk][c];
      ts[r][c] = acc;
    }
  Real a0 = 0, b0 = 0, c0 = 0;
  for (int c = 0; c < 3; c++) {
    a0 += ts[0][c] * tmat[0][c];
    b0 += ts[0][c] * tmat[1][c];
    c0 += ts[1][c] * tmat[1][c];
  }
  Real det0 = a0 * c0 - b0 * b0;
  Real a = a0 + opts.eps2d;
  Real b = b0;
  Real c = c0 + opts.eps2d;
  Real det = a * c - b * b;
  if (det != det || det <= (Real)0) return false;
  Real inv_det = (Real)1 / det;
  k.conic[0] = c * inv_det;
  k.conic[1] = -b * inv_det;
  k.conic[2] = a * inv_det;
  Real comp;
  if (opts.antialias)
    comp = det0 > (Real)0 ? std::sqrt(det0 * inv_det) : (Real)0;
  else
    comp = 1;

  Real mid = ORA_L(0.5) * (a + c);
  Real lambda1 = mid + std::sqrt(rmax(mid * mid - det, ORA_L(0.1)));
  Real radius = std::ceil((Real)3 * std::sqrt(lambda1));

  k.mean2d[0] = cam.fx * rx + cam.cx;
  k.mean2d[1] = cam.fy * ry + cam.cy;
  Real o_raw = sigmoid(g.opacity);

  V3<Real> d = p - cam.center();
  Real dist = d.norm();
  V3<Real> dir = d * ((Real)1 / dist);
  sh_basis(opts.sh_degree, dir, k.basis);
  int n = num_coeffs(opts.sh_degree);
  for (int ch = 0; ch < 3; ch++) k.color_raw[ch] = ORA_L(0.5);
  for (int kk = 0; kk < n; kk++)
    for (int ch = 0; ch < 3; ch++) k.color_raw[ch] += k.basis[kk] * g.sh[kk][ch];

  k.t = t;
  k.txc = txc;
  k.tyc = tyc;
  k.clamped_x = cx_flag;
  k.clamped_y = cy_flag;
  k.s = s;
  k.q = q;
  k.rq = rq;
  k.m = m;
  k.sigma = sigma;
  std::memcpy(k.tmat, tmat, sizeof(tmat));
  k.a0 = a0;
  k.b0 = b0;
  k.c0 = c0;
  k.det0 = det0;
  k.a = a;
  k.b = b;
  k.c = c;
  k.det = det;
  k.comp = comp;
  k.radius = radius;
  k.o_raw = o_raw;
  k.dir = dir;
  k.dist = dist;
  return true;
}

// project.rs:272
inline void tile_grid(uint32_t width, uint32_t height, uint32_t* tx, uint32_t* ty) {
  *tx = (width + TILE - 1) / TILE;
  *ty = (height + TILE - 1) / TILE;
}

// project.rs:277-317
template <class Real>
Proj<Real> project_one(const Gaussian<Real>& g, const Camera<Real>& cam, const ProjOpts<Real>& opts) {
  Core<Real> k;
  if (!core(g, cam, opts, k)) return Proj<Real>();
  uint32_t tiles_x, tiles_y;
  tile_grid(cam.width, cam.height, &tiles_x, &tiles_y);
  Real r = k.radius;
  if (r != r || r <= (Real)0) return Proj<Real>();
  const Real tile = (Real)TILE;
  auto clamp_tile = [](Real v, uint32_t n) -> uint32_t {
    if (v <= (Real)0) return 0;
    if (v >= (Real)n) return n;
    return (uint32_t)v;
  };
  uint32_t tx0 = clamp_tile(std::floor((k.mean2d[0] - r) / tile), tiles_x);
  uint32_t tx1 = clamp_tile(std::ceil((k.mean2d[0] + r) / tile), tiles_x);
  uint32_t ty0 = clamp_tile(std::floor((k.mean2d[1] - r) / tile), tiles_y);
  uint32_t ty1 = clamp_tile(std::ceil((k.mean2d[1] + r) / tile), tiles_y);
  if (tx0 >= tx1 || ty0 >= ty1) return Proj<Real>();
  Proj<Real> p;
  for (int ch = 0; ch < 3; ch++) p.color[ch] = rmax(k.color_raw[ch], (Real)0);
  p.mean2d[0] = k.mean2d[0];
  p.mean2d[1] = k.mean2d[1];
  for (int i = 0; i < 3; i++) p.conic[i] = k.conic[i];
  p.depth = k.t.z;
  p.radius = as_u32(r);
  p.opacity = k.o_raw * k.comp;
  p.tile_min[0] = tx0;
  p.tile_min[1] = ty0;
  p.tile_max[0] = tx1;
  p.tile_max[1] = ty1;
  return p;
}

// project.rs:320-330 (the caller passes the model's active SH degree in opts)
template <class Real>
void project_all(const Gaussian<Real>* gs, int64_t n, const Camera<Real>& cam, const ProjOpts<Real>& opts,
                 Proj<Real>* out) {
  parallel_for(n, 4096, [&](int64_t lo, int64_t hi) {
    for (int64_t i = lo; i < hi; i++) out[i] = project_one(gs[i], cam, opts);
  });
}

// project.rs:335-474
template <class Real>
Gaussian<Real> project_backward_one(const Gaussian<Real>& g, const Camera<Real>& cam,
                                    const ProjOpts<Real>& opts, const ProjGrad<Real>& dp) {
  Gaussian<Real> out = zero_gaussian<Real>();
  Core<Real> k;
  if (!core(g, cam, opts, k)) return out;

  int n = num_coeffs(opts.sh_degree);
  V3<Real> bgrad[MAX_COEFFS];
  sh_basis_grad(opts.sh_degree, k.dir, bgrad);
  V3<Real> ddir;
  for (int ch = 0; ch < 3; ch++) {
    if (k.color_raw[ch] > (Real)0) {
      Real dc = dp.color[ch];
      for (int kk = 0; kk < n; kk++) {
        out.sh[kk][ch] = dc * k.basis[kk];
        ddir += bgrad[kk] * (dc * g.sh[kk][ch]);
      }
    }
  }
  V3<Real> dmean_color = (ddir - k.dir * k.dir.dot(ddir)) * ((Real)1 / k.dist);

  Real do_raw = dp.opacity * k.comp;
  Real dcomp = dp.opacity * k.o_raw;
  out.opacity = do_raw * k.o_raw * ((Real)1 - k.o_raw);

  const Real a = k.a, b = k.b, c = k.c, det = k.det;
  const Real da_ = dp.conic[0], db_ = dp.conic[1], dc_ = dp.conic[2];
  const Real two = 2;
  Real inv_det2 = (Real)1 / (det * det);
  Real da = (-c * c * da_ + b * c * db_ - b * b * dc_) * inv_det2;
  Real db = (two * b * c * da_ - (a * c + b * b) * db_ + two * a * b * dc_) * inv_det2;
  Real dc = (-b * b * da_ + a * b * db_ - a * a * dc_) * inv_det2;

  if (opts.antialias && k.det0 > (Real)0) {
    Real ddet0 = dcomp * ORA_L(0.5) * k.comp / k.det0;
    Real ddet = -dcomp * ORA_L(0.5) * k.comp / det;
    da += ddet0 * k.c0 + ddet * c;
    dc += ddet0 * k.a0 + ddet * a;
    db += ddet0 * (-two * k.b0) + ddet * (-two * b);
  }

  Real gmat[2][2] = {{da, ORA_L(0.5) * db}, {ORA_L(0.5) * db, dc}};
  const Real(*tm)[3] = k.tmat;
  Real gt[2][3];
  for (int r = 0; r < 2; r++)
    for (int col = 0; col < 3; col++) gt[r][col] = gmat[r][0] * tm[0][col] + gmat[r][1] * tm[1][col];
  M3<Real> dsigma;
  for (int i = 0; i < 3; i++)
    for (int jj = 0; jj < 3; jj++) dsigma.m[i][jj] = tm[0][i] * gt[0][jj] + tm[1][i] * gt[1][jj];
  Real dt[2][3];
  for (int r = 0; r < 2; r++)
    for (int col = 0; col < 3; col++) {
      Real acc = 0;
      for (int kk = 0; kk < 3; kk++) acc += gt[r][kk] * k.sigma.m[kk][col];
      dt[r][col] = two * acc;
    }
  Real dj[2][3];
  for (int r = 0; r < 2; r++)
    for (int col = 0; col < 3; col++) {
      Real acc = 0;
      for (int kk = 0; kk < 3; kk++) acc += dt[r][kk] * cam.rot.m[col][kk];
      dj[r][col] = acc;
    }

  const Real fx = cam.fx, fy = cam.fy;
  Real rz = (Real)1 / k.t.z;
  Real rz2 = rz * rz;
  Real rz3 = rz2 * rz;
  Real dtxc = dj[0][2] * (-fx * rz2);
  Real dtyc = dj[1][2] * (-fy * rz2);
  Real dtx = 0, dty = 0;
  Real dtz = dj[0][0] * (-fx * rz2) + dj[1][1] * (-fy * rz2) + dj[0][2] * (two * fx * k.txc * rz3) +
             dj[1][2] * (two * fy * k.tyc * rz3);
  if (k.clamped_x)
    dtz += dtxc * k.txc * rz;
  else
    dtx += dtxc;
  if (k.clamped_y)
    dtz += dtyc * k.tyc * rz;
  else
    dty += dtyc;

  dtx += dp.mean2d[0] * fx * rz;
  dtz += dp.mean2d[0] * (-fx * k.t.x * rz2);
  dty += dp.mean2d[1] * fy * rz;
  dtz += dp.mean2d[1] * (-fy * k.t.y * rz2);

  V3<Real> dmean = cam.rot.transpose().mul_v(V3<Real>(dtx, dty, dtz)) + dmean_color;
  out.mean[0] = dmean.x;
  out.mean[1] = dmean.y;
  out.mean[2] = dmean.z;

  M3<Real> dm = dsigma.mul_m(k.m).scaled(two);
  Real ds[3] = {0, 0, 0};
  M3<Real> dr;
  for (int r = 0; r < 3; r++)
    for (int col = 0; col < 3; col++) {
      ds[col] += dm.m[r][col] * k.rq.m[r][col];
      dr.m[r][col] = dm.m[r][col] * k.s.get(col);
    }
  for (int i = 0; i < 3; i++) out.log_scale[i] = ds[i] * k.s.get(i);
  Real dq_unit[4];
  quat_to_mat_backward(k.q, dr, dq_unit);
  normalize_backward(g.quat, dq_unit, out.quat);
  return out;
}

// project.rs:477-493
template <class Real>
void project_backward_all(const Gaussian<Real>* gs, int64_t n, const Camera<Real>& cam,
                          const ProjOpts<Real>& opts, const ProjGrad<Real>* grads, Gaussian<Real>* out) {
  parallel_for(n, 4096, [&](int64_t lo, int64_t hi) {
    for (int64_t i = lo; i < hi; i++) out[i] = project_backward_one(gs[i], cam, opts, grads[i]);
  });
}

// ---------------------------------------------------------------------------------------
// src/rasterize.rs
// ---------------------------------------------------------------------------------------
template <class Real> struct RasterSettings {  // rasterize.rs:15-22
  uint32_t width, height;
  Real background[3];
};

struct Binning {  // rasterize.rs:26-39
  uint32_t tiles_x = 0, tiles_y = 0;
  std::vector<uint32_t> entry_gaussian;
  std::vector<uint32_t> entry_offset;
  std::vector<std::pair<uint64_t, uint32_t>> sorted;
  std::vector<std::pair<uint32_t, uint32_t>> tile_range;
};

template <class Real> struct RasterOutput {  // rasterize.rs:43-50
  std::vector<Real> image;
  std::vector<Real> final_t;
  std::vector<uint32_t> n_contrib;
};

template <class Real> struct RC {  // rasterize.rs:53-57
  static Real alpha_min() { return (Real)1 / (Real)255; }
  static Real alpha_max() { return ORA_L(0.99); }
  static Real t_min() { return ORA_L(1e-4); }
};

// Parallel sort of unique (key, entry) pairs: the result is fully determined, as with
// `par_sort_unstable` (rasterize.rs:106).
void parallel_sort_pairs(std::vector<std::pair<uint64_t, uint32_t>>& v);

// rasterize.rs:60-128. Returns false if a tile rectangle exceeds the grid (the reference
// panics there).
template <class Real>
bool bin(const Proj<Real>* projs, int64_t n, uint32_t width, uint32_t height, Binning& out) {
  uint32_t tiles_x, tiles_y;
  tile_grid(width, height, &tiles_x, &tiles_y);
  out.tiles_x = tiles_x;
  out.tiles_y = tiles_y;
  out.entry_offset.resize(n + 1);
  uint64_t total = 0;
  for (int64_t i = 0; i < n; i++) {
    const Proj<Real>& p = projs[i];
    if (p.visible() && !(p.tile_max[0] <= tiles_x && p.tile_max[1] <= tiles_y)) return false;
    out.entry_offset[i] = (uint32_t)total;
    total += p.num_tiles();
  }
  out.entry_offset[n] = (uint32_t)total;
  if (total >= 0xffffffffull) return false;
  out.entry_gaussian.resize(total);
  out.sorted.resize(total);
  parallel_for(n, 4096, [&](int64_t lo, int64_t hi) {
    for (int64_t gi = lo; gi < hi; gi++) {
      const Proj<Real>& p = projs[gi];
      if (!p.visible()) continue;
      uint64_t depth_bits = f32_bits((float)p.depth);
      uint32_t e = out.entry_offset[gi];
      for (uint32_t ty = p.tile_min[1]; ty < p.tile_max[1]; ty++)
        for (uint32_t tx = p.tile_min[0]; tx < p.tile_max[0]; tx++) {
          uint64_t tile = (uint64_t)(ty * tiles_x + tx);
          out.entry_gaussian[e] = (uint32_t)gi;
          out.sorted[e] = std::make_pair((tile << 32) | depth_bits, e);
          e++;
        }
    }
  });
  parallel_sort_pairs(out.sorted);
  size_t num_tiles = (size_t)tiles_x * tiles_y;
  out.tile_range.assign(num_tiles, std::make_pair(0u, 0u));
  size_t s = 0;
  while (s < out.sorted.size()) {
    size_t tile = (size_t)(out.sorted[s].first >> 32);
    size_t e = s + 1;
    while (e < out.sorted.size() && (size_t)(out.sorted[e].first >> 32) == tile) e++;
    out.tile_range[tile] = std::make_pair((uint32_t)s, (uint32_t)e);
    s = e;
  }
  return true;
}

template <class Real> struct TileGauss {  // rasterize.rs:132-145
  Real mean[2];
  Real conic[3];
  Real opacity;
  Real color[3];
  Real sigma_max;
  uint32_t x0, x1, y0, y1;
  bool is_empty() const { return x0 >= x1 || y0 >= y1; }
};

// rasterize.rs:149-182
template <class Real>
TileGauss<Real> make_tile_gauss(const Proj<Real>& p, uint32_t tx0, uint32_t ty0, uint32_t w, uint32_t h) {
  TileGauss<Real> tg;
  Real sigma_max = rln(p.opacity / RC<Real>::alpha_min());
  const Real a = p.conic[0], b = p.conic[1], c = p.conic[2];
  Real det = a * c - b * b;
  uint32_t x0 = 0, x1 = 0, y0 = 0, y1 = 0;
  if (sigma_max > (Real)0 && det > (Real)0) {
    Real half_x = std::sqrt((Real)2 * sigma_max * c / det) + ORA_L(1e-3);
    Real half_y = std::sqrt((Real)2 * sigma_max * a / det) + ORA_L(1e-3);
    auto clip = [](Real lo, Real hi, uint32_t offset, uint32_t n, uint32_t* olo, uint32_t* ohi) {
      Real l = std::ceil(lo - ORA_L(0.5)) - (Real)offset;
      Real hh = std::floor(hi - ORA_L(0.5)) - (Real)offset + (Real)1;
      *olo = as_u32(rclamp(l, (Real)0, (Real)n));
      *ohi = as_u32(rclamp(hh, (Real)0, (Real)n));
    };
    clip(p.mean2d[0] - half_x, p.mean2d[0] + half_x, tx0, w, &x0, &x1);
    clip(p.mean2d[1] - half_y, p.mean2d[1] + half_y, ty0, h, &y0, &y1);
  }
  tg.mean[0] = p.mean2d[0];
  tg.mean[1] = p.mean2d[1];
  for (int i = 0; i < 3; i++) tg.conic[i] = p.conic[i];
  tg.opacity = p.opacity;
  for (int i = 0; i < 3; i++) tg.color[i] = p.color[i];
  tg.sigma_max = sigma_max;
  tg.x0 = x0;
  tg.x1 = x1;
  tg.y0 = y0;
  tg.y1 = y1;
  return tg;
}

struct TileGeom {  // rasterize.rs:191-196
  uint32_t x0, y0, w, h;
};

inline TileGeom tile_geom(const Binning& b, uint32_t width, uint32_t height, size_t tile) {  // :198
  uint32_t tx = (uint32_t)tile % b.tiles_x;
  uint32_t ty = (uint32_t)tile / b.tiles_x;
  uint32_t x0 = tx * TILE, y0 = ty * TILE;
  return TileGeom{x0, y0, std::min(width - x0, TILE), std::min(height - y0, TILE)};
}

// rasterize.rs:211-220
template <class Real>
void gather(const Proj<Real>* projs, const Binning& b, size_t tile, const TileGeom& geom,
            std::vector<TileGauss<Real>>& list) {
  uint32_t s = b.tile_range[tile].first, e = b.tile_range[tile].second;
  list.clear();
  for (uint32_t i = s; i < e; i++) {
    uint32_t entry = b.sorted[i].second;
    const Proj<Real>& p = projs[b.entry_gaussian[entry]];
    list.push_back(make_tile_gauss(p, geom.x0, geom.y0, geom.w, geom.h));
  }
}

// rasterize.rs:231-244. Returns false when skipped.
template <class Real>
inline bool evaluate(const TileGauss<Real>& g, Real px, Real py, Real* gauss_out, Real* alpha_out) {
  Real dx = px - g.mean[0];
  Real dy = py - g.mean[1];
  Real sigma = ORA_L(0.5) * (g.conic[0] * dx * dx + g.conic[2] * dy * dy) + g.conic[1] * dx * dy;
  if (sigma < (Real)0 || sigma > g.sigma_max) return false;
  Real gauss = rexp(-sigma);
  Real og = g.opacity * gauss;
  if (og < RC<Real>::alpha_min()) return false;
  *gauss_out = gauss;
  *alpha_out = rmin(og, RC<Real>::alpha_max());
  return true;
}

// Work counters (not in the reference): evaluated (entry, pixel) pairs, used to express
// CPU and GPU throughput per pair, and the pairs that pass the alpha threshold, the unit of
// the reference's published per-core cost (README.md:153: ~15 ns forward, ~25 ns backward).
struct RasterCounters {
  std::atomic<uint64_t> pairs_fwd{0};
  std::atomic<uint64_t> pairs_bwd{0};
  std::atomic<uint64_t> passed_fwd{0};
  std::atomic<uint64_t> passed_bwd{0};
};

// rasterize.rs:249-337
template <class Real>
void rasterize_forward(const Proj<Real>* projs, const Binning& b, const RasterSettings<Real>& st,
                       RasterOutput<Real>& out, RasterCounters* counters = nullptr) {
  const size_t num_tiles = (size_t)b.tiles_x * b.tiles_y;
  const size_t npix = (size_t)st.width * st.height;
  out.image.assign(npix * 3, (Real)0);
  out.final_t.assign(npix, (Real)1);
  out.n_contrib.assign(npix, 0);
  const size_t width = st.width;
  parallel_for((int64_t)num_tiles, 1, [&](int64_t lo, int64_t hi) {
    std::vector<TileGauss<Real>> list;
    Real color[TILE * TILE * 3];
    Real trans[TILE * TILE];
    uint32_t ncon[TILE * TILE];
    bool done[TILE * TILE];
    uint64_t pairs = 0, passed = 0;
    for (int64_t tile = lo; tile < hi; tile++) {
      TileGeom geom = tile_geom(b, st.width, st.height, (size_t)tile);
      gather(projs, b, (size_t)tile, geom, list);
      const size_t n = (size_t)geom.w * geom.h;
      for (size_t i = 0; i < n * 3; i++) color[i] = 0;
      for (size_t i = 0; i < n; i++) {
        trans[i] = 1;
        ncon[i] = 0;
        done[i] = false;
      }
      for (size_t k = 0; k < list.size(); k++) {
        const TileGauss<Real>& g = list[k];
        if (g.is_empty()) continue;
        for (uint32_t j = g.y0; j < g.y1; j++) {
          Real py = (Real)(geom.y0 + j) + ORA_L(0.5);
          for (uint32_t i = g.x0; i < g.x1; i++) {
            size_t pix = (size_t)(j * geom.w + i);
            if (done[pix]) continue;
            Real px = (Real)(geom.x0 + i) + ORA_L(0.5);
            pairs++;
            Real gauss, alpha;
            if (!evaluate(g, px, py, &gauss, &alpha)) continue;
            passed++;
            Real t = trans[pix];
            Real test_t = t * ((Real)1 - alpha);
            if (test_t < RC<Real>::t_min()) {
              done[pix] = true;
              continue;
            }
            for (int ch = 0; ch < 3; ch++) color[pix * 3 + ch] += alpha * t * g.color[ch];
            trans[pix] = test_t;
            ncon[pix] = (uint32_t)k + 1;
          }
        }
      }
      for (size_t pix = 0; pix < n; pix++)
        for (int ch = 0; ch < 3; ch++) color[pix * 3 + ch] += trans[pix] * st.background[ch];
      for (uint32_t j = 0; j < geom.h; j++)
        for (uint32_t i = 0; i < geom.w; i++) {
          size_t src = (size_t)j * geom.w + i;
          size_t dst = (size_t)(geom.y0 + j) * width + geom.x0 + i;
          for (int ch = 0; ch < 3; ch++) out.image[dst * 3 + ch] = color[src * 3 + ch];
          out.final_t[dst] = trans[src];
          out.n_contrib[dst] = ncon[src];
        }
    }
    if (counters) {
      counters->pairs_fwd += pairs;
      counters->passed_fwd += passed;
    }
  });
}

constexpr int SLOTS = 11;  // rasterize.rs:341

// rasterize.rs:354-505. `abs_out` receives the AbsGS accumulators (2 per Gaussian).
template <class Real>
void rasterize_backward(const Proj<Real>* projs, int64_t n_gauss, const Binning& b,
                        const RasterSettings<Real>& st, const RasterOutput<Real>& out, const Real* dimage,
                        ProjGrad<Real>* grads, Real* abs_out, RasterCounters* counters = nullptr) {
  const size_t num_entries = b.sorted.size();
  std::vector<Real> slots(num_entries * SLOTS, (Real)0);
  const size_t num_tiles = (size_t)b.tiles_x * b.tiles_y;
  const size_t width = st.width;
  const Real* bg = st.background;
  parallel_for((int64_t)num_tiles, 1, [&](int64_t lo, int64_t hi) {
    std::vector<TileGauss<Real>> list;
    std::vector<std::array<Real, SLOTS>> acc;
    struct PixelBack {
      Real t;
      Real accum[3];
      Real last_alpha;
      Real last_color[3];
    };
    PixelBack state[TILE * TILE];
    Real dl[TILE * TILE][3];
    Real bg_dot[TILE * TILE];
    uint32_t last[TILE * TILE];
    Real t_final[TILE * TILE];
    uint64_t pairs = 0, passed = 0;
    for (int64_t tile = lo; tile < hi; tile++) {
      TileGeom geom = tile_geom(b, st.width, st.height, (size_t)tile);
      uint32_t start = b.tile_range[tile].first;
      gather(projs, b, (size_t)tile, geom, list);
      if (list.empty()) continue;
      size_t q = 0;
      for (uint32_t j = 0; j < geom.h; j++)
        for (uint32_t i = 0; i < geom.w; i++, q++) {
          size_t pix = (size_t)(geom.y0 + j) * width + geom.x0 + i;
          for (int ch = 0; ch < 3; ch++) dl[q][ch] = dimage[pix * 3 + ch];
          bg_dot[q] = bg[0] * dl[q][0] + bg[1] * dl[q][1] + bg[2] * dl[q][2];
          last[q] = out.n_contrib[pix];
          t_final[q] = out.final_t[pix];
          state[q].t = out.final_t[pix];
          state[q].accum[0] = state[q].accum[1] = state[q].accum[2] = 0;
          state[q].last_alpha = 0;
          state[q].last_color[0] = state[q].last_color[1] = state[q].last_color[2] = 0;
        }
      acc.assign(list.size(), std::array<Real, SLOTS>{});
      for (size_t k = list.size(); k-- > 0;) {
        const TileGauss<Real>& g = list[k];
        if (g.is_empty()) continue;
        Real* a = acc[k].data();
        for (uint32_t j = g.y0; j < g.y1; j++) {
          Real py = (Real)(geom.y0 + j) + ORA_L(0.5);
          for (uint32_t i = g.x0; i < g.x1; i++) {
            size_t pix = (size_t)(j * geom.w + i);
            if (k >= last[pix]) continue;
            Real px = (Real)(geom.x0 + i) + ORA_L(0.5);
            pairs++;
            Real gauss, alpha;
            if (!evaluate(g, px, py, &gauss, &alpha)) continue;
            passed++;
            PixelBack& s = state[pix];
            const Real* d = dl[pix];
            s.t /= (Real)1 - alpha;
            Real t = s.t;
            Real dalpha = 0;
            for (int ch = 0; ch < 3; ch++) {
              s.accum[ch] = s.last_alpha * s.last_color[ch] + ((Real)1 - s.last_alpha) * s.accum[ch];
              dalpha += (g.color[ch] - s.accum[ch]) * d[ch];
              a[6 + ch] += alpha * t * d[ch];
            }
            dalpha *= t;
            for (int ch = 0; ch < 3; ch++) s.last_color[ch] = g.color[ch];
            s.last_alpha = alpha;
            dalpha += -t_final[pix] / ((Real)1 - alpha) * bg_dot[pix];
            if (g.opacity * gauss < RC<Real>::alpha_max()) {
              a[5] += gauss * dalpha;
              Real dgauss = g.opacity * dalpha;
              Real dsigma = -dgauss * gauss;
              Real dx = px - g.mean[0];
              Real dy = py - g.mean[1];
              Real ddx = dsigma * (g.conic[0] * dx + g.conic[1] * dy);
              Real ddy = dsigma * (g.conic[1] * dx + g.conic[2] * dy);
              a[0] -= ddx;
              a[1] -= ddy;
              a[2] += dsigma * ORA_L(0.5) * dx * dx;
              a[3] += dsigma * dx * dy;
              a[4] += dsigma * ORA_L(0.5) * dy * dy;
              a[9] += std::fabs(ddx);
              a[10] += std::fabs(ddy);
            }
          }
        }
      }
      for (size_t k = 0; k < acc.size(); k++) {
        size_t entry = b.sorted[start + k].second;
        for (int s = 0; s < SLOTS; s++) slots[entry * SLOTS + s] = acc[k][s];
      }
    }
    if (counters) {
      counters->pairs_bwd += pairs;
      counters->passed_bwd += passed;
    }
  });
  parallel_for(n_gauss, 4096, [&](int64_t lo, int64_t hi) {
    for (int64_t gi = lo; gi < hi; gi++) {
      Real sum[SLOTS] = {0};
      size_t s = b.entry_offset[gi], e = b.entry_offset[gi + 1];
      for (size_t entry = s; entry < e; entry++)
        for (int k = 0; k < SLOTS; k++) sum[k] += slots[entry * SLOTS + k];
      ProjGrad<Real>& g = grads[gi];
      g.mean2d[0] = sum[0];
      g.mean2d[1] = sum[1];
      g.conic[0] = sum[2];
      g.conic[1] = sum[3];
      g.conic[2] = sum[4];
      g.opacity = sum[5];
      g.color[0] = sum[6];
      g.color[1] = sum[7];
      g.color[2] = sum[8];
      if (abs_out) {
        abs_out[gi * 2] = sum[9];
        abs_out[gi * 2 + 1] = sum[10];
      }
    }
  });
}

// The reference's second compositor (tests/pipeline.rs:134-186): every visible Gaussian
// whose tile rectangle covers the pixel's tile, in (depth bits, index) order.
template <class Real>
void naive_render(const Proj<Real>* projs, int64_t n, uint32_t width, uint32_t height, const Real bg[3],
                  Real* image) {
  std::vector<int64_t> order;
  for (int64_t i = 0; i < n; i++)
    if (projs[i].visible()) order.push_back(i);
  std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
    uint32_t da = f32_bits((float)projs[a].depth), db = f32_bits((float)projs[b].depth);
    return da != db ? da < db : a < b;
  });
  parallel_for(height, 1, [&](int64_t lo, int64_t hi) {
    for (int64_t y = lo; y < hi; y++)
      for (uint32_t x = 0; x < width; x++) {
        uint32_t tx = x / TILE, ty = (uint32_t)y / TILE;
        Real px = (Real)x + ORA_L(0.5), py = (Real)y + ORA_L(0.5);
        Real t = 1;
        Real c[3] = {0, 0, 0};
        for (int64_t i : order) {
          const Proj<Real>& p = projs[i];
          if (tx < p.tile_min[0] || tx >= p.tile_max[0] || ty < p.tile_min[1] || ty >= p.tile_max[1]) continue;
          Real dx = px - p.mean2d[0];
          Real dy = py - p.mean2d[1];
          Real sigma = ORA_L(0.5) * (p.conic[0] * dx * dx + p.conic[2] * dy * dy) + p.conic[1] * dx * dy;
          if (sigma < (Real)0) continue;
          Real og = p.opacity * rexp(-sigma);
          if (og < (Real)1 / (Real)255) continue;
          Real alpha = rmin(og, ORA_L(0.99));
          Real test_t = t * ((Real)1 - alpha);
          if (test_t < ORA_L(1e-4)) break;
          for (int ch = 0; ch < 3; ch++) c[ch] += alpha * t * p.color[ch];
          t = test_t;
        }
        size_t pix = (size_t)y * width + x;
        for (int ch = 0; ch < 3; ch++) image[pix * 3 + ch] = c[ch] + t * bg[ch];
      }
  });
}

// ---------------------------------------------------------------------------------------
// src/loss.rs
// ---------------------------------------------------------------------------------------
constexpr int SSIM_WINDOW = 11;

template <class Real> void gaussian_kernel(Real k[SSIM_WINDOW]) {  // loss.rs:14-27
  const Real sigma = ORA_L(1.5);
  Real sum = 0;
  for (int i = 0; i < SSIM_WINDOW; i++) {
    Real x = (Real)i - (Real)(SSIM_WINDOW / 2);
    k[i] = rexp(-(x * x) / ((Real)2 * sigma * sigma));
    sum += k[i];
  }
  for (int i = 0; i < SSIM_WINDOW; i++) k[i] /= sum;
}

// loss.rs:31-72
template <class Real>
void blur(const Real* src, size_t width, size_t height, size_t channels, const Real kernel[SSIM_WINDOW],
          Real* dst) {
  const int64_t half = SSIM_WINDOW / 2;
  const size_t row = width * channels;
  std::vector<Real> tmp(row * height);
  parallel_for((int64_t)height, 8, [&](int64_t lo, int64_t hi) {
    for (int64_t y = lo; y < hi; y++) {
      const Real* line = src + y * row;
      Real* out = tmp.data() + y * row;
      for (size_t x = 0; x < width; x++)
        for (size_t c = 0; c < channels; c++) {
          Real acc = 0;
          for (int k = 0; k < SSIM_WINDOW; k++) {
            int64_t xs = (int64_t)x + k - half;
            if (xs >= 0 && (size_t)xs < width) acc += kernel[k] * line[xs * channels + c];
          }
          out[x * channels + c] = acc;
        }
    }
  });
  parallel_for((int64_t)height, 8, [&](int64_t lo, int64_t hi) {
    for (int64_t y = lo; y < hi; y++) {
      Real* out = dst + y * row;
      for (size_t i = 0; i < row; i++) out[i] = 0;
      for (int k = 0; k < SSIM_WINDOW; k++) {
        int64_t ys = y + k - half;
        if (ys >= 0 && (size_t)ys < height) {
          const Real* line = tmp.data() + ys * row;
          Real kv = kernel[k];
          for (size_t i = 0; i < row; i++) out[i] += kv * line[i];
        }
      }
    }
  });
}

// Sum of per-chunk partial sums in chunk order: one fixed order standing in for rayon's
// parallel `sum` (loss.rs:96-121, :147-152), whose grouping is not specified.
template <class Real> Real chunked_sum(int64_t n, const std::function<Real(int64_t)>& term) {
  const int64_t chunk = 1 << 14;
  int64_t nchunks = (n + chunk - 1) / chunk;
  std::vector<Real> part(nchunks, (Real)0);
  parallel_for(nchunks, 1, [&](int64_t lo, int64_t hi) {
    for (int64_t c = lo; c < hi; c++) {
      Real s = 0;
      for (int64_t i = c * chunk; i < std::min(n, (c + 1) * chunk); i++) s += term(i);
      part[c] = s;
    }
  });
  Real s = 0;
  for (Real p : part) s += p;
  return s;
}

// loss.rs:75-134
template <class Real>
Real ssim_with_grad(const Real* x, const Real* y, size_t width, size_t height, Real* grad) {
  const size_t n = width * height * 3;
  Real kernel[SSIM_WINDOW];
  gaussian_kernel(kernel);
  const Real c1 = ORA_L(0.01) * ORA_L(0.01);
  const Real c2 = ORA_L(0.03) * ORA_L(0.03);
  std::vector<Real> mu_x(n), mu_y(n), xx(n), yy(n), xy(n), e_xx(n), e_yy(n), e_xy(n);
  blur(x, width, height, 3, kernel, mu_x.data());
  blur(y, width, height, 3, kernel, mu_y.data());
  for (size_t i = 0; i < n; i++) {
    xx[i] = x[i] * x[i];
    yy[i] = y[i] * y[i];
    xy[i] = x[i] * y[i];
  }
  blur(xx.data(), width, height, 3, kernel, e_xx.data());
  blur(yy.data(), width, height, 3, kernel, e_yy.data());
  blur(xy.data(), width, height, 3, kernel, e_xy.data());
  std::vector<Real> d_mu(n), d_exx(n), d_exy(n);
  const Real two = 2;
  Real ssim_sum = chunked_sum<Real>((int64_t)n, [&](int64_t i) -> Real {
    Real mx = mu_x[i], my = mu_y[i];
    Real sx2 = e_xx[i] - mx * mx;
    Real sy2 = e_yy[i] - my * my;
    Real sxy = e_xy[i] - mx * my;
    Real n1 = two * mx * my + c1;
    Real n2 = two * sxy + c2;
    Real d1 = mx * mx + my * my + c1;
    Real d2 = sx2 + sy2 + c2;
    Real num = n1 * n2;
    Real den = d1 * d2;
    Real s = num / den;
    Real dn_dmx = two * my * n2 - two * my * n1;
    Real dd_dmx = two * mx * d2 - two * mx * d1;
    d_mu[i] = (dn_dmx * den - num * dd_dmx) / (den * den);
    d_exx[i] = -num * d1 / (den * den);
    d_exy[i] = two * n1 / den;
    return s;
  });
  Real mean = ssim_sum / (Real)n;
  std::vector<Real> b_mu(n), b_exx(n), b_exy(n);
  blur(d_mu.data(), width, height, 3, kernel, b_mu.data());
  blur(d_exx.data(), width, height, 3, kernel, b_exx.data());
  blur(d_exy.data(), width, height, 3, kernel, b_exy.data());
  Real inv_n = (Real)1 / (Real)n;
  for (size_t i = 0; i < n; i++) grad[i] = (b_mu[i] + two * x[i] * b_exx[i] + y[i] * b_exy[i]) * inv_n;
  return mean;
}

// loss.rs:137-171. Returns the loss; `grad` (n) receives d loss / d pred.
template <class Real>
Real photometric_loss(const Real* pred, const Real* target, size_t width, size_t height, Real lambda_dssim,
                      Real* grad) {
  const size_t n = width * height * 3;
  Real inv_n = (Real)1 / (Real)n;
  Real l1 = chunked_sum<Real>((int64_t)n, [&](int64_t i) -> Real { return std::fabs(pred[i] - target[i]); }) * inv_n;
  std::vector<Real> dssim(n);
  Real ssim = ssim_with_grad(pred, target, width, height, dssim.data());
  Real loss = ((Real)1 - lambda_dssim) * l1 + lambda_dssim * ((Real)1 - ssim);
  Real w1 = ((Real)1 - lambda_dssim) * inv_n;
  for (size_t i = 0; i < n; i++) {
    Real d = pred[i] - target[i];
    Real sign = d > (Real)0 ? (Real)1 : (d < (Real)0 ? (Real)-1 : (Real)0);
    grad[i] = w1 * sign - lambda_dssim * dssim[i];
  }
  return loss;
}

// loss.rs:175-190
template <class Real> Real psnr(const Real* pred, const Real* target, size_t n) {
  double mse = 0;
  for (size_t i = 0; i < n; i++) {
    double d = (double)rclamp(pred[i], (Real)0, (Real)1) - (double)rclamp(target[i], (Real)0, (Real)1);
    mse += d * d;
  }
  mse /= (double)std::max<size_t>(n, 1);
  if (mse <= 0) return std::numeric_limits<Real>::infinity();
  return (Real)(-10.0 * std::log10(mse));
}

// ---------------------------------------------------------------------------------------
// src/adam.rs
// ---------------------------------------------------------------------------------------
template <class Real> struct LearningRates {  // adam.rs:11-24
  Real mean, log_scale, quat, opacity, sh_dc, sh_rest;
};

// Right-to-left binary exponentiation, the runtime routine Rust's `powi` lowers to.
template <class Real> Real powi(Real a, int b) {
  bool recip = b < 0;
  Real r = 1;
  while (true) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return recip ? (Real)1 / r : r;
}

template <class Real> struct Adam {  // adam.rs:28-41
  std::vector<Gaussian<Real>> m, v;
  uint64_t step = 0;
  Real beta1 = ORA_L(0.9), beta2 = ORA_L(0.999), eps = ORA_L(1e-15);

  explicit Adam(size_t n = 0) : m(n, zero_gaussian<Real>()), v(n, zero_gaussian<Real>()) {}

  // adam.rs:44-61
  static inline void update(Real& p, Real g, Real& m, Real& v, Real lr, Real b1, Real b2, Real c1, Real c2,
                            Real eps) {
    m = b1 * m + ((Real)1 - b1) * g;
    v = b2 * v + ((Real)1 - b2) * g * g;
    Real m_hat = m / c1;
    Real v_hat = v / c2;
    p -= lr * m_hat / (std::sqrt(v_hat) + eps);
  }

  // adam.rs:77-161
  void do_step(Gaussian<Real>* params, const Gaussian<Real>* grads, size_t n, const LearningRates<Real>& lr) {
    step += 1;
    const Real b1 = beta1, b2 = beta2, e = eps;
    const Real c1 = (Real)1 - powi(b1, (int)step);
    const Real c2 = (Real)1 - powi(b2, (int)step);
    parallel_for((int64_t)n, 4096, [&](int64_t lo, int64_t hi) {
      for (int64_t i = lo; i < hi; i++) {
        Gaussian<Real>& p = params[i];
        const Gaussian<Real>& g = grads[i];
        Gaussian<Real>& mm = m[i];
        Gaussian<Real>& vv = v[i];
        for (int k = 0; k < 3; k++) {
          update(p.mean[k], g.mean[k], mm.mean[k], vv.mean[k], lr.mean, b1, b2, c1, c2, e);
          update(p.log_scale[k], g.log_scale[k], mm.log_scale[k], vv.log_scale[k], lr.log_scale, b1, b2, c1, c2, e);
        }
        for (int k = 0; k < 4; k++) update(p.quat[k], g.quat[k], mm.quat[k], vv.quat[k], lr.quat, b1, b2, c1, c2, e);
        update(p.opacity, g.opacity, mm.opacity, vv.opacity, lr.opacity, b1, b2, c1, c2, e);
        for (int k = 0; k < MAX_COEFFS; k++) {
          Real rate = k == 0 ? lr.sh_dc : lr.sh_rest;
          for (int c = 0; c < 3; c++) update(p.sh[k][c], g.sh[k][c], mm.sh[k][c], vv.sh[k][c], rate, b1, b2, c1, c2, e);
        }
      }
    });
  }
  void retain_mask(const std::vector<char>& keep) {  // adam.rs:164
    retain_by_mask(m, keep);
    retain_by_mask(v, keep);
  }
  void append_zeros(size_t k) {  // adam.rs:170
    m.insert(m.end(), k, zero_gaussian<Real>());
    v.insert(v.end(), k, zero_gaussian<Real>());
  }
  void reset_opacity_state() {  // adam.rs:176-183
    for (auto& x : m) x.opacity = 0;
    for (auto& x : v) x.opacity = 0;
  }
};

// ---------------------------------------------------------------------------------------
// Seeded generator shared by the oracle trainer and the CUDA trainer's host code (not in
// the reference, whose ChaCha8 stream is not reproduced): SplitMix64 (Steele, Lea &
// Flood 2014) for 64-bit words, 53-bit uniform doubles, Box-Muller normals, Fisher-Yates.
// ---------------------------------------------------------------------------------------
struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  // densify.rs:116-121: Box-Muller with u1 kept away from zero.
  double normal() {
    double u1 = std::max(uniform(), 1e-12);
    double u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * 3.14159265358979323846 * u2);
  }
  // Uniform index in [0, n) by rejection-free multiply-shift (n < 2^32).
  uint32_t index(uint32_t n) { return (uint32_t)(((next() >> 32) * (uint64_t)n) >> 32); }
};

// ---------------------------------------------------------------------------------------
// src/densify.rs
// ---------------------------------------------------------------------------------------
template <class Real> struct DensifyStats {  // densify.rs:15-65
  std::vector<Real> grad_accum;
  std::vector<uint32_t> denom;
  std::vector<uint32_t> max_radii;
  explicit DensifyStats(size_t n = 0) : grad_accum(n, (Real)0), denom(n, 0), max_radii(n, 0) {}
  // densify.rs:36-60
  void accumulate(const Proj<Real>* projs, const ProjGrad<Real>* grads, const Real* abs_grads, size_t n,
                  uint32_t width, uint32_t height) {
    Real sx = (Real)width * ORA_L(0.5);
    Real sy = (Real)height * ORA_L(0.5);
    for (size_t i = 0; i < n; i++) {
      if (!projs[i].visible()) continue;
      Real g0 = abs_grads ? abs_grads[2 * i] : grads[i].mean2d[0];
      Real g1 = abs_grads ? abs_grads[2 * i + 1] : grads[i].mean2d[1];
      Real gx = g0 * sx;
      Real gy = g1 * sy;
      grad_accum[i] += std::sqrt(gx * gx + gy * gy);
      denom[i] += 1;
      max_radii[i] = std::max(max_radii[i], projs[i].radius);
    }
  }
};

template <class Real> struct DensifyConfig {  // densify.rs:69-103
  Real grad_threshold = ORA_L(0.0002);
  Real percent_dense = ORA_L(0.01);
  Real min_opacity = ORA_L(0.005);
  bool prune_big_world = false;
  Real max_world_size_frac = ORA_L(0.1);
  int64_t max_screen_size = -1;  // None
  int split_children = 2;
};

struct DensifyReport {  // densify.rs:107-114
  size_t cloned = 0, split = 0, pruned = 0;
};

// densify.rs:125-221. Split offsets are drawn from `normal()` in the reference's order:
// per split parent (ascending index), per child, x then y then z.
template <class Real>
DensifyReport densify_and_prune(std::vector<Gaussian<Real>>& model, Adam<Real>& adam, DensifyStats<Real>& stats,
                                const DensifyConfig<Real>& cfg, Real extent,
                                const std::function<double()>& normal) {
  const size_t n0 = model.size();
  std::vector<Real> grads(n0);
  for (size_t i = 0; i < n0; i++)
    grads[i] = stats.denom[i] > 0 ? stats.grad_accum[i] / (Real)stats.denom[i] : (Real)0;
  const Real size_limit = cfg.percent_dense * extent;
  DensifyReport report;
  std::vector<int64_t> origin(n0);
  for (size_t i = 0; i < n0; i++) origin[i] = (int64_t)i;

  std::vector<Gaussian<Real>> clones;
  for (size_t i = 0; i < n0; i++)
    if (grads[i] >= cfg.grad_threshold && model[i].scales().max_elem() <= size_limit) clones.push_back(model[i]);
  report.cloned = clones.size();
  adam.append_zeros(clones.size());
  origin.insert(origin.end(), clones.size(), -1);
  model.insert(model.end(), clones.begin(), clones.end());

  std::vector<size_t> split_idx;
  for (size_t i = 0; i < n0; i++)
    if (grads[i] >= cfg.grad_threshold && model[i].scales().max_elem() > size_limit) split_idx.push_back(i);
  report.split = split_idx.size();
  std::vector<Gaussian<Real>> children;
  const Real shrink = rln(ORA_L(0.8) * (Real)cfg.split_children);
  for (size_t i : split_idx) {
    Gaussian<Real> g = model[i];
    V3<Real> s = g.scales();
    M3<Real> rot = g.rotation().to_mat();
    for (int c = 0; c < cfg.split_children; c++) {
      Real nx = (Real)normal();
      Real ny = (Real)normal();
      Real nz = (Real)normal();
      V3<Real> local(nx * s.x, ny * s.y, nz * s.z);
      V3<Real> mean = g.mean_v() + rot.mul_v(local);
      Gaussian<Real> child = g;
      child.mean[0] = mean.x;
      child.mean[1] = mean.y;
      child.mean[2] = mean.z;
      for (int k = 0; k < 3; k++) child.log_scale[k] = g.log_scale[k] - shrink;
      children.push_back(child);
    }
  }
  adam.append_zeros(children.size());
  origin.insert(origin.end(), children.size(), -1);
  model.insert(model.end(), children.begin(), children.end());
  std::vector<char> keep(model.size(), 1);
  for (size_t i : split_idx) keep[i] = 0;
  retain_by_mask(model, keep);
  adam.retain_mask(keep);
  retain_by_mask(origin, keep);

  const size_t n2 = model.size();
  keep.assign(n2, 1);
  for (size_t i = 0; i < n2; i++) {
    const Gaussian<Real>& g = model[i];
    bool prune = g.alpha() < cfg.min_opacity;
    if (cfg.prune_big_world) prune |= g.scales().max_elem() > cfg.max_world_size_frac * extent;
    if (cfg.max_screen_size >= 0 && origin[i] >= 0) prune |= stats.max_radii[origin[i]] > (uint32_t)cfg.max_screen_size;
    keep[i] = !prune;
  }
  for (size_t i = 0; i < n2; i++) report.pruned += keep[i] ? 0 : 1;
  retain_by_mask(model, keep);
  adam.retain_mask(keep);
  stats = DensifyStats<Real>(model.size());
  return report;
}

// densify.rs:224-230
template <class Real> void reset_opacity(std::vector<Gaussian<Real>>& model, Adam<Real>& adam, Real max_alpha) {
  Real limit = inverse_sigmoid(max_alpha);
  for (auto& g : model) g.opacity = rmin(g.opacity, limit);
  adam.reset_opacity_state();
}

// ---------------------------------------------------------------------------------------
// src/model.rs:77-186: initialisation from a point cloud (exact 3-NN in f64).
// ---------------------------------------------------------------------------------------
void mean_nn_dist2(const float* pts, int64_t n, double* out);

template <class Real>
void from_points(const float* pts, const uint8_t* rgb, int64_t n, std::vector<Gaussian<Real>>& model) {
  std::vector<double> d2(n);
  mean_nn_dist2(pts, n, d2.data());
  Real opacity = inverse_sigmoid(ORA_L(0.1));
  model.resize(n);
  for (int64_t i = 0; i < n; i++) {
    Real d = rmax((Real)d2[i], ORA_L(1e-7));
    Real log_s = rln(std::sqrt(d));
    Gaussian<Real> g = zero_gaussian<Real>();
    for (int k = 0; k < 3; k++) {
      g.mean[k] = (Real)pts[3 * i + k];
      g.log_scale[k] = log_s;
    }
    g.quat[0] = 1;
    g.opacity = opacity;
    for (int c = 0; c < 3; c++) g.sh[0][c] = rgb_to_sh((Real)rgb[3 * i + c] / (Real)255);
    model[i] = g;
  }
}

}  // namespace ora
