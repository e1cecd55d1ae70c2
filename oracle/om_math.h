// Oracle (test infrastructure only): CPU restatement of the reference engine's
// fixed-size math, used to check the CUDA backend. Nothing in the product links
// this file.
//
// Restates crates/pippin/src/math.rs and crates/pippin/src/simd.rs. Operation
// order follows the reference exactly (no reassociation, no FMA contraction:
// build with -ffp-contract=off), so results equal the Rust engine's bit for bit
// wherever the same libm is used.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>

namespace om {

using Real = double;

// ---------------------------------------------------------------- Vec3
// math.rs:9-128
struct Vec3 {
  Real v[3];
  Real& operator[](int i) { return v[i]; }
  Real operator[](int i) const { return v[i]; }
};

inline Vec3 v3(Real x, Real y, Real z) { return Vec3{{x, y, z}}; }
inline Vec3 v3zero() { return Vec3{{0.0, 0.0, 0.0}}; }
inline Vec3 operator+(Vec3 a, Vec3 b) { return v3(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
inline Vec3 operator-(Vec3 a, Vec3 b) { return v3(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
inline Vec3 operator-(Vec3 a) { return v3(-a[0], -a[1], -a[2]); }
inline Vec3 operator*(Vec3 a, Real s) { return v3(a[0] * s, a[1] * s, a[2] * s); }
inline Vec3& operator+=(Vec3& a, Vec3 b) { a = a + b; return a; }
inline Vec3& operator-=(Vec3& a, Vec3 b) { a = a - b; return a; }
// math.rs:21-23
inline Real dot(Vec3 a, Vec3 b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
// math.rs:25-29
inline Vec3 cross(Vec3 a, Vec3 b) {
  return v3(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
inline Real norm2(Vec3 a) { return dot(a, a); }
inline Real norm(Vec3 a) { return std::sqrt(norm2(a)); }
// math.rs:38-46: multiply by the reciprocal, zero below 1e-15
inline Vec3 normalized(Vec3 a) {
  Real n = norm(a);
  if (n > 1e-15) return a * (1.0 / n);
  return v3zero();
}
inline Vec3 vabs(Vec3 a) { return v3(std::fabs(a[0]), std::fabs(a[1]), std::fabs(a[2])); }
inline Vec3 mul_elem(Vec3 a, Vec3 b) { return v3(a[0] * b[0], a[1] * b[1], a[2] * b[2]); }
// Rust f64::min/max: ignore NaN; ties irrelevant for finite values
inline Real rmin(Real a, Real b) { return std::fmin(a, b); }
inline Real rmax(Real a, Real b) { return std::fmax(a, b); }
inline Vec3 vmin(Vec3 a, Vec3 b) { return v3(rmin(a[0], b[0]), rmin(a[1], b[1]), rmin(a[2], b[2])); }
inline Vec3 vmax(Vec3 a, Vec3 b) { return v3(rmax(a[0], b[0]), rmax(a[1], b[1]), rmax(a[2], b[2])); }
inline Real clampr(Real x, Real lo, Real hi) { return x < lo ? lo : (x > hi ? hi : x); }
inline Real signum(Real x) { return std::signbit(x) ? -1.0 : 1.0; }  // Rust f64::signum (non-NaN)

// math.rs:65-70: two unit vectors completing a frame with a unit vector
inline void tangents(Vec3 n, Vec3* t1, Vec3* t2) {
  Vec3 a = std::fabs(n[0]) < 0.57 ? v3(1, 0, 0) : v3(0, 1, 0);
  *t1 = normalized(cross(n, a));
  *t2 = cross(n, *t1);
}

// ---------------------------------------------------------------- Mat3 (row-major)
// math.rs:130-212
struct Mat3 {
  Real m[9];
  Real& operator[](int i) { return m[i]; }
  Real operator[](int i) const { return m[i]; }
};
inline Mat3 m3identity() { return Mat3{{1, 0, 0, 0, 1, 0, 0, 0, 1}}; }
inline Mat3 m3zero() { return Mat3{{0, 0, 0, 0, 0, 0, 0, 0, 0}}; }
inline Mat3 m3diag(Vec3 d) { return Mat3{{d[0], 0, 0, 0, d[1], 0, 0, 0, d[2]}}; }
inline Mat3 m3cols(Vec3 a, Vec3 b, Vec3 c) { return Mat3{{a[0], b[0], c[0], a[1], b[1], c[1], a[2], b[2], c[2]}}; }
inline Vec3 col(const Mat3& m, int j) { return v3(m[j], m[3 + j], m[6 + j]); }
inline Vec3 mul_vec(const Mat3& m, Vec3 v) {
  return v3(m[0] * v[0] + m[1] * v[1] + m[2] * v[2], m[3] * v[0] + m[4] * v[1] + m[5] * v[2],
            m[6] * v[0] + m[7] * v[1] + m[8] * v[2]);
}
inline Vec3 tmul_vec(const Mat3& m, Vec3 v) {
  return v3(m[0] * v[0] + m[3] * v[1] + m[6] * v[2], m[1] * v[0] + m[4] * v[1] + m[7] * v[2],
            m[2] * v[0] + m[5] * v[1] + m[8] * v[2]);
}
// math.rs:172-180: each entry is a left-to-right sum of three products
inline Mat3 mul_mat(const Mat3& a, const Mat3& b) {
  Mat3 r;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      r[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
  return r;
}
inline Mat3 transpose(const Mat3& m) { return Mat3{{m[0], m[3], m[6], m[1], m[4], m[7], m[2], m[5], m[8]}}; }
inline Mat3 skew(Vec3 v) { return Mat3{{0.0, -v[2], v[1], v[2], 0.0, -v[0], -v[1], v[0], 0.0}}; }
inline Mat3 mscale(const Mat3& m, Real s) {
  Mat3 r;
  for (int i = 0; i < 9; i++) r[i] = m[i] * s;
  return r;
}
inline Mat3 madd(const Mat3& a, const Mat3& b) {
  Mat3 r;
  for (int i = 0; i < 9; i++) r[i] = a[i] + b[i];
  return r;
}
// math.rs:209-211: R * I * R^T
inline Mat3 mrotate(const Mat3& I, const Mat3& R) { return mul_mat(mul_mat(R, I), transpose(R)); }

// ---------------------------------------------------------------- Quat (w, x, y, z)
// math.rs:214-301
struct Quat {
  Real q[4];
  Real& operator[](int i) { return q[i]; }
  Real operator[](int i) const { return q[i]; }
};
inline Quat qidentity() { return Quat{{1, 0, 0, 0}}; }
inline Quat qaxis_angle(Vec3 axis, Real angle) {
  Vec3 a = normalized(axis);
  Real s = std::sin(0.5 * angle), c = std::cos(0.5 * angle);
  return Quat{{c, a[0] * s, a[1] * s, a[2] * s}};
}
// math.rs:229-235: divide by the norm; identity below 1e-15
inline Quat qnormalized(Quat q) {
  Real n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (n < 1e-15) return qidentity();
  return Quat{{q[0] / n, q[1] / n, q[2] / n, q[3] / n}};
}
inline Quat qmul(Quat p, Quat o) {
  Real a = p[0], b = p[1], c = p[2], d = p[3];
  Real e = o[0], f = o[1], g = o[2], h = o[3];
  return Quat{{a * e - b * f - c * g - d * h, a * f + b * e + c * h - d * g, a * g - b * h + c * e + d * f,
               a * h + b * g - c * f + d * e}};
}
inline Mat3 qto_mat(Quat q) {
  Real w = q[0], x = q[1], y = q[2], z = q[3];
  Real ww = w * w, xx = x * x, yy = y * y, zz = z * z;
  Real xy = x * y, xz = x * z, yz = y * z, wx = w * x, wy = w * y, wz = w * z;
  return Mat3{{ww + xx - yy - zz, 2.0 * (xy - wz), 2.0 * (xz + wy), 2.0 * (xy + wz), ww - xx + yy - zz,
               2.0 * (yz - wx), 2.0 * (xz - wy), 2.0 * (yz + wx), ww - xx - yy + zz}};
}
inline Vec3 qrotate(Quat q, Vec3 v) { return mul_vec(qto_mat(q), v); }
// math.rs:294-300: q * exp(omega h / 2) for a body-frame angular velocity
inline Quat qintegrate_local(Quat q, Vec3 omega, Real h) {
  Real n = norm(omega);
  if (n * h < 1e-15) return q;
  return qnormalized(qmul(q, qaxis_angle(omega * (1.0 / n), n * h)));
}

// ---------------------------------------------------------------- Spatial [ang; lin]
// math.rs:303-378: motion/force vectors in world axes about the world origin
struct Spatial {
  Vec3 ang, lin;
};
inline Spatial sp(Vec3 a, Vec3 l) { return Spatial{a, l}; }
inline Spatial spzero() { return Spatial{v3zero(), v3zero()}; }
inline Real spdot(const Spatial& a, const Spatial& b) { return dot(a.ang, b.ang) + dot(a.lin, b.lin); }
inline Spatial spscale(const Spatial& a, Real s) { return Spatial{a.ang * s, a.lin * s}; }
inline Spatial spadd(const Spatial& a, const Spatial& b) { return Spatial{a.ang + b.ang, a.lin + b.lin}; }
// self x m (motion cross motion)
inline Spatial cross_motion(const Spatial& s, const Spatial& m) {
  return Spatial{cross(s.ang, m.ang), cross(s.ang, m.lin) + cross(s.lin, m.ang)};
}
// self x* f (motion cross force)
inline Spatial cross_force(const Spatial& s, const Spatial& f) {
  return Spatial{cross(s.ang, f.ang) + cross(s.lin, f.lin), cross(s.ang, f.lin)};
}
inline Vec3 point_velocity(const Spatial& s, Vec3 p) { return s.lin + cross(s.ang, p); }

// ---------------------------------------------------------------- SpatialInertia
// math.rs:380-410: mass, first moment m*c, rotational inertia about the origin
struct SpInertia {
  Real mass;
  Vec3 mc;
  Mat3 io;
};
inline SpInertia spi_zero() { return SpInertia{0.0, v3zero(), m3zero()}; }
inline SpInertia spi_from_com(Real mass, Vec3 com, const Mat3& icom) {
  Mat3 cx = skew(com);
  Mat3 io = madd(icom, mscale(mul_mat(cx, transpose(cx)), mass));
  return SpInertia{mass, com * mass, io};
}
inline SpInertia spi_add(const SpInertia& a, const SpInertia& b) {
  return SpInertia{a.mass + b.mass, a.mc + b.mc, madd(a.io, b.io)};
}
inline Spatial spi_mul(const SpInertia& I, const Spatial& v) {
  return Spatial{mul_vec(I.io, v.ang) + cross(I.mc, v.lin), v.lin * I.mass - cross(I.mc, v.ang)};
}

// ---------------------------------------------------------------- dot / axpy
// simd.rs:14-64 (x86 branch :47-63): sequential below 8 terms, else four
// interleaved accumulators combined as (s0+s1)+(s2+s3), then the tail.
inline Real vdot(const Real* a, const Real* b, size_t n) {
  if (n < 8) {
    Real s = 0.0;
    for (size_t k = 0; k < n; k++) s += a[k] * b[k];
    return s;
  }
  Real s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  size_t k = 0;
  while (k + 4 <= n) {
    s0 += a[k] * b[k];
    s1 += a[k + 1] * b[k + 1];
    s2 += a[k + 2] * b[k + 2];
    s3 += a[k + 3] * b[k + 3];
    k += 4;
  }
  Real t = (s0 + s1) + (s2 + s3);
  while (k < n) {
    t += a[k] * b[k];
    k++;
  }
  return t;
}
// simd.rs:68-72
inline void vaxpy(Real alpha, const Real* x, Real* y, size_t n) {
  for (size_t k = 0; k < n; k++) y[k] += alpha * x[k];
}

// ---------------------------------------------------------------- Cholesky
// math.rs:425-447: in-place lower Cholesky of the diagonal block [s0, s1) of a
// row-major matrix with row stride `stride`; false if not positive definite.
inline bool cholesky_block(Real* a, size_t stride, size_t s0, size_t s1) {
  for (size_t j = s0; j < s1; j++) {
    Real* rj = a + j * stride + s0;
    Real d = a[j * stride + j] - vdot(rj, rj, j - s0);
    if (d <= 0.0) return false;
    d = std::sqrt(d);
    a[j * stride + j] = d;
    Real inv = 1.0 / d;
    for (size_t i = j + 1; i < s1; i++) {
      Real* ri = a + i * stride + s0;
      size_t k = j - s0;
      ri[k] = (ri[k] - vdot(ri, rj, k)) * inv;
    }
  }
  return true;
}
// math.rs:451-463
inline void cholesky_solve_block(const Real* l, size_t stride, size_t s0, size_t s1, Real* x) {
  for (size_t i = s0; i < s1; i++)
    x[i] = (x[i] - vdot(l + i * stride + s0, x + s0, i - s0)) / l[i * stride + i];
  for (size_t i = s1; i-- > s0;) {
    x[i] /= l[i * stride + i];
    Real xi = x[i];
    vaxpy(-xi, l + i * stride + s0, x + s0, i - s0);
  }
}
inline bool cholesky(Real* a, size_t n) { return cholesky_block(a, n, 0, n); }
inline void cholesky_solve(const Real* l, size_t n, Real* x) { cholesky_solve_block(l, n, 0, n, x); }

}  // namespace om
