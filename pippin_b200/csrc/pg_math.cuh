// Device math for the batched FP64 substep: 3-vectors, row-major 3x3
// matrices, (w, x, y, z) quaternions, spatial vectors [ang; lin] about the
// world origin and compact spatial inertias (mass, m*c, I about the origin).
// Conventions and operation order follow crates/pippin/src/math.rs:9-410 so
// results agree with the reference to rounding (nvcc may contract a*b+c into
// one FMA; the tolerance in the parity tests covers that).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace pg {

struct V3 {
  double x, y, z;
};
struct M3 {
  double m[9];
};
struct Q4 {
  double w, x, y, z;
};
struct Sp {  // spatial motion/force vector, world axes about the origin
  V3 ang, lin;
};
struct SpI {  // spatial inertia about the origin
  double mass;
  V3 mc;
  M3 io;
};

__host__ __device__ inline V3 v3(double x, double y, double z) { return V3{x, y, z}; }
__host__ __device__ inline V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
__host__ __device__ inline V3 operator*(V3 a, double s) { return V3{a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline V3 cross(V3 a, V3 b) {
  return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ inline double norm2(V3 a) { return dot(a, a); }
__host__ __device__ inline double norm(V3 a) { return sqrt(norm2(a)); }
// math.rs:38-46
__host__ __device__ inline V3 normalized(V3 a) {
  double n = norm(a);
  return n > 1e-15 ? a * (1.0 / n) : V3{0.0, 0.0, 0.0};
}
__host__ __device__ inline V3 vabs(V3 a) { return V3{fabs(a.x), fabs(a.y), fabs(a.z)}; }
__host__ __device__ inline V3 mul_elem(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__host__ __device__ inline V3 vmax(V3 a, V3 b) { return V3{fmax(a.x, b.x), fmax(a.y, b.y), fmax(a.z, b.z)}; }
__host__ __device__ inline double clampd(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }
__host__ __device__ inline double signum(double x) { return signbit(x) ? -1.0 : 1.0; }
__host__ __device__ inline double comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
__host__ __device__ inline void set_comp(V3& a, int i, double v) {
  if (i == 0) a.x = v;
  else if (i == 1) a.y = v;
  else a.z = v;
}
// math.rs:65-70
__host__ __device__ inline void tangents(V3 n, V3* t1, V3* t2) {
  V3 a = fabs(n.x) < 0.57 ? V3{1, 0, 0} : V3{0, 1, 0};
  *t1 = normalized(cross(n, a));
  *t2 = cross(n, *t1);
}

__host__ __device__ inline M3 m3_identity() { return M3{{1, 0, 0, 0, 1, 0, 0, 0, 1}}; }
__host__ __device__ inline V3 col(const M3& m, int j) { return V3{m.m[j], m.m[3 + j], m.m[6 + j]}; }
__host__ __device__ inline V3 mv(const M3& m, V3 v) {
  return V3{m.m[0] * v.x + m.m[1] * v.y + m.m[2] * v.z, m.m[3] * v.x + m.m[4] * v.y + m.m[5] * v.z,
            m.m[6] * v.x + m.m[7] * v.y + m.m[8] * v.z};
}
__host__ __device__ inline V3 mtv(const M3& m, V3 v) {
  return V3{m.m[0] * v.x + m.m[3] * v.y + m.m[6] * v.z, m.m[1] * v.x + m.m[4] * v.y + m.m[7] * v.z,
            m.m[2] * v.x + m.m[5] * v.y + m.m[8] * v.z};
}
__host__ __device__ inline M3 mm(const M3& a, const M3& b) {
  M3 r;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) r.m[3 * i + j] = a.m[3 * i] * b.m[j] + a.m[3 * i + 1] * b.m[3 + j] + a.m[3 * i + 2] * b.m[6 + j];
  return r;
}
__host__ __device__ inline M3 mt(const M3& a) {
  return M3{{a.m[0], a.m[3], a.m[6], a.m[1], a.m[4], a.m[7], a.m[2], a.m[5], a.m[8]}};
}
// R * I * R^T (math.rs:209-211)
__host__ __device__ inline M3 mrot(const M3& I, const M3& R) { return mm(mm(R, I), mt(R)); }

// ---- quaternions (math.rs:214-301)
__host__ __device__ inline Q4 q_identity() { return Q4{1, 0, 0, 0}; }
__device__ inline Q4 q_axis_angle(V3 axis, double angle) {
  V3 a = normalized(axis);
  double s, c;
  sincos(0.5 * angle, &s, &c);
  return Q4{c, a.x * s, a.y * s, a.z * s};
}
__host__ __device__ inline Q4 q_normalized(Q4 q) {
  double n = sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
  if (n < 1e-15) return q_identity();
  return Q4{q.w / n, q.x / n, q.y / n, q.z / n};
}
__host__ __device__ inline Q4 q_mul(Q4 p, Q4 o) {
  return Q4{p.w * o.w - p.x * o.x - p.y * o.y - p.z * o.z, p.w * o.x + p.x * o.w + p.y * o.z - p.z * o.y,
            p.w * o.y - p.x * o.z + p.y * o.w + p.z * o.x, p.w * o.z + p.x * o.y - p.y * o.x + p.z * o.w};
}
__host__ __device__ inline M3 q_mat(Q4 q) {
  double ww = q.w * q.w, xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z;
  double xy = q.x * q.y, xz = q.x * q.z, yz = q.y * q.z, wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
  return M3{{ww + xx - yy - zz, 2.0 * (xy - wz), 2.0 * (xz + wy), 2.0 * (xy + wz), ww - xx + yy - zz, 2.0 * (yz - wx),
             2.0 * (xz - wy), 2.0 * (yz + wx), ww - xx - yy + zz}};
}
__host__ __device__ inline V3 q_rot(Q4 q, V3 v) { return mv(q_mat(q), v); }
// q * exp(omega h / 2), body-frame angular velocity (math.rs:294-300)
__device__ inline Q4 q_integrate_local(Q4 q, V3 w, double h) {
  double n = norm(w);
  if (n * h < 1e-15) return q;
  return q_normalized(q_mul(q, q_axis_angle(w * (1.0 / n), n * h)));
}

// ---- spatial algebra (math.rs:303-410)
__host__ __device__ inline Sp sp(V3 a, V3 l) { return Sp{a, l}; }
__host__ __device__ inline Sp sp_zero() { return Sp{{0, 0, 0}, {0, 0, 0}}; }
__host__ __device__ inline double sp_dot(const Sp& a, const Sp& b) { return dot(a.ang, b.ang) + dot(a.lin, b.lin); }
__host__ __device__ inline Sp sp_add(const Sp& a, const Sp& b) { return Sp{a.ang + b.ang, a.lin + b.lin}; }
__host__ __device__ inline Sp sp_scale(const Sp& a, double s) { return Sp{a.ang * s, a.lin * s}; }
__host__ __device__ inline Sp cross_motion(const Sp& s, const Sp& m) {
  return Sp{cross(s.ang, m.ang), cross(s.ang, m.lin) + cross(s.lin, m.ang)};
}
__host__ __device__ inline Sp cross_force(const Sp& s, const Sp& f) {
  return Sp{cross(s.ang, f.ang) + cross(s.lin, f.lin), cross(s.ang, f.lin)};
}
__host__ __device__ inline V3 point_vel(const Sp& s, V3 p) { return s.lin + cross(s.ang, p); }
__host__ __device__ inline SpI spi_from_com(double mass, V3 com, const M3& icom) {
  // I_O = I_c + m [c]x [c]x^T  ([c]x [c]x^T = |c|^2 1 - c c^T, written out as the product)
  M3 cx{{0.0, -com.z, com.y, com.z, 0.0, -com.x, -com.y, com.x, 0.0}};
  M3 p = mm(cx, mt(cx));
  SpI r;
  r.mass = mass;
  r.mc = com * mass;
#pragma unroll
  for (int k = 0; k < 9; k++) r.io.m[k] = icom.m[k] + p.m[k] * mass;
  return r;
}
__host__ __device__ inline Sp spi_mul(const SpI& I, const Sp& v) {
  return Sp{mv(I.io, v.ang) + cross(I.mc, v.lin), v.lin * I.mass - cross(I.mc, v.ang)};
}

// ---- packed loads/stores (a SpI is 13 doubles: mass, mc[3], io[9])
__host__ __device__ inline V3 ld3(const double* p) { return V3{p[0], p[1], p[2]}; }
__host__ __device__ inline void st3(double* p, V3 v) {
  p[0] = v.x;
  p[1] = v.y;
  p[2] = v.z;
}
__host__ __device__ inline M3 ld9(const double* p) {
  M3 r;
#pragma unroll
  for (int k = 0; k < 9; k++) r.m[k] = p[k];
  return r;
}
__host__ __device__ inline void st9(double* p, const M3& m) {
#pragma unroll
  for (int k = 0; k < 9; k++) p[k] = m.m[k];
}
__host__ __device__ inline Q4 ld4(const double* p) { return Q4{p[0], p[1], p[2], p[3]}; }
__host__ __device__ inline void st4(double* p, Q4 q) {
  p[0] = q.w;
  p[1] = q.x;
  p[2] = q.y;
  p[3] = q.z;
}
__host__ __device__ inline Sp ld6(const double* p) { return Sp{ld3(p), ld3(p + 3)}; }
__host__ __device__ inline void st6(double* p, const Sp& s) {
  st3(p, s.ang);
  st3(p + 3, s.lin);
}
__host__ __device__ inline SpI ld13(const double* p) { return SpI{p[0], ld3(p + 1), ld9(p + 4)}; }
__host__ __device__ inline void st13(double* p, const SpI& s) {
  p[0] = s.mass;
  st3(p + 1, s.mc);
  st9(p + 4, s.io);
}

// Dot product with the reference's summation order (simd.rs:14-64, x86
// branch): sequential below 8 terms, else 4 interleaved accumulators
// combined as (s0+s1)+(s2+s3) followed by the tail. `sa`/`sb` are strides.
__device__ inline double dot_ref(const double* a, int sa, const double* b, int sb, int n) {
  if (n < 8) {
    double s = 0.0;
    for (int k = 0; k < n; k++) s += a[k * sa] * b[k * sb];
    return s;
  }
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int k = 0;
  for (; k + 4 <= n; k += 4) {
    s0 += a[k * sa] * b[k * sb];
    s1 += a[(k + 1) * sa] * b[(k + 1) * sb];
    s2 += a[(k + 2) * sa] * b[(k + 2) * sb];
    s3 += a[(k + 3) * sa] * b[(k + 3) * sb];
  }
  double t = (s0 + s1) + (s2 + s3);
  for (; k < n; k++) t += a[k * sa] * b[k * sb];
  return t;
}

}  // namespace pg
