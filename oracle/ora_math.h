// FP64 CPU oracle — TEST INFRASTRUCTURE ONLY.
// Vector / quaternion / symmetric-matrix helpers restating the host-side
// semantics of the reference math layer:
//   FunDEM/kernel/CUDAKernelFunction/myUtility/myVec.h  (dot, cross, normalize via 1/sqrt, isZero |x|<=1e-20)
//   FunDEM/kernel/CUDAKernelFunction/myUtility/myQua.h  (rotateVectorByQuaternion :104-114,
//        reverseRotateVectorByQuaternion :120-129, quaternionIntegration :77-93)
//   FunDEM/kernel/CUDAKernelFunction/myUtility/myMat.h  (rotateInverseInertiaTensorByQuaternion :107-158,
//        inverse :163-195)
// The expression order follows those functions so that the CPU results match
// the reference's host arithmetic. Compiled with -ffp-contract=off.
#pragma once
#include <cmath>

namespace ora {

struct d3 { double x, y, z; };
struct qt { double q0, q1, q2, q3; };          // q0 = scalar part
struct sm { double xx, yy, zz, xy, xz, yz; };   // symmetric 3x3

inline d3 mk(double x, double y, double z) { return d3{x, y, z}; }
inline d3 operator+(d3 a, d3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline d3 operator-(d3 a, d3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline d3 operator-(d3 a) { return mk(-a.x, -a.y, -a.z); }
inline d3 operator*(d3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
inline d3 operator*(double s, d3 a) { return mk(a.x * s, a.y * s, a.z * s); }
inline d3 operator/(d3 a, double s) { double inv = 1.0 / s; return mk(a.x * inv, a.y * inv, a.z * inv); }
inline d3& operator+=(d3& a, d3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
inline d3& operator-=(d3& a, d3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
inline d3& operator*=(d3& a, double s) { a.x *= s; a.y *= s; a.z *= s; return a; }

inline bool is_zero(double x) { return std::fabs(x) <= 1.0e-20; }
inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline d3 cross(d3 a, d3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline double len2(d3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
inline double len(d3 v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
inline d3 normalize(d3 v) {
  double l2 = v.x * v.x + v.y * v.y + v.z * v.z;
  if (is_zero(l2)) return mk(0.0, 0.0, 0.0);
  double inv = 1.0 / std::sqrt(l2);
  return mk(v.x * inv, v.y * inv, v.z * inv);
}

inline qt normalize(qt q) {
  double l2 = q.q0 * q.q0 + q.q1 * q.q1 + q.q2 * q.q2 + q.q3 * q.q3;
  if (is_zero(l2)) return q;
  double inv = 1.0 / std::sqrt(l2);
  return qt{q.q0 * inv, q.q1 * inv, q.q2 * inv, q.q3 * inv};
}

// v' = v + q0*t + qv x t,  t = 2 (qv x v)
inline d3 rotate(qt q, d3 v) {
  d3 qv = mk(q.q1, q.q2, q.q3);
  d3 t = cross(qv, v) * 2.0;
  return v + (t * q.q0) + cross(qv, t);
}
// rotation by the conjugate
inline d3 rotate_inv(d3 v, qt q) {
  d3 qv = mk(-q.q1, -q.q2, -q.q3);
  d3 t = cross(qv, v) * 2.0;
  return v + (t * q.q0) + cross(qv, t);
}

// explicit Euler on q_dot = 1/2 (0, w) (x) q, then normalise
inline qt integrate_q(qt q, d3 w, double dt) {
  d3 v = w * (0.5 * dt);
  qt d;
  d.q0 = -q.q1 * v.x - q.q2 * v.y - q.q3 * v.z;
  d.q1 = q.q0 * v.x + q.q3 * v.y - q.q2 * v.z;
  d.q2 = -q.q3 * v.x + q.q0 * v.y + q.q1 * v.z;
  d.q3 = q.q2 * v.x - q.q1 * v.y + q.q0 * v.z;
  return normalize(qt{q.q0 + d.q0, q.q1 + d.q1, q.q2 + d.q2, q.q3 + d.q3});
}

// R * invI * R^T with R built from q
inline sm rotate_inv_inertia(qt q, sm I) {
  double q0 = q.q0, q1 = q.q1, q2 = q.q2, q3 = q.q3;
  double q11 = 2 * q1 * q1, q22 = 2 * q2 * q2, q33 = 2 * q3 * q3;
  double a = 1.0 - q22 - q33, b = 2 * (q1 * q2 - q0 * q3), c = 2 * (q1 * q3 + q0 * q2);
  double d = 2 * (q1 * q2 + q0 * q3), e = 1.0 - q11 - q33, f = 2 * (q2 * q3 - q0 * q1);
  double g = 2 * (q1 * q3 - q0 * q2), h = 2 * (q2 * q3 + q0 * q1), i = 1.0 - q11 - q22;
  double r0x = I.xx * a + I.xy * b + I.xz * c, r0y = I.xy * a + I.yy * b + I.yz * c, r0z = I.xz * a + I.yz * b + I.zz * c;
  double r1x = I.xx * d + I.xy * e + I.xz * f, r1y = I.xy * d + I.yy * e + I.yz * f, r1z = I.xz * d + I.yz * e + I.zz * f;
  double r2x = I.xx * g + I.xy * h + I.xz * i, r2y = I.xy * g + I.yy * h + I.yz * i, r2z = I.xz * g + I.yz * h + I.zz * i;
  return sm{r0x * a + r0y * b + r0z * c, r1x * d + r1y * e + r1z * f, r2x * g + r2y * h + r2z * i,
            r0x * d + r0y * e + r0z * f, r0x * g + r0y * h + r0z * i, r1x * g + r1y * h + r1z * i};
}
inline d3 mul(sm m, d3 v) {
  return mk(m.xx * v.x + m.xy * v.y + m.xz * v.z, m.xy * v.x + m.yy * v.y + m.yz * v.z,
            m.xz * v.x + m.yz * v.y + m.zz * v.z);
}
inline sm inverse(sm A) {
  double det = A.xx * (A.yy * A.zz - A.yz * A.yz) + A.xy * (A.yz * A.xz - A.xy * A.zz) +
               A.xz * (A.xy * A.yz - A.yy * A.xz);
  if (std::fabs(det) < 1e-30) return sm{0, 0, 0, 0, 0, 0};
  double di = 1.0 / det;
  return sm{(A.yy * A.zz - A.yz * A.yz) * di, (A.xx * A.zz - A.xz * A.xz) * di, (A.xx * A.yy - A.xy * A.xy) * di,
            -(A.xy * A.zz - A.xz * A.yz) * di, (A.xy * A.yz - A.xz * A.yy) * di, -(A.xx * A.yz - A.xz * A.xy) * di};
}

inline int lin3(int x, int y, int z, int nx, int ny) { return z * ny * nx + y * nx + x; }

}  // namespace ora
