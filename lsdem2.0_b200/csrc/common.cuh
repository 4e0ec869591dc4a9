// Shared device types and math for the B200 level-set DEM step.
//
// Arithmetic conventions follow the reference device code so that integer
// outcomes (cell keys, contact pairs) coincide with it:
//   rotation by a quaternion      FunDEM/kernel/CUDAKernelFunction/myUtility/myQua.h:104-129
//   quaternion Euler update       myQua.h:77-93 (normalised with rsqrt on the device)
//   vector normalise (rsqrt)      myVec.h:121-137
//   inverse-inertia rotation      myMat.h:107-158
//   cell coordinate (int trunc.)  mySpatialGrid.h:24-31
//   linear cell index             myVec.h:232-235
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace lsdem {

struct Quat { double q0, q1, q2, q3; };           // q0 = scalar part, local -> world
struct Sym6 { double xx, yy, zz, xy, xz, yz; };   // symmetric 3x3

#define LD __device__ __forceinline__
#define HD __host__ __device__ __forceinline__

HD double3 d3(double x, double y, double z) { return make_double3(x, y, z); }
HD double3 operator+(double3 a, double3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
HD double3 operator-(double3 a, double3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
HD double3 operator-(double3 a) { return d3(-a.x, -a.y, -a.z); }
HD double3 operator*(double3 a, double s) { return d3(a.x * s, a.y * s, a.z * s); }
HD double3 operator*(double s, double3 a) { return d3(a.x * s, a.y * s, a.z * s); }
HD double3 operator/(double3 a, double s) { double inv = 1.0 / s; return d3(a.x * inv, a.y * inv, a.z * inv); }
HD double3& operator+=(double3& a, double3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
HD double3& operator-=(double3& a, double3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
HD double3& operator*=(double3& a, double s) { a.x *= s; a.y *= s; a.z *= s; return a; }
HD double dot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
HD double3 cross(double3 a, double3 b) { return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
HD double len2(double3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
HD double len(double3 v) { return sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
HD bool is_zero(double x) { return fabs(x) <= 1.0e-20; }

LD double3 normalize_dev(double3 v) {
  double l2 = v.x * v.x + v.y * v.y + v.z * v.z;
  if (is_zero(l2)) return d3(0., 0., 0.);
  double inv = rsqrt(l2);
  return d3(v.x * inv, v.y * inv, v.z * inv);
}

HD double3 rotate(Quat q, double3 v) {
  double3 qv = d3(q.q1, q.q2, q.q3);
  double3 t = cross(qv, v) * 2.0;
  return v + (t * q.q0) + cross(qv, t);
}
HD double3 rotate_inv(double3 v, Quat q) {
  double3 qv = d3(-q.q1, -q.q2, -q.q3);
  double3 t = cross(qv, v) * 2.0;
  return v + (t * q.q0) + cross(qv, t);
}

LD Quat quat_integrate(Quat q, double3 w, double dt) {
  double3 v = w * (0.5 * dt);
  Quat d;
  d.q0 = -q.q1 * v.x - q.q2 * v.y - q.q3 * v.z;
  d.q1 = q.q0 * v.x + q.q3 * v.y - q.q2 * v.z;
  d.q2 = -q.q3 * v.x + q.q0 * v.y + q.q1 * v.z;
  d.q3 = q.q2 * v.x - q.q1 * v.y + q.q0 * v.z;
  Quat r{q.q0 + d.q0, q.q1 + d.q1, q.q2 + d.q2, q.q3 + d.q3};
  double l2 = r.q0 * r.q0 + r.q1 * r.q1 + r.q2 * r.q2 + r.q3 * r.q3;
  if (is_zero(l2)) return r;
  double inv = rsqrt(l2);
  return Quat{r.q0 * inv, r.q1 * inv, r.q2 * inv, r.q3 * inv};
}

// Rotation of v by the rotation vector om (axis om / |om|, angle |om|), Rodrigues'
// formula with a second-order expansion below |om|^2 = 1e-20 and the device's rsqrt
// and sincos, as the reference's device rotateVector (myVec.h:143-182).
LD double3 rotate_vector_dev(double3 v, double3 om) {
  const double theta2 = dot(om, om);
  const double3 oxv = cross(om, v);
  const double3 oxoxv = cross(om, oxv);
  if (is_zero(theta2)) return v + oxv + 0.5 * oxoxv;
  const double inv = rsqrt(theta2);
  const double theta = theta2 * inv;
  double s, c;
  sincos(theta, &s, &c);
  const double A = s * inv;
  const double B = (1.0 - c) * (inv * inv);
  return v + A * oxv + B * oxoxv;
}

// q turned by the rotation vector om in the global frame, rot(om) * q, normalised
// with the device's rsqrt (rotateQuaternion, myQua.h:131-179).
LD Quat rotate_quaternion_dev(Quat q, double3 om) {
  const double theta2 = om.x * om.x + om.y * om.y + om.z * om.z;
  if (is_zero(theta2)) return q;
  const double theta = sqrt(theta2);
  const double inv = 1.0 / theta;
  const double ux = om.x * inv, uy = om.y * inv, uz = om.z * inv;
  const double half = 0.5 * theta;
  const double c = cos(half), s = sin(half);
  const double r0 = c, r1 = s * ux, r2 = s * uy, r3 = s * uz;
  Quat r;
  r.q0 = r0 * q.q0 - r1 * q.q1 - r2 * q.q2 - r3 * q.q3;
  r.q1 = r0 * q.q1 + r1 * q.q0 + r2 * q.q3 - r3 * q.q2;
  r.q2 = r0 * q.q2 - r1 * q.q3 + r2 * q.q0 + r3 * q.q1;
  r.q3 = r0 * q.q3 + r1 * q.q2 - r2 * q.q1 + r3 * q.q0;
  const double l2 = r.q0 * r.q0 + r.q1 * r.q1 + r.q2 * r.q2 + r.q3 * r.q3;
  if (is_zero(l2)) return r;
  const double il = rsqrt(l2);
  return Quat{r.q0 * il, r.q1 * il, r.q2 * il, r.q3 * il};
}

HD Sym6 rotate_inv_inertia(Quat q, Sym6 I) {
  double q0 = q.q0, q1 = q.q1, q2 = q.q2, q3 = q.q3;
  double q11 = 2 * q1 * q1, q22 = 2 * q2 * q2, q33 = 2 * q3 * q3;
  double a = 1.0 - q22 - q33, b = 2 * (q1 * q2 - q0 * q3), c = 2 * (q1 * q3 + q0 * q2);
  double d = 2 * (q1 * q2 + q0 * q3), e = 1.0 - q11 - q33, f = 2 * (q2 * q3 - q0 * q1);
  double g = 2 * (q1 * q3 - q0 * q2), h = 2 * (q2 * q3 + q0 * q1), i = 1.0 - q11 - q22;
  double r0x = I.xx * a + I.xy * b + I.xz * c, r0y = I.xy * a + I.yy * b + I.yz * c, r0z = I.xz * a + I.yz * b + I.zz * c;
  double r1x = I.xx * d + I.xy * e + I.xz * f, r1y = I.xy * d + I.yy * e + I.yz * f, r1z = I.xz * d + I.yz * e + I.zz * f;
  double r2x = I.xx * g + I.xy * h + I.xz * i, r2y = I.xy * g + I.yy * h + I.yz * i, r2z = I.xz * g + I.yz * h + I.zz * i;
  return Sym6{r0x * a + r0y * b + r0z * c, r1x * d + r1y * e + r1z * f, r2x * g + r2y * h + r2z * i,
              r0x * d + r0y * e + r0z * f, r0x * g + r0y * h + r0z * i, r1x * g + r1y * h + r1z * i};
}
HD double3 mul(Sym6 m, double3 v) {
  return d3(m.xx * v.x + m.xy * v.y + m.xz * v.z, m.xy * v.x + m.yy * v.y + m.yz * v.z,
            m.xz * v.x + m.yz * v.y + m.zz * v.z);
}

// Row-major rotation matrix of q (used only for conservative culling).
struct Mat3 { double m[9]; };
HD Mat3 quat_to_mat(Quat q) {
  double q0 = q.q0, q1 = q.q1, q2 = q.q2, q3 = q.q3;
  Mat3 r;
  r.m[0] = 1.0 - 2 * (q2 * q2 + q3 * q3); r.m[1] = 2 * (q1 * q2 - q0 * q3); r.m[2] = 2 * (q1 * q3 + q0 * q2);
  r.m[3] = 2 * (q1 * q2 + q0 * q3); r.m[4] = 1.0 - 2 * (q1 * q1 + q3 * q3); r.m[5] = 2 * (q2 * q3 - q0 * q1);
  r.m[6] = 2 * (q1 * q3 - q0 * q2); r.m[7] = 2 * (q2 * q3 + q0 * q1); r.m[8] = 1.0 - 2 * (q1 * q1 + q2 * q2);
  return r;
}
HD double3 mat_mul(const Mat3& r, double3 v) {
  return d3(r.m[0] * v.x + r.m[1] * v.y + r.m[2] * v.z, r.m[3] * v.x + r.m[4] * v.y + r.m[5] * v.z,
            r.m[6] * v.x + r.m[7] * v.y + r.m[8] * v.z);
}
HD double3 mat_tmul(const Mat3& r, double3 v) {
  return d3(r.m[0] * v.x + r.m[3] * v.y + r.m[6] * v.z, r.m[1] * v.x + r.m[4] * v.y + r.m[7] * v.z,
            r.m[2] * v.x + r.m[5] * v.y + r.m[8] * v.z);
}

// Uniform hash grid parameters (mySpatialGrid.h:162-240).
struct GridP {
  double3 mn, mx, inv;
  int3 size;
  int ncells;
};

HD int3 cell_of(double3 p, const GridP& g) {
  return make_int3(int((p.x - g.mn.x) * g.inv.x), int((p.y - g.mn.y) * g.inv.y), int((p.z - g.mn.z) * g.inv.z));
}
HD int lin3(int3 c, int3 s) { return c.z * s.y * s.x + c.y * s.x + c.x; }
HD int3 clamp_cell(int3 c, int3 s) {
  c.x = c.x <= 0 ? 0 : (c.x >= s.x - 1 ? s.x - 1 : c.x);
  c.y = c.y <= 0 ? 0 : (c.y >= s.y - 1 ? s.y - 1 : c.y);
  c.z = c.z <= 0 ? 0 : (c.z >= s.z - 1 ? s.z - 1 : c.z);
  return c;
}
// Cell key of a body centre, -1 outside [mn, mx) (mySpatialGrid.cu:4-26).
HD int hash_key(double3 p, const GridP& g) {
  if (p.x < g.mn.x || p.x >= g.mx.x || p.y < g.mn.y || p.y >= g.mx.y || p.z < g.mn.z || p.z >= g.mx.z) return -1;
  return lin3(cell_of(p, g), g.size);
}
// The neighbourhood a node at p scans: clamped cell c, offsets [lo, hi] per axis
// (LSParticleContactDetectionKernel.cu:35-43).
HD void node_window(double3 p, const GridP& g, int3& c, int3& lo, int3& hi) {
  c = cell_of(p, g);
  lo = make_int3(-1, -1, -1);
  hi = make_int3(1, 1, 1);
  if (c.x <= 0) { c.x = 0; lo.x = 0; }
  if (c.x >= g.size.x - 1) { c.x = g.size.x - 1; hi.x = 0; }
  if (c.y <= 0) { c.y = 0; lo.y = 0; }
  if (c.y >= g.size.y - 1) { c.y = g.size.y - 1; hi.y = 0; }
  if (c.z <= 0) { c.z = 0; lo.z = 0; }
  if (c.z >= g.size.z - 1) { c.z = g.size.z - 1; hi.z = 0; }
}
HD bool in_window(int key, const GridP& g, int3 c, int3 lo, int3 hi) {
  int kx = key % g.size.x;
  int ky = (key / g.size.x) % g.size.y;
  int kz = key / (g.size.x * g.size.y);
  return kx >= c.x + lo.x && kx <= c.x + hi.x && ky >= c.y + lo.y && ky <= c.y + hi.y && kz >= c.z + lo.z &&
         kz <= c.z + hi.z;
}

}  // namespace lsdem
