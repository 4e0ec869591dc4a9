// App-facing quaternion type with the names the reference's apps and host
// helpers use (FunDEM/kernel/CUDAKernelFunction/myUtility/myQua.h): q0 is the
// scalar part, the rotation maps the body frame to the world frame.
#pragma once
#include "myVec.h"

struct quaternion {
  double q0, q1, q2, q3;
};

HOST_DEVICE inline quaternion make_quaternion(double q0, double q1, double q2, double q3) {
  quaternion q;
  q.q0 = q0; q.q1 = q1; q.q2 = q2; q.q3 = q3;
  return q;
}
HOST_DEVICE inline quaternion operator+(quaternion a, quaternion b) {
  return make_quaternion(a.q0 + b.q0, a.q1 + b.q1, a.q2 + b.q2, a.q3 + b.q3);
}
HOST_DEVICE inline quaternion operator*(quaternion q, double c) { return make_quaternion(q.q0 * c, q.q1 * c, q.q2 * c, q.q3 * c); }
HOST_DEVICE inline quaternion operator*(double c, quaternion q) { return q * c; }
HOST_DEVICE inline quaternion operator/(quaternion q, double c) { return q * (1.0 / c); }

HOST_DEVICE inline quaternion normalize(quaternion q) {
  const double l2 = q.q0 * q.q0 + q.q1 * q.q1 + q.q2 * q.q2 + q.q3 * q.q3;
  if (isZero(l2)) return q;
#ifdef __CUDA_ARCH__
  const double inv = rsqrt(l2);
#else
  const double inv = 1.0 / sqrt(l2);
#endif
  return make_quaternion(q.q0 * inv, q.q1 * inv, q.q2 * inv, q.q3 * inv);
}
HOST_DEVICE inline quaternion conjugate(quaternion q) { return make_quaternion(q.q0, -q.q1, -q.q2, -q.q3); }

// Explicit Euler step of q_dot = 1/2 (0, w) (x) q with world-frame w, then normalise.
HOST_DEVICE inline quaternion quaternionIntegration(quaternion q, double3 w, double dt) {
  const double3 v = w * (0.5 * dt);
  quaternion d;
  d.q0 = -q.q1 * v.x - q.q2 * v.y - q.q3 * v.z;
  d.q1 = q.q0 * v.x + q.q3 * v.y - q.q2 * v.z;
  d.q2 = -q.q3 * v.x + q.q0 * v.y + q.q1 * v.z;
  d.q3 = q.q2 * v.x - q.q1 * v.y + q.q0 * v.z;
  return normalize(q + d);
}

// v' = v + q0 t + qv x t with t = 2 qv x v.
HOST_DEVICE inline double3 rotateVectorByQuaternion(quaternion q, double3 v) {
  const double3 qv = make_double3(q.q1, q.q2, q.q3);
  const double3 t = cross(qv, v) * 2.0;
  return v + (t * q.q0) + cross(qv, t);
}
HOST_DEVICE inline double3 reverseRotateVectorByQuaternion(double3 v, quaternion q) {
  return rotateVectorByQuaternion(conjugate(q), v);
}

// World-frame rotation by the rotation vector omega applied to q, normalised.
HOST_DEVICE inline quaternion rotateQuaternion(const quaternion& q, const double3& omega) {
  const double t2 = dot(omega, omega);
  if (isZero(t2)) return q;
  const double t = sqrt(t2);
  const double s = sin(0.5 * t) / t, c = cos(0.5 * t);
  const double r0 = c, r1 = s * omega.x, r2 = s * omega.y, r3 = s * omega.z;
  quaternion r;
  r.q0 = r0 * q.q0 - r1 * q.q1 - r2 * q.q2 - r3 * q.q3;
  r.q1 = r0 * q.q1 + r1 * q.q0 + r2 * q.q3 - r3 * q.q2;
  r.q2 = r0 * q.q2 - r1 * q.q3 + r2 * q.q0 + r3 * q.q1;
  r.q3 = r0 * q.q3 + r1 * q.q2 - r2 * q.q1 + r3 * q.q0;
  return normalize(r);
}
