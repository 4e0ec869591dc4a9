// App-facing symmetric 3x3 matrix (xx, yy, zz, xy, xz, yz) with the names the
// reference's apps and host helpers use (FunDEM/kernel/CUDAKernelFunction/myUtility/myMat.h).
#pragma once
#include "myQua.h"

struct symMatrix {
  double xx, yy, zz, xy, xz, yz;
  HOST_DEVICE symMatrix() : xx(0.0), yy(0.0), zz(0.0), xy(0.0), xz(0.0), yz(0.0) {}
  HOST_DEVICE symMatrix(double a, double b, double c, double d, double e, double f)
      : xx(a), yy(b), zz(c), xy(d), xz(e), yz(f) {}
};

HOST_DEVICE inline symMatrix make_symMatrix(double xx, double yy, double zz, double xy, double xz, double yz) {
  return symMatrix(xx, yy, zz, xy, xz, yz);
}
HOST_DEVICE inline double norm(symMatrix m) {
  return sqrt(m.xx * m.xx + m.yy * m.yy + m.zz * m.zz + 2.0 * (m.xy * m.xy + m.xz * m.xz + m.yz * m.yz));
}
HOST_DEVICE inline symMatrix deviatoric(symMatrix m) {
  const double tr = (m.xx + m.yy + m.zz) / 3.0;
  return symMatrix(m.xx - tr, m.yy - tr, m.zz - tr, m.xy, m.xz, m.yz);
}
HOST_DEVICE inline symMatrix operator+(symMatrix a, symMatrix b) {
  return symMatrix(a.xx + b.xx, a.yy + b.yy, a.zz + b.zz, a.xy + b.xy, a.xz + b.xz, a.yz + b.yz);
}
HOST_DEVICE inline symMatrix operator-(symMatrix a, symMatrix b) {
  return symMatrix(a.xx - b.xx, a.yy - b.yy, a.zz - b.zz, a.xy - b.xy, a.xz - b.xz, a.yz - b.yz);
}
HOST_DEVICE inline symMatrix operator*(symMatrix m, double a) {
  return symMatrix(m.xx * a, m.yy * a, m.zz * a, m.xy * a, m.xz * a, m.yz * a);
}
HOST_DEVICE inline symMatrix operator*(double a, symMatrix m) { return m * a; }
HOST_DEVICE inline double3 operator*(symMatrix m, double3 v) {
  return make_double3(m.xx * v.x + m.xy * v.y + m.xz * v.z, m.xy * v.x + m.yy * v.y + m.yz * v.z,
                      m.xz * v.x + m.yz * v.y + m.zz * v.z);
}
HOST_DEVICE inline double3 operator*(double3 v, symMatrix m) { return m * v; }

// R invI R^T with R the rotation matrix of q.
HOST_DEVICE inline symMatrix rotateInverseInertiaTensorByQuaternion(quaternion q, symMatrix I) {
  const double q0 = q.q0, q1 = q.q1, q2 = q.q2, q3 = q.q3;
  const double R[3][3] = {{1.0 - 2 * (q2 * q2 + q3 * q3), 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2)},
                          {2 * (q1 * q2 + q0 * q3), 1.0 - 2 * (q1 * q1 + q3 * q3), 2 * (q2 * q3 - q0 * q1)},
                          {2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), 1.0 - 2 * (q1 * q1 + q2 * q2)}};
  const double M[3][3] = {{I.xx, I.xy, I.xz}, {I.xy, I.yy, I.yz}, {I.xz, I.yz, I.zz}};
  double RM[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) RM[r][c] = R[r][0] * M[0][c] + R[r][1] * M[1][c] + R[r][2] * M[2][c];
  double W[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) W[r][c] = RM[r][0] * R[c][0] + RM[r][1] * R[c][1] + RM[r][2] * R[c][2];
  return symMatrix(W[0][0], W[1][1], W[2][2], W[0][1], W[0][2], W[1][2]);
}

// Inverse of a symmetric matrix; zero matrix when |det| < 1e-30.
HOST_DEVICE inline symMatrix inverse(symMatrix A) {
  const double c00 = A.yy * A.zz - A.yz * A.yz, c01 = A.xz * A.yz - A.xy * A.zz, c02 = A.xy * A.yz - A.xz * A.yy;
  const double det = A.xx * c00 + A.xy * c01 + A.xz * c02;
  if (fabs(det) < 1e-30) return symMatrix(0, 0, 0, 0, 0, 0);
  const double d = 1.0 / det;
  return symMatrix(c00 * d, (A.xx * A.zz - A.xz * A.xz) * d, (A.xx * A.yy - A.xy * A.xy) * d, c01 * d, c02 * d,
                   (A.xy * A.xz - A.xx * A.yz) * d);
}
