// App-facing vector math with the names and signatures the reference's apps
// and host helpers use (FunDEM/kernel/CUDAKernelFunction/myUtility/myVec.h),
// so that they compile unchanged against this library's headers. Semantics:
// device normalise uses rsqrt, host normalise 1/sqrt; |x| <= 1e-20 is zero.
#pragma once
#include <cuda_runtime.h>
#include <cmath>

#ifdef __CUDACC__
#define HOST_DEVICE __host__ __device__
#else
#define HOST_DEVICE
#endif

HOST_DEVICE constexpr double pi() { return 3.14159265358979323846; }
HOST_DEVICE inline bool isZero(const double x) { return fabs(x) <= 1.0e-20; }

HOST_DEVICE inline double3 operator+(double3 a, double3 b) { return make_double3(a.x + b.x, a.y + b.y, a.z + b.z); }
HOST_DEVICE inline double3 operator-(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
HOST_DEVICE inline double3 operator*(double3 a, double s) { return make_double3(a.x * s, a.y * s, a.z * s); }
HOST_DEVICE inline double3 operator*(double s, double3 a) { return make_double3(a.x * s, a.y * s, a.z * s); }
HOST_DEVICE inline double3 operator/(double3 a, double s) {
  const double inv = 1.0 / s;
  return make_double3(a.x * inv, a.y * inv, a.z * inv);
}
HOST_DEVICE inline double3& operator+=(double3& a, double3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
HOST_DEVICE inline double3& operator-=(double3& a, double3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
HOST_DEVICE inline double3& operator*=(double3& a, double s) { a.x *= s; a.y *= s; a.z *= s; return a; }
HOST_DEVICE inline double3& operator/=(double3& a, double s) {
  const double inv = 1.0 / s;
  a.x *= inv; a.y *= inv; a.z *= inv;
  return a;
}
HOST_DEVICE inline double3 operator-(double3 a) { return make_double3(-a.x, -a.y, -a.z); }

HOST_DEVICE inline double dot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
HOST_DEVICE inline double3 cross(double3 a, double3 b) {
  return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
HOST_DEVICE inline double lengthSquared(double3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
HOST_DEVICE inline double length(double3 v) { return sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
HOST_DEVICE inline double3 normalize(double3 v) {
  const double l2 = v.x * v.x + v.y * v.y + v.z * v.z;
  if (isZero(l2)) return make_double3(0.0, 0.0, 0.0);
#ifdef __CUDA_ARCH__
  const double inv = rsqrt(l2);
#else
  const double inv = 1.0 / sqrt(l2);
#endif
  return make_double3(v.x * inv, v.y * inv, v.z * inv);
}

// exp([omega]x) v (Rodrigues), with a second-order expansion for tiny angles.
HOST_DEVICE inline double3 rotateVector(const double3 v, const double3 omega) {
  const double t2 = dot(omega, omega);
  const double3 oxv = cross(omega, v);
  const double3 oxoxv = cross(omega, oxv);
  if (isZero(t2)) return v + oxv + 0.5 * oxoxv;
  const double t = sqrt(t2);
  const double A = sin(t) / t;
  const double B = (1.0 - cos(t)) / t2;
  return v + A * oxv + B * oxoxv;
}

// Rotation about `axis` by the angle whose sine is sinTheta (cos >= 0 assumed).
HOST_DEVICE inline double3 rotateVectorAxisSin(const double3 v, const double3 axis, const double sinTheta) {
  const double a2 = dot(axis, axis);
  if (isZero(a2)) return v;
  const double3 k = axis * (1.0 / sqrt(a2));
  const double c = sqrt(fmax(0.0, 1.0 - sinTheta * sinTheta));
  return v * c + cross(k, v) * sinTheta + k * (dot(k, v) * (1.0 - c));
}

// Packed upper-triangular index of the unordered pair (row, col) of n items,
// capacity - 1 for out-of-range input.
HOST_DEVICE inline int upperTriangularIndex(int row, int col, int n, int capacity) {
  if (n <= 0 || capacity <= 0) return 0;
  if (row < 0 || col < 0 || row >= n || col >= n) return capacity - 1;
  const long long i = row < col ? row : col, j = row < col ? col : row;
  long long idx = i * (2LL * n - i + 1LL) / 2LL + (j - i);
  if (idx < 0) idx = 0;
  if (idx >= capacity) idx = capacity - 1;
  return (int)idx;
}

HOST_DEVICE inline int linearIndex3D(const int3 ijk, const int3 dims) { return ijk.z * dims.y * dims.x + ijk.y * dims.x + ijk.x; }
