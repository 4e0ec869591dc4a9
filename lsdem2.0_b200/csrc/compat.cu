// The reference's separable extern "C" launchers, re-implemented on this library's
// kernels for host code written against the reference's internal launcher layer
// (declared in include/lsdem_compat.h with the reference's signatures):
//   launchUpdateSpatialGridHashStartEnd   (mySpatialGrid.h:33-49, buildHashStartEnd.cu:69-137):
//     cell keys, then the stable bucket sort of this library (sort_scan.cu), which leaves the
//     keys sorted in hashValue, the sorted object indices in hashIndex and the per-cell
//     [start, end) (-1 when empty) as thrust::sort_by_key + findStartAndEnd do;
//   launchParticleVelocityAngularVelocityIntegration / launchParticlePositionOrientationIntegration
//     (particleIntegrationKernel.cuh:4-30): velocity and angular velocity kick, position drift
//     and quaternion integration with the step length given (callers pass dt / 2 for a half kick);
//   launchUpdatePositionOutOfBoundaryXD / YD (mySpatialGrid.h:51-65): the periodic wrap.
// The reference's grid and block arguments are accepted and not used (each launch sizes its
// own grid). Errors surface, as in the reference, through cudaGetLastError.
#include <mutex>

#include "kernels.h"

namespace lsdem {
namespace {

__global__ void k_compat_keys(const double3* __restrict__ pos, int n, GridP g, int* __restrict__ key) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) key[i] = hash_key(pos[i], g);
}

__global__ void k_compat_kick(double3* __restrict__ vel, double3* __restrict__ angvel, const double3* __restrict__ force,
                              const double3* __restrict__ torque, const double* __restrict__ invm,
                              const Quat* __restrict__ quat, const Sym6* __restrict__ invI, double3 g, double h,
                              long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double im = invm[i];
  if (is_zero(im)) return;
  vel[i] += (force[i] * im + g) * h;
  angvel[i] += (mul(rotate_inv_inertia(quat[i], invI[i]), torque[i])) * h;
}

__global__ void k_compat_drift(double3* __restrict__ pos, Quat* __restrict__ quat, const double3* __restrict__ vel,
                               const double3* __restrict__ angvel, double dt, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  pos[i] += dt * vel[i];
  quat[i] = quat_integrate(quat[i], angvel[i], dt);
}

__global__ void k_compat_wrap(double3* __restrict__ pos, double3 mn, double3 mx, int axis, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double3 p = pos[i];
  double& c = axis == 0 ? p.x : p.y;
  const double lo = axis == 0 ? mn.x : mn.y, hi = axis == 0 ? mx.x : mx.y;
  if (c < lo) c += hi - lo;
  else if (c >= hi) c -= hi - lo;
  pos[i] = p;
}

// Scratch of the sort, per device, grown on demand (the reference's thrust sort
// allocates its temporary storage the same way).
struct SortScratch {
  int n = 0, cells = 0;
  int *key = nullptr, *counts = nullptr, *fill = nullptr, *offs = nullptr, *scan = nullptr, *big = nullptr,
      *bigc = nullptr, *tmp = nullptr;
};
std::mutex g_mu;
SortScratch g_s[64];

cudaError_t ensure(SortScratch& w, int n, int cells) {
  if (n <= w.n && cells <= w.cells) return cudaSuccess;
  int* ptrs[8] = {w.key, w.counts, w.fill, w.offs, w.scan, w.big, w.bigc, w.tmp};
  for (int* p : ptrs)
    if (p) cudaFree(p);
  w = SortScratch{};
  const int nb = cells + 3;
  cudaError_t e = cudaSuccess;
  auto take = [&](int*& p, size_t m) {
    if (e == cudaSuccess) e = cudaMalloc((void**)&p, sizeof(int) * (m > 0 ? m : 1));
  };
  take(w.key, n);
  take(w.counts, nb);
  take(w.fill, nb);
  take(w.offs, nb);
  take(w.scan, scan_temp_elems(nb));
  take(w.big, (size_t)n / 65 + 1);
  take(w.bigc, 2);
  take(w.tmp, n);
  if (e == cudaSuccess) {
    w.n = n;
    w.cells = cells;
  }
  return e;
}

}  // namespace
}  // namespace lsdem

using lsdem::Quat;
using lsdem::Sym6;

extern "C" {

void launchUpdateSpatialGridHashStartEnd(int* hashIndex, int* hashValue, const double3* position, int* gridHashStart,
                                         int* gridHashEnd, const double3 minBound, const double3 maxBound,
                                         const double3 inverseCellSize, const int3 gridSize3D, const size_t numGrid,
                                         const size_t numObject, const size_t, const size_t, cudaStream_t stream) {
  using namespace lsdem;
  if (numObject > 0x7fffffffu || numGrid > 0x7ffffff0u) return;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  const int n = (int)numObject, nc = (int)numGrid;
  GridP g;
  g.mn = minBound;
  g.mx = maxBound;
  g.inv = inverseCellSize;
  g.size = gridSize3D;
  g.ncells = nc;
  std::lock_guard<std::mutex> lk(g_mu);
  SortScratch& w = g_s[dev];
  if (ensure(w, n, nc) != cudaSuccess) return;  // cudaGetLastError reports the failed allocation
  if (n > 0) k_compat_keys<<<(n + 255) / 256, 256, 0, stream>>>(position, n, g, w.key);
  BucketScratch b{w.counts, w.fill, w.offs, w.scan, w.big, w.bigc, w.tmp};
  bucket_sort(w.key, n, nc, b, hashIndex, hashValue, gridHashStart, gridHashEnd, stream);
}

void launchParticleVelocityAngularVelocityIntegration(double3* velocity, double3* angularVelocity,
                                                      const double3* force, const double3* torque,
                                                      const double* invMass, const Quat* orientation,
                                                      const Sym6* inverseInertiaTensor, const double3 gravity,
                                                      const double timeStep, const size_t num, const size_t,
                                                      const size_t, cudaStream_t stream) {
  if (num == 0) return;
  lsdem::k_compat_kick<<<(unsigned)((num + 255) / 256), 256, 0, stream>>>(
      velocity, angularVelocity, force, torque, invMass, orientation, inverseInertiaTensor, gravity, timeStep,
      (long long)num);
}

void launchParticlePositionOrientationIntegration(double3* position, Quat* orientation, const double3* velocity,
                                                  const double3* angularVelocity, const double timeStep,
                                                  const size_t num, const size_t, const size_t, cudaStream_t stream) {
  if (num == 0) return;
  lsdem::k_compat_drift<<<(unsigned)((num + 255) / 256), 256, 0, stream>>>(position, orientation, velocity,
                                                                          angularVelocity, timeStep, (long long)num);
}

void launchUpdatePositionOutOfBoundaryXD(double3* position, const double3 minBound, const double3 maxBound,
                                         const size_t numObject, const size_t, const size_t, cudaStream_t stream) {
  if (numObject == 0) return;
  lsdem::k_compat_wrap<<<(unsigned)((numObject + 255) / 256), 256, 0, stream>>>(position, minBound, maxBound, 0,
                                                                               (long long)numObject);
}

void launchUpdatePositionOutOfBoundaryYD(double3* position, const double3 minBound, const double3 maxBound,
                                         const size_t numObject, const size_t, const size_t, cudaStream_t stream) {
  if (numObject == 0) return;
  lsdem::k_compat_wrap<<<(unsigned)((numObject + 255) / 256), 256, 0, stream>>>(position, minBound, maxBound, 1,
                                                                               (long long)numObject);
}

}  // extern "C"
