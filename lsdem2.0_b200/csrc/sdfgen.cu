// Level-set grid of a closed triangle mesh, computed on the device.
//
// Per grid node this is the work of LevelSetObject::Base::buildGrid
// (FunDEM/kernel/helper/LevelSetObjectGenerator.h:122-224) over
// TriangleMeshParticle::evaluateImplicitFunctionValueAndGradient (:888-914):
//   * the closest point of the mesh: per triangle, the Voronoi-region tests of
//     C. Ericson, "Real-Time Collision Detection" (2005), section 5.1.5 — the
//     reference's closestPointOnTriangle (:454-500); the nearest over all
//     triangles (the reference's BVH prunes only boxes farther than the best
//     so far, so it finds the same distance);
//   * inside or outside: the sum of the signed solid angles of all triangles
//     seen from the node, A. Van Oosterom and J. Strackee, IEEE Trans. Biomed.
//     Eng. 30 (1983) 125-126 (the reference's solidAngleFromPointToTriangle and
//     isPointInsideClosedTriangleMesh, :758-802), summed in triangle order;
//   * value = -+d, gradient -+(p - cp)/d, optionally negated (level set positive
//     inside), then buildGrid's value / |gradient|, or -+h/2 where |gradient|
//     <= 1e-12.
//
// One thread per grid node; the mesh streams through shared memory in tiles of
// kTile triangles, so every node sees every triangle once (brute force, no
// tree: a 64^3 grid against 2e4 triangles is a few 1e9 node-triangle pairs).
// The file is compiled with --fmad=false so that products and sums round as the
// reference's host arithmetic does; distances are then bit-identical to the
// host computation and only the solid-angle sum can differ in its last bits
// (atan2), which moves the inside decision only for nodes on the surface.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../include/lsdem_b200.h"
#include "common.cuh"

namespace lsdem {
namespace {

constexpr int kTile = 128;
constexpr int kThreads = 128;

LD double3 closest_on_triangle(double3 p, double3 a, double3 b, double3 c) {
  const double3 ab = b - a;
  const double3 ac = c - a;
  const double3 ap = p - a;
  const double d1 = dot(ab, ap);
  const double d2 = dot(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) return a;
  const double3 bp = p - b;
  const double d3v = dot(ab, bp);
  const double d4 = dot(ac, bp);
  if (d3v >= 0.0 && d4 <= d3v) return b;
  const double vc = d1 * d4 - d3v * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3v <= 0.0) return a + (d1 / (d1 - d3v)) * ab;
  const double3 cp = p - c;
  const double d5 = dot(ab, cp);
  const double d6 = dot(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return c;
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return a + (d2 / (d2 - d6)) * ac;
  const double va = d3v * d6 - d5 * d4;
  if (va <= 0.0 && (d4 - d3v) >= 0.0 && (d5 - d6) >= 0.0) {
    const double3 bc = c - b;
    return b + ((d4 - d3v) / ((d4 - d3v) + (d5 - d6))) * bc;
  }
  const double denom = 1.0 / (va + vb + vc);
  const double v = vb * denom;
  const double w = vc * denom;
  return a + ab * v + ac * w;
}

LD double solid_angle(double3 p, double3 a, double3 b, double3 c) {
  const double3 r0 = a - p;
  const double3 r1 = b - p;
  const double3 r2 = c - p;
  const double l0 = len(r0);
  const double l1 = len(r1);
  const double l2 = len(r2);
  if (l0 < 1e-30 || l1 < 1e-30 || l2 < 1e-30) return 0.0;
  const double num = dot(r0, cross(r1, r2));
  const double den = l0 * l1 * l2 + dot(r0, r1) * l2 + dot(r1, r2) * l0 + dot(r2, r0) * l1;
  return 2.0 * atan2(num, den);
}

// tri: 9 doubles per triangle (vertex a, b, c).
__global__ void __launch_bounds__(kThreads) k_mesh_grid(const double* __restrict__ tri, int nt, double3 origin,
                                                        int nx, int ny, int nz, double h, int positive_inside,
                                                        double* __restrict__ out) {
  __shared__ double s_tri[kTile * 9];
  const long long n = (long long)nx * ny * nz;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i < n;
  const long long ii = active ? i : 0;
  const int ix = (int)(ii % nx);
  const int iy = (int)((ii / nx) % ny);
  const int iz = (int)(ii / ((long long)nx * ny));
  const double3 p = d3(origin.x + double(ix) * h, origin.y + double(iy) * h, origin.z + double(iz) * h);
  double best = 1.7976931348623157e308;
  double3 cp = d3(0., 0., 0.);
  double sum = 0.0;
  for (int t0 = 0; t0 < nt; t0 += kTile) {
    const int m = min(kTile, nt - t0);
    __syncthreads();
    for (int k = threadIdx.x; k < m * 9; k += blockDim.x) s_tri[k] = tri[(long long)t0 * 9 + k];
    __syncthreads();
    for (int k = 0; k < m; ++k) {
      const double* q = s_tri + 9 * k;
      const double3 a = d3(q[0], q[1], q[2]);
      const double3 b = d3(q[3], q[4], q[5]);
      const double3 c = d3(q[6], q[7], q[8]);
      const double3 x = closest_on_triangle(p, a, b, c);
      const double d2 = len2(p - x);
      if (d2 < best) {
        best = d2;
        cp = x;
      }
      sum += solid_angle(p, a, b, c);
    }
  }
  if (!active) return;
  const double d = len(p - cp);
  const bool inside = fabs(sum / (4.0 * 3.14159265358979323846)) > 0.5;
  double value = inside ? -d : d;
  double3 g = d3(0., 0., 0.);
  if (d > 1e-30) {
    const double3 u = (p - cp) / d;
    g = inside ? -u : u;
  }
  if (positive_inside) {
    value = -value;
    g = -g;
  }
  const double gn = len(g);
  out[i] = gn > 1e-12 ? value / gn : (value <= 0.0 ? -1.0 : 1.0) * 0.5 * h;
}

bool mesh_valid(int nv, const int* tris, int nt) {
  if (nv <= 0 || nt <= 0) return false;
  for (int t = 0; t < nt; ++t) {
    const int a = tris[3 * t], b = tris[3 * t + 1], c = tris[3 * t + 2];
    if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv) return false;
    if (a == b || b == c || c == a) return false;
  }
  return true;
}

}  // namespace
}  // namespace lsdem

extern "C" int lsdem_mesh_grid_box(const double* verts, int n_verts, double spacing, int pad, double* origin3,
                                   int* size3) {
  if (!verts || n_verts <= 0 || !(spacing > 0.0) || !origin3 || !size3) return LSDEM_ERR_ARG;
  double mn[3] = {verts[0], verts[1], verts[2]}, mx[3] = {verts[0], verts[1], verts[2]};
  for (int v = 1; v < n_verts; ++v)
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::min(mn[a], verts[3 * v + a]);
      mx[a] = std::max(mx[a], verts[3 * v + a]);
    }
  const double padding = double(std::max(1, pad)) * spacing;
  for (int a = 0; a < 3; ++a) {
    const double lo = spacing * std::floor((mn[a] - padding) / spacing);
    const double hi = spacing * std::ceil((mx[a] + padding) / spacing);
    const int n = int(std::floor((hi - lo) / spacing + 0.5)) + 1;
    if (n <= 0) return LSDEM_ERR_ARG;
    origin3[a] = lo;
    size3[a] = n;
  }
  return LSDEM_OK;
}

extern "C" int lsdem_mesh_grid(const double* verts, int n_verts, const int* tris, int n_tris, const double* origin3,
                               const int* size3, double spacing, int positive_inside, double* sdf_out, int device) {
  using namespace lsdem;
  if (!verts || !tris || !origin3 || !size3 || !sdf_out || !(spacing > 0.0)) return LSDEM_ERR_ARG;
  if (size3[0] <= 0 || size3[1] <= 0 || size3[2] <= 0) return LSDEM_ERR_ARG;
  if (!mesh_valid(n_verts, tris, n_tris)) return LSDEM_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return LSDEM_ERR_NODEVICE;
  if (device < 0 || device >= ndev) return LSDEM_ERR_ARG;
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return LSDEM_ERR_CUDA;
  std::vector<double> tv((size_t)n_tris * 9);
  for (int t = 0; t < n_tris; ++t)
    for (int k = 0; k < 3; ++k)
      for (int a = 0; a < 3; ++a) tv[9 * (size_t)t + 3 * k + a] = verts[3 * (size_t)tris[3 * t + k] + a];
  const long long n = (long long)size3[0] * size3[1] * size3[2];
  double* d_tri = nullptr;
  double* d_out = nullptr;
  int rc = LSDEM_OK;
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) rc = LSDEM_ERR_CUDA;
  if (rc == LSDEM_OK && (cudaMalloc(&d_tri, tv.size() * sizeof(double)) != cudaSuccess ||
                         cudaMalloc(&d_out, (size_t)n * sizeof(double)) != cudaSuccess))
    rc = LSDEM_ERR_NOMEM;
  if (rc == LSDEM_OK) {
    cudaMemcpyAsync(d_tri, tv.data(), tv.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    const long long blocks = (n + kThreads - 1) / kThreads;
    k_mesh_grid<<<(unsigned)blocks, kThreads, 0, st>>>(d_tri, n_tris, d3(origin3[0], origin3[1], origin3[2]), size3[0],
                                                       size3[1], size3[2], spacing, positive_inside, d_out);
    cudaMemcpyAsync(sdf_out, d_out, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = LSDEM_ERR_CUDA;
  }
  if (d_tri) cudaFree(d_tri);
  if (d_out) cudaFree(d_out);
  if (st) cudaStreamDestroy(st);
  cudaSetDevice(prev);
  return rc;
}
