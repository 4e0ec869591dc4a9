// Mass properties of a level-set body on the GPU: the smoothed-Heaviside integrals of
// LSSolver::addLSParticle (LSSolver.h:66-135) — mass, centroid, inertia about the
// centroid and its inverse — as parallel sums over the grid nodes. Pass 1 sums H, H x,
// H y, H z (mass and the centroid's moments), pass 2 the six second moments about the
// centroid; each block reduces its nodes in a fixed tree, the block partials are summed
// on the host in block order, so a result is reproducible run to run. The sums are
// ordered differently from the host routine's triple loop: the results agree with it to
// rounding (relative 1e-12 in the tests), not bit for bit.
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/lsdem_b200.h"
#include "kernels.h"

namespace lsdem {
namespace {

constexpr int MP_THREADS = 256;

// Smoothed Heaviside of phi / h with half width 1.5 (LSSolver.h:66-80): 1 inside, 0 outside.
__device__ __forceinline__ double heaviside(double phi, double eps) {
  if (phi < -eps) return 1.0;
  if (phi > eps) return 0.0;
  const double x = -phi / eps;
  return 0.5 * (1.0 + x + sin(M_PI * x) / M_PI);
}

template <int K>
__device__ void block_sum(double (&v)[K], double* sm, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) sm[warp * K + k] = v[k];
  __syncthreads();
  if (threadIdx.x < K) {
    double s = 0.0;
    for (int w = 0; w < MP_THREADS / 32; ++w) s += sm[w * K + threadIdx.x];
    out[blockIdx.x * K + threadIdx.x] = s;
  }
}

__global__ void __launch_bounds__(MP_THREADS) k_mass_moments(const double* __restrict__ sdf, int3 n, double3 o,
                                                            double h, double* __restrict__ part) {
  __shared__ double sm[(MP_THREADS / 32) * 4];
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  const long long total = (long long)n.x * n.y * n.z;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % n.x), y = (int)((i / n.x) % n.y), z = (int)(i / ((long long)n.x * n.y));
    const double H = heaviside(sdf[i] / h, 1.5);
    v[0] += H;
    v[1] += H * (o.x + double(x) * h);
    v[2] += H * (o.y + double(y) * h);
    v[3] += H * (o.z + double(z) * h);
  }
  block_sum<4>(v, sm, part);
}

__global__ void __launch_bounds__(MP_THREADS) k_inertia_moments(const double* __restrict__ sdf, int3 n, double3 o,
                                                               double h, double3 c, double* __restrict__ part) {
  __shared__ double sm[(MP_THREADS / 32) * 6];
  double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const long long total = (long long)n.x * n.y * n.z;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % n.x), y = (int)((i / n.x) % n.y), z = (int)(i / ((long long)n.x * n.y));
    const double H = heaviside(sdf[i] / h, 1.5);
    const double rx = o.x + h * double(x) - c.x, ry = o.y + h * double(y) - c.y, rz = o.z + h * double(z) - c.z;
    v[0] += H * (ry * ry + rz * rz);
    v[1] += H * (rx * rx + rz * rz);
    v[2] += H * (ry * ry + rx * rx);
    v[3] -= H * rx * ry;
    v[4] -= H * rx * rz;
    v[5] -= H * ry * rz;
  }
  block_sum<6>(v, sm, part);
}

}  // namespace
}  // namespace lsdem

extern "C" int lsdem_mass_properties_gpu(const double* sdf, const int* size3, const double* origin3, double spacing,
                                         double density, double* out16, int device) {
  using namespace lsdem;
  if (!sdf || !size3 || !origin3 || !out16 || !(spacing > 0.0)) return LSDEM_ERR_ARG;
  if (size3[0] < 1 || size3[1] < 1 || size3[2] < 1) return LSDEM_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return LSDEM_ERR_NODEVICE;
  if (device < 0 || device >= ndev) return LSDEM_ERR_ARG;
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return LSDEM_ERR_NODEVICE;
  const size_t total = (size_t)size3[0] * size3[1] * size3[2];
  const int blocks = (int)std::min<size_t>((total + MP_THREADS - 1) / MP_THREADS, 148 * 4);
  double *d_sdf = nullptr, *d_part = nullptr;
  int rc = LSDEM_OK;
  std::vector<double> part((size_t)blocks * 6);
  const int3 n = make_int3(size3[0], size3[1], size3[2]);
  const double3 o = make_double3(origin3[0], origin3[1], origin3[2]);
  const double h = spacing;
  double mass = 0.0, c[3] = {0.0, 0.0, 0.0}, I[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const double mg = density * h * h * h;
  do {
    if (cudaMalloc((void**)&d_sdf, total * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&d_part, part.size() * sizeof(double)) != cudaSuccess) {
      rc = LSDEM_ERR_NOMEM;
      break;
    }
    if (cudaMemcpy(d_sdf, sdf, total * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) { rc = LSDEM_ERR_CUDA; break; }
    k_mass_moments<<<blocks, MP_THREADS>>>(d_sdf, n, o, h, d_part);
    if (cudaMemcpy(part.data(), d_part, (size_t)blocks * 4 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
      rc = LSDEM_ERR_CUDA;
      break;
    }
    double m[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = 0; b < blocks; ++b)
      for (int k = 0; k < 4; ++k) m[k] += part[(size_t)b * 4 + k];
    mass = m[0] * mg;
    if (!(mass > 0.0)) break;
    for (int a = 0; a < 3; ++a) c[a] = m[1 + a] * (mg / mass);
    k_inertia_moments<<<blocks, MP_THREADS>>>(d_sdf, n, o, h, make_double3(c[0], c[1], c[2]), d_part);
    if (cudaMemcpy(part.data(), d_part, (size_t)blocks * 6 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
      rc = LSDEM_ERR_CUDA;
      break;
    }
    for (int b = 0; b < blocks; ++b)
      for (int k = 0; k < 6; ++k) I[k] += part[(size_t)b * 6 + k];
    for (int k = 0; k < 6; ++k) I[k] *= mg;
  } while (false);
  if (d_sdf) cudaFree(d_sdf);
  if (d_part) cudaFree(d_part);
  cudaSetDevice(prev);
  if (rc != LSDEM_OK) return rc;
  // inverse of the symmetric inertia (myMat.h:163-195), zero when singular
  double inv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (mass > 0.0) {
    const double xx = I[0], yy = I[1], zz = I[2], xy = I[3], xz = I[4], yz = I[5];
    const double det = xx * (yy * zz - yz * yz) + xy * (yz * xz - xy * zz) + xz * (xy * yz - yy * xz);
    if (!(std::fabs(det) < 1e-30)) {
      const double di = 1.0 / det;
      inv[0] = (yy * zz - yz * yz) * di;
      inv[1] = (xx * zz - xz * xz) * di;
      inv[2] = (xx * yy - xy * xy) * di;
      inv[3] = -(xy * zz - xz * yz) * di;
      inv[4] = (xy * yz - xz * yy) * di;
      inv[5] = -(xx * yz - xz * xy) * di;
    }
  }
  out16[0] = mass;
  for (int a = 0; a < 3; ++a) out16[1 + a] = c[a];
  for (int a = 0; a < 6; ++a) out16[4 + a] = I[a];
  for (int a = 0; a < 6; ++a) out16[10 + a] = inv[a];
  return LSDEM_OK;
}
