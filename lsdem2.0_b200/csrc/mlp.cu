// Learned per-shape SDF: training data, forward/backward/Adam training kernels,
// inference tables and the validation pass that measures each network's error
// (with the tensor-core inference code of mlp.cuh, the code the narrowphase uses).
//
// Training data of shape s: points of the template's grid box, half uniform and
// half near the surface (a surface node moved by a normal-distributed offset of
// two grid spacings per axis), with targets from the FP64 trilinear grid
// interpolation (the reference's SDF semantics, LSParticleContactDetectionKernel.cuh:4-32).
// The loss is the mean squared error of phi / R. One launch of k_mlp_grad per
// iteration computes block-partial gradients of all shapes (grid.y = shape);
// k_mlp_adam sums them and applies Adam to the FP32 master weights.
#include <cstdint>

#include "kernels.h"
#include "mlp.cuh"

namespace lsdem {

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // SplitMix64 finaliser
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double unit01(uint64_t z) { return (double)(mix64(z) >> 11) * (1.0 / 9007199254740992.0); }

// FP64 trilinear interpolation of a template grid at template-frame point p
// (clamped into the grid box).
__device__ double grid_phi(const double* sdf, int3 gs, double3 o, double h, double3 p) {
  double g[3] = {(p.x - o.x) / h, (p.y - o.y) / h, (p.z - o.z) / h};
  const int n[3] = {gs.x, gs.y, gs.z};
  int i[3];
  double f[3];
  for (int a = 0; a < 3; ++a) {
    g[a] = fmin(fmax(g[a], 0.0), (double)(n[a] - 1) * (1.0 - 1e-12));
    i[a] = min((int)floor(g[a]), n[a] - 2);
    f[a] = g[a] - i[a];
  }
  const double* b = sdf + ((size_t)i[2] * gs.y + i[1]) * gs.x + i[0];
  const size_t sy = gs.x, sz = (size_t)gs.x * gs.y;
  const double c00 = b[0] * (1 - f[0]) + b[1] * f[0], c10 = b[sy] * (1 - f[0]) + b[sy + 1] * f[0];
  const double c01 = b[sz] * (1 - f[0]) + b[sz + 1] * f[0], c11 = b[sz + sy] * (1 - f[0]) + b[sz + sy + 1] * f[0];
  const double c0 = c00 * (1 - f[1]) + c10 * f[1], c1 = c01 * (1 - f[1]) + c11 * f[1];
  return c0 * (1 - f[2]) + c1 * f[2];
}

__device__ __forceinline__ float silu_f(float x) { return x / (1.f + __expf(-x)); }
__device__ __forceinline__ float dsilu_f(float x) {
  const float s = 1.f / (1.f + __expf(-x));
  return s * (1.f + x * (1.f - s));
}

}  // namespace

// Samples of all shapes: samples[s * S + k] = (u.x, u.y, u.z, phi / R clipped to
// [opt.clip_lo, opt.clip_hi]); a share opt.near of them near the surface.
__global__ void k_mlp_samples(MlpShapeData D, int S, unsigned long long seed, MlpTrainOpts opt, float4* samples) {
  const int s = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= S) return;
  const MlpNorm nm = D.norm[s];
  const int3 gs = D.gsize[s];
  const double3 o = D.origin[s];
  const double h = D.h[s];
  const double3 hi = make_double3(o.x + (gs.x - 1) * h, o.y + (gs.y - 1) * h, o.z + (gs.z - 1) * h);
  const uint64_t base = seed ^ ((uint64_t)s << 40) ^ ((uint64_t)k << 2);
  double3 p;
  if (unit01(base ^ 0x5851f42d4c957f2dull) >= (double)opt.near || D.node_cnt[s] == 0) {  // uniform in the box
    p = make_double3(o.x + (hi.x - o.x) * unit01(base), o.y + (hi.y - o.y) * unit01(base + 1),
                     o.z + (hi.z - o.z) * unit01(base + 2));
  } else {             // near the surface: a node plus N(0, (2h)^2) per axis (Box-Muller)
    const int nn = D.node_cnt[s];
    const int ni = (int)(unit01(base) * nn) % nn;
    const double3 q = D.node_pos[D.node_off[s] + ni];
    const double r1 = sqrt(-2.0 * log(fmax(unit01(base + 1), 1e-300))), t1 = 6.283185307179586 * unit01(base + 2);
    const double r2 = sqrt(-2.0 * log(fmax(unit01(base + 3), 1e-300)));
    p = make_double3(q.x + 2 * h * r1 * cos(t1), q.y + 2 * h * r1 * sin(t1), q.z + 2 * h * r2 * cos(t1 + 1.0));
    p.x = fmin(fmax(p.x, o.x), hi.x);
    p.y = fmin(fmax(p.y, o.y), hi.y);
    p.z = fmin(fmax(p.z, o.z), hi.z);
  }
  const double phi = grid_phi(D.sdf + D.sdf_off[s], gs, o, h, p);
  samples[(size_t)s * S + k] = make_float4((float)((p.x - nm.cx) / nm.R), (float)((p.y - nm.cy) / nm.R),
                                           (float)((p.z - nm.cz) / nm.R),
                                           (float)fmin(fmax(phi / nm.R, (double)opt.clip_lo), (double)opt.clip_hi));
}

// Block-partial gradients of the mean squared error over points of the batch:
// block b of shape s takes points (it * B + b * 128 + t) mod S, 128 per block.
// partial[(s * nblk + b) * MLP_NP + param]; loss[s * nblk + b] = sum of squared errors.
static constexpr int MLP_T = 128;
static constexpr int MLP_LD = 65;  // padded row of the activation tiles
__global__ void __launch_bounds__(MLP_T) k_mlp_grad(const float* __restrict__ params, const float4* __restrict__ samples,
                                                    int S, int B, long long it, int nblk, float* __restrict__ partial,
                                                    float* __restrict__ loss) {
  extern __shared__ float sm[];
  float* W = sm;                         // MLP_NP
  float* A1 = W + MLP_NP;                // [128][65] layer-1 activations, later dL/dh1
  float* H2 = A1 + MLP_T * MLP_LD;       // [128][65] layer-2 pre-activations, later dL/dh2
  float* A2 = H2 + MLP_T * MLP_LD;       // [128][65] layer-2 activations
  float* U = A2 + MLP_T * MLP_LD;        // [128][4] inputs
  float* DY = U + MLP_T * 4;             // [128]
  float* RED = DY + MLP_T;               // [128] reduction scratch
  const int s = blockIdx.y, t = threadIdx.x;
  const float* P = params + (size_t)s * MLP_NP;
  for (int k = t; k < MLP_NP; k += MLP_T) W[k] = P[k];
  const long long idx = ((long long)it * B + (long long)blockIdx.x * MLP_T + t) % S;
  const float4 smp = samples[(size_t)s * S + idx];
  U[t * 4 + 0] = smp.x; U[t * 4 + 1] = smp.y; U[t * 4 + 2] = smp.z;
  __syncthreads();
  // forward
  float* a1 = A1 + t * MLP_LD;
  float* h2 = H2 + t * MLP_LD;
  float* a2 = A2 + t * MLP_LD;
  for (int j = 0; j < 64; ++j) {
    const float h = W[MLP_B1 + j] + W[MLP_W1 + 3 * j] * smp.x + W[MLP_W1 + 3 * j + 1] * smp.y + W[MLP_W1 + 3 * j + 2] * smp.z;
    a1[j] = silu_f(h);
  }
  float y = W[MLP_B3];
  for (int j = 0; j < 64; ++j) {
    float h = W[MLP_B2 + j];
    const float* w = W + MLP_W2 + 64 * j;
    for (int i = 0; i < 64; ++i) h = fmaf(w[i], a1[i], h);
    h2[j] = h;
    const float a = silu_f(h);
    a2[j] = a;
    y = fmaf(W[MLP_W3 + j], a, y);
  }
  const float r = y - smp.w;
  const float dy = 2.f * r / (float)B;
  DY[t] = dy;
  RED[t] = r * r;
  for (int j = 0; j < 64; ++j) h2[j] = dy * W[MLP_W3 + j] * dsilu_f(h2[j]);  // dL/dh2
  __syncthreads();
  float* out = partial + ((size_t)s * nblk + blockIdx.x) * MLP_NP;
  // dW2[j][i] = sum_p dh2[p][j] a1[p][i]
  for (int e = t; e < 4096; e += MLP_T) {
    const int j = e >> 6, i = e & 63;
    float g = 0.f;
    for (int p = 0; p < MLP_T; ++p) g = fmaf(H2[p * MLP_LD + j], A1[p * MLP_LD + i], g);
    out[MLP_W2 + e] = g;
  }
  if (t < 64) {
    float g = 0.f;
    for (int p = 0; p < MLP_T; ++p) g += H2[p * MLP_LD + t];
    out[MLP_B2 + t] = g;
  } else {
    const int j = t - 64;
    float g = 0.f;
    for (int p = 0; p < MLP_T; ++p) g = fmaf(DY[p], A2[p * MLP_LD + j], g);
    out[MLP_W3 + j] = g;
  }
  if (t == 0) {
    float g = 0.f, l = 0.f;
    for (int p = 0; p < MLP_T; ++p) { g += DY[p]; l += RED[p]; }
    out[MLP_B3] = g;
    loss[s * nblk + blockIdx.x] = l;
  }
  __syncthreads();
  // dL/dh1 = (W2^T dh2) * silu'(h1), into A1
  for (int i = 0; i < 64; ++i) {
    float da = 0.f;
    for (int j = 0; j < 64; ++j) da = fmaf(W[MLP_W2 + 64 * j + i], h2[j], da);
    const float h = W[MLP_B1 + i] + W[MLP_W1 + 3 * i] * smp.x + W[MLP_W1 + 3 * i + 1] * smp.y + W[MLP_W1 + 3 * i + 2] * smp.z;
    a1[i] = da * dsilu_f(h);
  }
  __syncthreads();
  for (int e = t; e < 256; e += MLP_T) {
    float g = 0.f;
    if (e < 192) {
      const int j = e / 3, k = e % 3;
      for (int p = 0; p < MLP_T; ++p) g = fmaf(A1[p * MLP_LD + j], U[p * 4 + k], g);
      out[MLP_W1 + e] = g;
    } else {
      const int j = e - 192;
      for (int p = 0; p < MLP_T; ++p) g += A1[p * MLP_LD + j];
      out[MLP_B1 + j] = g;
    }
  }
}

size_t mlp_grad_smem() { return sizeof(float) * (MLP_NP + 3 * MLP_T * MLP_LD + MLP_T * 4 + 2 * MLP_T); }

// Sums the block partials and applies Adam (bias-corrected) to the FP32 weights.
__global__ void k_mlp_adam(float* params, float* m1, float* m2, const float* __restrict__ partial, int nblk,
                           float lr, float b1, float b2, float eps, int step) {
  const int s = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > MLP_B3) return;
  const size_t at = (size_t)s * MLP_NP + k;
  float g = 0.f;
  for (int b = 0; b < nblk; ++b) g += partial[((size_t)s * nblk + b) * MLP_NP + k];
  const float m = b1 * m1[at] + (1.f - b1) * g;
  const float v = b2 * m2[at] + (1.f - b2) * g * g;
  m1[at] = m;
  m2[at] = v;
  const float mh = m / (1.f - powf(b1, (float)step)), vh = v / (1.f - powf(b2, (float)step));
  params[at] -= lr * mh / (sqrtf(vh) + eps);
}

// Inference tables from the FP32 weights (one block per shape): W2 in BF16 in the
// swizzled B-operand layout, layer-1 rows with their bias, b2, w3, b3.
__global__ void k_mlp_pack(const float* __restrict__ params, MlpInfer* out) {
  const int s = blockIdx.x;
  const float* P = params + (size_t)s * MLP_NP;
  MlpInfer& M = out[s];
  for (int k = threadIdx.x; k < 512; k += blockDim.x) {
    const int n = k >> 3, c = k & 7;  // output unit n, inputs 8c .. 8c + 7
    const float* w = P + MLP_W2 + 64 * n + 8 * c;
    M.w2[n * 8 + (c ^ (n & 7))] = make_uint4(pack_bf16x2(w[0], w[1]), pack_bf16x2(w[2], w[3]),
                                             pack_bf16x2(w[4], w[5]), pack_bf16x2(w[6], w[7]));
  }
  for (int k = threadIdx.x; k < 64; k += blockDim.x) {
    M.w1[k] = make_float4(P[MLP_W1 + 3 * k], P[MLP_W1 + 3 * k + 1], P[MLP_W1 + 3 * k + 2], P[MLP_B1 + k]);
    M.b2[k] = P[MLP_B2 + k];
    M.w3[k] = P[MLP_W3 + k];
  }
  if (threadIdx.x == 0) {
    M.b3 = P[MLP_B3];
    M.pad[0] = M.pad[1] = M.pad[2] = 0.f;
  }
}

// Error of each shape's network, with the inference code of the narrowphase,
// over validation points: every grid node of the box, then S2 further points
// drawn like the training data with another seed (template units).
// err_bits[2 s]: largest |phi_net - clip(phi_grid)|; err_bits[2 s + 1]: largest
// phi_net - clip(phi_grid) over the points with phi_grid <= delta[s] (the one-sided
// bound that makes a rejection by the network safe; clip as the training target, in
// units of R). Float bits of running maxima of non-negative values (which order as
// integers).
__global__ void __launch_bounds__(MLP_TILE) k_mlp_validate(MlpShapeData D, const MlpInfer* __restrict__ inf, int S2,
                                                           unsigned long long seed, MlpTrainOpts opt,
                                                           const float* __restrict__ delta, unsigned* err_bits,
                                                           int* fail) {
  extern __shared__ unsigned char dyn[];
  MlpTcSmem* T = mlp_tc_smem(dyn);
  mlp_tc_setup(T);
  const int s = blockIdx.y;
  mlp_tc_stage(T, inf[s], s);
  const MlpNorm nm = D.norm[s];
  const int3 gs = D.gsize[s];
  const double3 o = D.origin[s];
  const double h = D.h[s];
  const long long ngrid = (long long)gs.x * gs.y * gs.z;
  const long long total = ngrid + S2;
  const float dlt = delta[s];
  float emax = 0.f, ein = 0.f;
  bool ok = true;
  for (long long k0 = (long long)blockIdx.x * MLP_TILE; k0 < total && ok; k0 += (long long)gridDim.x * MLP_TILE) {
    const long long k = k0 + threadIdx.x;
    double3 p = o;
    double phi = 0.0;
    const bool act = k < total;
    if (act && k < ngrid) {
      const int ix = (int)(k % gs.x), iy = (int)((k / gs.x) % gs.y), iz = (int)(k / ((long long)gs.x * gs.y));
      p = make_double3(o.x + ix * h, o.y + iy * h, o.z + iz * h);
      phi = D.sdf[D.sdf_off[s] + k];
    } else if (act && D.node_cnt[s] > 0) {
      const uint64_t base = seed ^ ((uint64_t)s << 40) ^ ((uint64_t)(k - ngrid) << 2);
      const int nn = D.node_cnt[s];
      const double3 q = D.node_pos[D.node_off[s] + (int)(unit01(base) * nn) % nn];
      const double r1 = sqrt(-2.0 * log(fmax(unit01(base + 1), 1e-300))), t1 = 6.283185307179586 * unit01(base + 2);
      const double r2 = sqrt(-2.0 * log(fmax(unit01(base + 3), 1e-300)));
      const double3 hi = make_double3(o.x + (gs.x - 1) * h, o.y + (gs.y - 1) * h, o.z + (gs.z - 1) * h);
      p = make_double3(fmin(fmax(q.x + 2 * h * r1 * cos(t1), o.x), hi.x), fmin(fmax(q.y + 2 * h * r1 * sin(t1), o.y), hi.y),
                       fmin(fmax(q.z + 2 * h * r2 * cos(t1 + 1.0), o.z), hi.z));
      phi = grid_phi(D.sdf + D.sdf_off[s], gs, o, h, p);
    } else if (act) {
      phi = D.sdf[D.sdf_off[s]];  // no nodes: the grid's first node again
    }
    mlp_tc_layer1(T, (float)((p.x - nm.cx) / nm.R), (float)((p.y - nm.cy) / nm.R), (float)((p.z - nm.cz) / nm.R));
    ok = mlp_tc_mma(T);
    const float net = mlp_tc_output(T) * nm.R;
    if (act && ok) {
      const float tgt = (float)fmin(fmax(phi, (double)(opt.clip_lo * nm.R)), (double)(opt.clip_hi * nm.R));
      emax = fmaxf(emax, fabsf(net - tgt));
      if (phi <= (double)dlt) ein = fmaxf(ein, net - tgt);
    }
  }
  if (!ok && threadIdx.x == 0) atomicExch(fail, 1);
  for (int off = 16; off > 0; off >>= 1) {
    emax = fmaxf(emax, __shfl_xor_sync(0xffffffffu, emax, off));
    ein = fmaxf(ein, __shfl_xor_sync(0xffffffffu, ein, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&err_bits[2 * s], __float_as_uint(emax));
    atomicMax(&err_bits[2 * s + 1], __float_as_uint(ein));
  }
  mlp_tc_teardown(T, ok);
}

// Forward pass of the FP32 master weights over n points (the gradient check and
// the loss report): y[k] = phi / R. One thread per point.
__global__ void k_mlp_forward(const float* __restrict__ P, const float4* __restrict__ pts, int n, float* y) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float4 u = pts[k];
  float a1[64];
  for (int j = 0; j < 64; ++j)
    a1[j] = silu_f(P[MLP_B1 + j] + P[MLP_W1 + 3 * j] * u.x + P[MLP_W1 + 3 * j + 1] * u.y + P[MLP_W1 + 3 * j + 2] * u.z);
  float out = P[MLP_B3];
  for (int j = 0; j < 64; ++j) {
    float h = P[MLP_B2 + j];
    for (int i = 0; i < 64; ++i) h = fmaf(P[MLP_W2 + 64 * j + i], a1[i], h);
    out = fmaf(P[MLP_W3 + j], silu_f(h), out);
  }
  y[k] = out;
}

// Network of the narrowphase at n points (template-frame units): phi for each,
// through the inference code (the ablation and the consistency checks).
__global__ void __launch_bounds__(MLP_TILE) k_mlp_infer(const MlpInfer* __restrict__ inf, MlpNorm nm, const double3* pts,
                                                        int n, float* phi, int* fail) {
  extern __shared__ unsigned char dyn[];
  MlpTcSmem* T = mlp_tc_smem(dyn);
  mlp_tc_setup(T);
  mlp_tc_stage(T, *inf, 0);
  bool ok = true;
  for (int k0 = blockIdx.x * MLP_TILE; k0 < n && ok; k0 += gridDim.x * MLP_TILE) {
    const int k = k0 + threadIdx.x;
    const double3 p = k < n ? pts[k] : make_double3(nm.cx, nm.cy, nm.cz);
    mlp_tc_layer1(T, (float)((p.x - nm.cx) / nm.R), (float)((p.y - nm.cy) / nm.R), (float)((p.z - nm.cz) / nm.R));
    ok = mlp_tc_mma(T);
    const float v = mlp_tc_output(T);
    if (k < n) phi[k] = ok ? v * nm.R : __int_as_float(0x7fc00000);
  }
  if (!ok && threadIdx.x == 0) atomicExch(fail, 1);
  mlp_tc_teardown(T, ok);
}

// ---------------------------------------------------------------------------
// Host launchers

void mlp_samples(const MlpShapeData& D, int nshapes, int S, unsigned long long seed, const MlpTrainOpts& opt,
                 float4* samples, cudaStream_t st) {
  k_mlp_samples<<<dim3((S + 255) / 256, nshapes), 256, 0, st>>>(D, S, seed, opt, samples);
}

cudaError_t mlp_train_step(float* params, const float4* samples, int nshapes, int S, int B, long long it,
                           float* partial, float* loss, float* m1, float* m2, float lr, int step, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp_grad_smem());
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int nblk = B / MLP_T;
  k_mlp_grad<<<dim3(nblk, nshapes), MLP_T, mlp_grad_smem(), st>>>(params, samples, S, B, it, nblk, partial, loss);
  k_mlp_adam<<<dim3((MLP_B3 + 1 + 255) / 256, nshapes), 256, 0, st>>>(params, m1, m2, partial, nblk, lr, 0.9f, 0.999f,
                                                                     1e-8f, step);
  return cudaGetLastError();
}

void mlp_pack(const float* params, int nshapes, MlpInfer* out, cudaStream_t st) {
  k_mlp_pack<<<nshapes, 256, 0, st>>>(params, out);
}

// The inference kernels' dynamic shared memory (above the 48 KB default only with the attribute).
static void mlp_tc_attr() {
  static bool done = false;
  if (done) return;
  cudaFuncSetAttribute(k_mlp_validate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MLP_TC_SMEM);
  cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MLP_TC_SMEM);
  done = true;
}

void mlp_validate(const MlpShapeData& D, int nshapes, const MlpInfer* inf, int S2, unsigned long long seed,
                  const MlpTrainOpts& opt, const float* delta, unsigned* err_bits, int* fail, cudaStream_t st) {
  mlp_tc_attr();
  k_mlp_validate<<<dim3(148, nshapes), MLP_TILE, MLP_TC_SMEM, st>>>(D, inf, S2, seed, opt, delta, err_bits, fail);
}

cudaError_t mlp_grad_once(const float* params, const float4* pts, int n, float* partial, float* loss, cudaStream_t st) {
  // n must be a multiple of 128; one "batch" of n points: block partials for B = n
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp_grad_smem());
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k_mlp_grad<<<dim3(n / MLP_T, 1), MLP_T, mlp_grad_smem(), st>>>(params, pts, n, n, 0, n / MLP_T, partial, loss);
  return cudaGetLastError();
}

void mlp_forward(const float* params, const float4* pts, int n, float* y, cudaStream_t st) {
  if (n > 0) k_mlp_forward<<<(n + 127) / 128, 128, 0, st>>>(params, pts, n, y);
}

void mlp_infer(const MlpInfer* inf, const MlpNorm& nm, const double3* pts, int n, float* phi, int* fail,
               cudaStream_t st) {
  mlp_tc_attr();
  const int tiles = (n + MLP_TILE - 1) / MLP_TILE;
  if (n > 0) k_mlp_infer<<<tiles < 1184 ? tiles : 1184, MLP_TILE, MLP_TC_SMEM, st>>>(inf, nm, pts, n, phi, fail);
}

}  // namespace lsdem
