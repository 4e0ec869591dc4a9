// Learned per-shape SDF: a 3-64-64-1 SiLU network per shape template.
//
// Input: the point in the template frame (template units) normalised by the
// shape's centre c and radius R, u = (p - c) / R; output phi / R. Training
// (mlp.cu) keeps FP32 master weights; inference runs 32 points per warp on the
// tensor cores (mma.sync m16n8k16, BF16 operands, FP32 accumulation) with the
// bias of layer 1 folded in as a fourth input column, the layer-1 accumulators
// reused in registers as layer-2 A fragments, and SiLU evaluated in packed BF16
// (x/2 (1 + tanh(x/2)) with tanh.approx.bf16x2). Every use of the network in the
// narrowphase is bounded by the error measured with this same inference code.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace lsdem {

// FP32 parameter layout of one shape (training and the gradient check)
enum : int {
  MLP_W1 = 0,      // [64][3], row j = hidden unit j
  MLP_B1 = 192,    // [64]
  MLP_W2 = 256,    // [64][64], row j = output unit j, column i = input i
  MLP_B2 = 4352,   // [64]
  MLP_W3 = 4416,   // [64]
  MLP_B3 = 4480,   // [1]
  MLP_NP = 4484    // stride (16-byte multiple)
};

// Inference tables of one shape, built from the FP32 weights.
//  w1b[nt * 32 + lane]: the layer-1 B fragment (bf16x2) of n-tile nt for lane
//    (rows 2t, 2t+1 of [W1^T; b1^T; 0] at column 8 nt + g, g = lane / 4, t = lane % 4);
//  w2[64][72]: W2 in BF16, row = output unit, 72-element rows (ldmatrix, no bank
//    conflicts); b2 and w3 in FP32; b3.
struct MlpInfer {
  unsigned w1b[256];
  __nv_bfloat16 w2[64 * 72];
  float b2[64];
  float w3[64];
  float b3;
  float pad[3];
};

// Per-shape normalisation and the measured error bound (template units).
struct MlpNorm {
  float cx, cy, cz, R;   // u = (p - c) / R
  float err;             // max |phi_net - phi_grid| over the validation points
  float err_in;          // max phi_net - phi_grid where phi_grid <= delta
  float delta;           // trust band: 2 % of the shape's size
  float pad;
};

#ifdef __CUDACC__

__device__ __forceinline__ unsigned pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const unsigned*>(&v);
}

// SiLU of two values in packed BF16: x/2 (1 + tanh(x/2)).
__device__ __forceinline__ unsigned silu_bf16x2(unsigned x) {
  unsigned h, t, r;
  const unsigned half = 0x3f003f00u;  // 0.5 | 0.5
  asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(h) : "r"(x), "r"(half));
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(h));
  asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(r) : "r"(h), "r"(t), "r"(h));  // h t + h = h (1 + t)
  return r;
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldmatrix_x4(unsigned (&r)[4], const void* smem_row) {
  const unsigned addr = (unsigned)__cvta_generic_to_shared(smem_row);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr));
}

// Copies one shape's W2 (64 x 72 BF16) into this warp's shared staging area.
__device__ __forceinline__ void mlp_stage_w2(const MlpInfer& M, __nv_bfloat16* sw2) {
  const int lane = threadIdx.x & 31;
  const uint4* src = reinterpret_cast<const uint4*>(M.w2);
  uint4* dst = reinterpret_cast<uint4*>(sw2);
  for (int k = lane; k < 64 * 72 / 8; k += 32) dst[k] = src[k];
  __syncwarp();
}

// phi / R of the network at this lane's point u (all 32 lanes call it; the
// result of an inactive lane is meaningless). sw2: this warp's staged W2.
// w1b: this lane's 8 layer-1 B fragments (M.w1b[nt * 32 + lane]).
__device__ __forceinline__ float mlp_eval_warp(const MlpInfer& M, const unsigned (&w1b)[8],
                                               const __nv_bfloat16* sw2, float ux, float uy, float uz) {
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  // layer-1 A fragments: rows = points, columns (u.x, u.y, u.z, 1, 0 ...)
  unsigned a1[2][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    const int r0 = mt * 16 + g, r1 = r0 + 8;
    const float x0 = __shfl_sync(0xffffffffu, ux, r0), y0 = __shfl_sync(0xffffffffu, uy, r0);
    const float z0 = __shfl_sync(0xffffffffu, uz, r0);
    const float x1 = __shfl_sync(0xffffffffu, ux, r1), y1 = __shfl_sync(0xffffffffu, uy, r1);
    const float z1 = __shfl_sync(0xffffffffu, uz, r1);
    a1[mt][0] = t == 0 ? pack_bf16x2(x0, y0) : (t == 1 ? pack_bf16x2(z0, 1.f) : 0u);
    a1[mt][1] = t == 0 ? pack_bf16x2(x1, y1) : (t == 1 ? pack_bf16x2(z1, 1.f) : 0u);
    a1[mt][2] = 0u;
    a1[mt][3] = 0u;
  }
  // layer 1 (+ SiLU) straight into the layer-2 A fragments: the accumulators of
  // n-tiles 2k and 2k+1 are the A fragment of k-step k
  unsigned a2[2][4][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
      mma_bf16(d, a1[mt], w1b[nt], 0u);
      const int ks = nt >> 1, hi = nt & 1;
      a2[mt][ks][hi * 2 + 0] = silu_bf16x2(pack_bf16x2(d[0], d[1]));
      a2[mt][ks][hi * 2 + 1] = silu_bf16x2(pack_bf16x2(d[2], d[3]));
    }
  // layer 2 + SiLU + output layer, accumulated per row
  float y[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    // B fragments of the 4 k-steps: rows nt*8 .. +7 of W2 (outputs), 16 inputs each
    unsigned b[8];
    {
      const int row = nt * 8 + (lane & 7);
      const int col = (lane >> 3) * 8;  // lanes 0-7: k 0-7, 8-15: k 8-15, 16-23: k 16-23, 24-31: k 24-31
      unsigned r[4];
      ldmatrix_x4(r, sw2 + row * 72 + col);
      b[0] = r[0]; b[1] = r[1]; b[2] = r[2]; b[3] = r[3];
      ldmatrix_x4(r, sw2 + row * 72 + 32 + col);
      b[4] = r[0]; b[5] = r[1]; b[6] = r[2]; b[7] = r[3];
    }
    const int c0 = nt * 8 + 2 * t;
    const float bb0 = M.b2[c0], bb1 = M.b2[c0 + 1], w0 = M.w3[c0], w1 = M.w3[c0 + 1];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        const unsigned a[4] = {a2[mt][ks][0], a2[mt][ks][1], a2[mt][ks][2], a2[mt][ks][3]};
        mma_bf16(d, a, b[2 * ks], b[2 * ks + 1]);
      }
      const unsigned s0 = silu_bf16x2(pack_bf16x2(d[0] + bb0, d[1] + bb1));
      const unsigned s1 = silu_bf16x2(pack_bf16x2(d[2] + bb0, d[3] + bb1));
      const __nv_bfloat162 v0 = *reinterpret_cast<const __nv_bfloat162*>(&s0);
      const __nv_bfloat162 v1 = *reinterpret_cast<const __nv_bfloat162*>(&s1);
      y[mt][0] = fmaf(w0, __low2float(v0), fmaf(w1, __high2float(v0), y[mt][0]));
      y[mt][1] = fmaf(w0, __low2float(v1), fmaf(w1, __high2float(v1), y[mt][1]));
    }
  }
  // row sums over the 4 lanes of a group, then to the lane that owns the row
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      y[mt][h] += __shfl_xor_sync(0xffffffffu, y[mt][h], 1);
      y[mt][h] += __shfl_xor_sync(0xffffffffu, y[mt][h], 2);
    }
  const int mt = lane >> 4, rr = lane & 15, src = (rr & 7) * 4, h = rr >> 3;
  const float v00 = __shfl_sync(0xffffffffu, y[0][0], src), v01 = __shfl_sync(0xffffffffu, y[0][1], src);
  const float v10 = __shfl_sync(0xffffffffu, y[1][0], src), v11 = __shfl_sync(0xffffffffu, y[1][1], src);
  const float v = mt == 0 ? (h == 0 ? v00 : v01) : (h == 0 ? v10 : v11);
  return v + M.b3;
}

#endif  // __CUDACC__

}  // namespace lsdem
