// Learned per-shape SDF: a 3-64-64-1 SiLU network per shape template.
//
// Input: the point in the template frame (template units) normalised by the
// shape's centre c and radius R, u = (p - c) / R; output phi / R. Training
// (mlp.cu) keeps FP32 master weights. Inference runs 128 points per CTA tile on
// the 5th-generation tensor cores:
//   layer 1 (3 -> 64) and its SiLU on the CUDA cores, one thread per point, the
//     activations rounded to BF16 and stored as the A operand in shared memory
//     (K-major, 128-byte swizzle);
//   layer 2 (64 -> 64) as one 128 x 64 x 64 tcgen05.mma (kind::f16, BF16
//     operands, FP32 accumulators in tensor memory), issued by one thread, its
//     completion signalled through an mbarrier by tcgen05.commit;
//   bias, SiLU and the output dot product (64 -> 1) read back from tensor memory
//     with tcgen05.ld, each warp its own 32 lanes (= its 32 points).
// SiLU is x/2 (1 + tanh(x/2)) in packed BF16 (tanh.approx.bf16x2). Every use of
// the network is bounded by the error measured with this same code.
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

// Inference tables of one shape, built from the FP32 weights (k_mlp_pack).
//  w2: W2 in BF16 as the tensor core's B operand (N = 64 output units x K = 64
//    inputs, K-major, 128-byte swizzle): row n holds the 64 inputs of output unit
//    n (128 bytes); its 16-byte chunk c is stored at chunk c ^ (n % 8). Copied
//    as is to a 1024-byte-aligned shared-memory tile.
//  w1: (W1 row j, b1[j]); b2, w3 in FP32; b3.
struct MlpInfer {
  uint4 w2[512];
  float4 w1[64];
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
  float r_over_h;        // R / template grid spacing (phi / R -> phi / spacing)
};

// Training target: phi / R clipped to [MLP_CLIP_LO, MLP_CLIP_HI]. A rejection only needs
// the network to tell phi > delta (a few per cent of R) apart, so the deep interior and the
// far corners of the grid box are flattened; the one-sided error is measured against the
// clipped value, and clip(phi) > delta implies phi > delta since delta lies inside the clip
// range.
constexpr float MLP_CLIP_LO = -0.25f;
constexpr float MLP_CLIP_HI = 0.5f;
// Training options: target clip range (units of R) and the share of samples drawn near the
// surface (a node moved by N(0, (2h)^2) per axis; the rest uniform in the grid box).
struct MlpTrainOpts {
  float clip_lo = MLP_CLIP_LO;
  float clip_hi = MLP_CLIP_HI;
  float near = 0.5f;
};

// Points per tensor-core tile (= threads of an inference CTA) and TMEM columns.
constexpr int MLP_TILE = 128;
constexpr int MLP_TMEM_COLS = 64;
// Shared memory of one inference CTA: A tile (16 KB) and B tile (8 KB), both
// 1024-byte aligned, layer-1/3 constants, mbarrier and the TMEM address; plus
// 1024 bytes of alignment slack in the dynamic allocation.
struct MlpTcSmem {
  uint4 a[MLP_TILE * 8];   // 128 rows x 128 B
  uint4 b[512];            // 64 rows x 128 B
  float4 w1[64];
  alignas(16) float b2[64];
  alignas(16) float w3[64];
  float b3;
  unsigned tmem;
  unsigned long long mbar;
  int staged;              // shape whose weights are in b / w1 / b2 / w3 (-1: none)
  int phase;               // parity of the next mbarrier completion
};
constexpr size_t MLP_TC_SMEM = sizeof(MlpTcSmem) + 1024;

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

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// The aligned shared-memory block of an inference CTA inside the dynamic allocation.
__device__ __forceinline__ MlpTcSmem* mlp_tc_smem(unsigned char* dyn) {
  const unsigned a = smem_u32(dyn);
  return reinterpret_cast<MlpTcSmem*>(dyn + ((1024u - (a & 1023u)) & 1023u));
}

// Shared-memory matrix descriptor of a K-major, 128-byte-swizzled tile whose 8-row
// groups are 1024 bytes apart (start address and stride in 16-byte units, version 1,
// layout type 2 = 128-byte swizzle).
__device__ __forceinline__ unsigned long long mlp_desc(unsigned saddr) {
  const unsigned long long start = (saddr & 0x3FFFFu) >> 4;
  const unsigned long long lbo = 1ull, sbo = 1024ull >> 4;
  return start | (lbo << 16) | (sbo << 32) | (1ull << 46) | (2ull << 61);
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major,
// N = 64, M = 128.
constexpr unsigned MLP_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

// One warp allocates the CTA's tensor-memory columns; thread 0 sets up the mbarrier.
__device__ __forceinline__ void mlp_tc_setup(MlpTcSmem* S) {
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S->tmem)),
                 "r"(MLP_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S->mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
    S->staged = -1;
    S->phase = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
}

// Releases the tensor memory. ok = false (a wait gave up): first waits once more, again
// bounded, for the outstanding MMA before the columns are freed.
__device__ __forceinline__ void mlp_tc_teardown(MlpTcSmem* S, bool ok = true) {
  if (!ok) {
    const unsigned mb = smem_u32(&S->mbar), par = (unsigned)S->phase;
    unsigned done = 0;
    for (int it = 0; it < (1 << 22) && !done; ++it)
      asm volatile(
          "{\n\t.reg .pred q;\n\tmbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
          : "=r"(done)
          : "r"(mb), "r"(par));
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S->tmem), "r"(MLP_TMEM_COLS));
}

// Copies one shape's inference tables into the CTA's tiles (all threads).
__device__ __forceinline__ void mlp_tc_stage(MlpTcSmem* S, const MlpInfer& M, int shape) {
  __syncthreads();  // the previous tile's MMA has completed and every thread has read it
  for (int k = threadIdx.x; k < 512; k += blockDim.x) S->b[k] = __ldg(&M.w2[k]);
  for (int k = threadIdx.x; k < 64; k += blockDim.x) {
    S->w1[k] = __ldg(&M.w1[k]);
    S->b2[k] = __ldg(&M.b2[k]);
    S->w3[k] = __ldg(&M.w3[k]);
  }
  if (threadIdx.x == 0) {
    S->b3 = __ldg(&M.b3);
    S->staged = shape;
  }
  asm volatile("fence.proxy.async.shared::cta;");
  __syncthreads();
}

// Layer 1 of this thread's point (row threadIdx.x of the tile) into the A tile:
// 64 hidden units in FP32, SiLU in BF16, 8 chunks of 8 units, swizzled.
__device__ __forceinline__ void mlp_tc_layer1(MlpTcSmem* S, float ux, float uy, float uz) {
  const int r = threadIdx.x;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    unsigned w[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 a = S->w1[8 * c + 2 * q], b = S->w1[8 * c + 2 * q + 1];
      const float h0 = fmaf(a.x, ux, fmaf(a.y, uy, fmaf(a.z, uz, a.w)));
      const float h1 = fmaf(b.x, ux, fmaf(b.y, uy, fmaf(b.z, uz, b.w)));
      w[q] = silu_bf16x2(pack_bf16x2(h0, h1));
    }
    S->a[r * 8 + (c ^ (r & 7))] = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// Layer 2 of the tile: makes the A tile visible to the tensor core, thread 0 issues
// the four K = 16 steps of the 128 x 64 x 64 MMA and commits them to the mbarrier,
// the first warp waits for the completion (bounded) and the CTA meets it at a barrier,
// after which every thread orders its tensor-memory reads. Returns false when the wait
// gave up (the accumulators are then not valid; the caller sets its error flag).
__device__ __forceinline__ bool mlp_tc_mma(MlpTcSmem* S) {
  asm volatile("fence.proxy.async.shared::cta;");
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    const unsigned a0 = smem_u32(S->a), b0 = smem_u32(S->b);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const unsigned long long da = mlp_desc(a0 + 32 * k), db = mlp_desc(b0 + 32 * k);
      asm volatile(
          "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
          "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(S->tmem),
          "l"(da), "l"(db), "r"(MLP_IDESC), "r"(k));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
        smem_u32(&S->mbar)));
  }
  // one warp waits for the completion (bounded); the others meet it at the barrier
  const unsigned mb = smem_u32(&S->mbar);
  const unsigned par = (unsigned)S->phase;
  unsigned done = 1;
  if (threadIdx.x < 32) {
    done = 0;
    for (int it = 0; it < (1 << 22) && !done; ++it) {
      asm volatile(
          "{\n\t.reg .pred q;\n\tmbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
          : "=r"(done)
          : "r"(mb), "r"(par));
    }
  }
  const bool all = __syncthreads_and(done) != 0;
  if (threadIdx.x == 0 && all) S->phase ^= 1;  // a wait that gave up keeps the parity it waits for
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  return all;
}

// Read-back of this thread's row: bias, SiLU and the output dot product; then the
// tile is released for the next one (every thread's loads have completed).
__device__ __forceinline__ float mlp_tc_output(MlpTcSmem* S) {
  const unsigned warp = threadIdx.x >> 5;
  const unsigned taddr = S->tmem + ((warp * 32u) << 16);
  float y = S->b3;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    unsigned v[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr + 16u * q));
    asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
    for (int j = 0; j < 16; j += 4) {
      const int n = 16 * q + j;
      // bias and output weights of four units in one 16-byte shared-memory load each
      const float4 b = *reinterpret_cast<const float4*>(S->b2 + n);
      const float4 w = *reinterpret_cast<const float4*>(S->w3 + n);
      const unsigned s0 = silu_bf16x2(pack_bf16x2(__uint_as_float(v[j]) + b.x, __uint_as_float(v[j + 1]) + b.y));
      const unsigned s1 = silu_bf16x2(pack_bf16x2(__uint_as_float(v[j + 2]) + b.z, __uint_as_float(v[j + 3]) + b.w));
      const __nv_bfloat162 h0 = *reinterpret_cast<const __nv_bfloat162*>(&s0);
      const __nv_bfloat162 h1 = *reinterpret_cast<const __nv_bfloat162*>(&s1);
      y = fmaf(w.x, __low2float(h0), fmaf(w.y, __high2float(h0), y));
      y = fmaf(w.z, __low2float(h1), fmaf(w.w, __high2float(h1), y));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  return y;
}

#endif  // __CUDACC__

}  // namespace lsdem
