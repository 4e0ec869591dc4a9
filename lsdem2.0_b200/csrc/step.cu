// Level-set DEM step kernels for sm_100a (FP64 "plain" form).
//
// Kernel map against the reference hot path (paths relative to the reference root):
//   k_integrate_first  half kick + drift + cell key (+ wall drift/key); replaces
//                      particleVelocityAngularVelocityIntegrationKernel + particlePositionOrientationIntegrationKernel
//                      (FunDEM/kernel/CUDAKernelFunction/particleIntegrationKernel.cu:3-40) and
//                      calculateHashKernel (myUtility/mySpatialGrid.cu:4-26)
//   k_candidates       particle-level candidate partners from the cell grid (new: replaces the
//                      per-node 27-cell scan of LSParticleContactDetectionKernel.cu:44-61)
//   k_narrowphase      node-vs-SDF tests (LSParticleContactDetectionKernel.cu:4-590), history
//                      carry-over (…cu:280-289) and the linear contact force
//                      (contactKernel.cuh:4-77, contactKernel.cu:46-271) fused in one pass
//   k_kick             second half kick (particleIntegrationKernel.cu:3-24)
//   k_periodic         wrap + ghost images + ghost keys (mySpatialGrid.cu:28-56, 87-152, 214-240)
//   k_bonds            V-bond forces (contactKernel.cuh:138-199, contactKernel.cu:273-351)
#include <cuda_fp16.h>

#include "kernels.h"

namespace lsdem {

static constexpr unsigned FULL = 0xffffffffu;
static constexpr int NP_WARPS = 4;     // warps per narrowphase block
static constexpr int MAXCL = 256;      // clusters of 32 nodes per shape (8192 nodes)
static constexpr int OLDCAP = 256;     // previous-segment node ids staged in shared memory per warp

LD unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <typename T>
LD T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}
LD double3 warp_sum3(double3 v) { return d3(warp_sum(v.x), warp_sum(v.y), warp_sum(v.z)); }
LD void atomic_add3(double3* arr, int i, double3 v) {
  atomicAdd(&arr[i].x, v.x);
  atomicAdd(&arr[i].y, v.y);
  atomicAdd(&arr[i].z, v.z);
}

// Absolute slack for conservative culling: covers FP64 rounding of coordinates.
LD double coord_slack(double3 a, double3 b) {
  return 1e-14 * (fabs(a.x) + fabs(a.y) + fabs(a.z) + fabs(b.x) + fabs(b.y) + fabs(b.z)) + 1e-300;
}

// ---------------------------------------------------------------------------
// Integration, first half of the step (reference step order, LSSolver.h:1000-1011).
__global__ void k_integrate_first(StepArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    // contacts of the previous step: largest demand of the batch, then reset
    if (a.C_old.count) atomicMax(&a.status->need_contact, *a.C_old.count);
    *a.C.count = 0;
    if (a.G.count) *a.G.count = 0;
    if (a.mb.ctr) a.mb.ctr[0] = a.mb.ctr[1] = a.mb.ctr[2] = 0;
    if (a.pl.ctr) a.pl.ctr[0] = a.pl.ctr[1] = a.pl.ctr[2] = 0;
    for (int l = 0; l < 2; ++l)
      if (a.net[l].ctr) {
        a.net[l].ctr[0] = a.net[l].ctr[1] = 0;
        for (int k = 0; k < a.nshapes; ++k) a.net[l].cnt[k] = 0;
      }
  }
  if (i < a.P.n) {
    const BodyView& P = a.P;
    const double h = 0.5 * a.dt;
    double3 v = P.vel[i], w = P.angvel[i];
    Quat q = P.quat[i];
    const double im = P.invmass[i];
    if (!is_zero(im)) {
      v += (P.force[i] * im + a.gravity) * h;
      w += (mul(rotate_inv_inertia(q, P.invI[i]), P.torque[i])) * h;
      P.vel[i] = v;
      P.angvel[i] = w;
    }
    double3 x = P.pos[i];
    x += a.dt * v;
    q = quat_integrate(q, w, a.dt);
    P.pos[i] = x;
    P.quat[i] = q;
    if (P.rotm) {  // precision form: FP32 rotation matrix (columns are rotate(q, e_j))
      const double3 c0 = rotate(q, d3(1., 0., 0.)), c1 = rotate(q, d3(0., 1., 0.)), c2 = rotate(q, d3(0., 0., 1.));
      P.rotm[3 * i] = make_float4((float)c0.x, (float)c1.x, (float)c2.x, 0.f);
      P.rotm[3 * i + 1] = make_float4((float)c0.y, (float)c1.y, (float)c2.y, 0.f);
      P.rotm[3 * i + 2] = make_float4((float)c0.z, (float)c1.z, (float)c2.z, 0.f);
    }
    P.force[i] = d3(0., 0., 0.);
    P.torque[i] = d3(0., 0., 0.);
    const int key = hash_key(x, a.pg);
    if (a.reuse) {
      // a move beyond the neighbour-list margin (a periodic wrap included) needs a new
      // sort and new lists; so does a body entering or leaving the domain, since the
      // lists hold only bodies that were in a cell at the build
      const double3 m = x - a.xb[i];
      if (dot(m, m) > a.move2 || (key < 0) != (P.key[i] < 0)) atomicOr(a.reuse, 2);
    }
    P.key[i] = key;
    if (a.pgh.cnt) a.pgh.cnt[i] = 0;
  } else if (i < a.P.n + a.W.n) {
    const int k = i - a.P.n;
    const BodyView& W = a.W;
    double3 x = W.pos[k];
    x += a.dt * W.vel[k];
    W.pos[k] = x;
    W.quat[k] = quat_integrate(W.quat[k], W.angvel[k], a.dt);
    W.key[k] = hash_key(x, a.wg);
  }
}

void launch_integrate_first(const StepArgs& a, cudaStream_t s) {
  int n = a.P.n + a.W.n;
  if (n < 1) n = 1;
  k_integrate_first<<<(n + 255) / 256, 256, 0, s>>>(a);
}

__global__ void k_kick(StepArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && a.reuse) *a.reuse = 0;  // the next step's first kernel sets it afresh
  if (i >= a.P.n) return;
  const BodyView& P = a.P;
  const double im = P.invmass[i];
  if (is_zero(im)) return;
  const double h = 0.5 * a.dt;
  double3 v = P.vel[i];
  v += (P.force[i] * im + a.gravity) * h;
  P.vel[i] = v;
  double3 w = P.angvel[i];
  w += (mul(rotate_inv_inertia(P.quat[i], P.invI[i]), P.torque[i])) * h;
  P.angvel[i] = w;
}

void launch_kick(const StepArgs& a, cudaStream_t s) {
  if (a.P.n > 0) k_kick<<<(a.P.n + 255) / 256, 256, 0, s>>>(a);
}

// ---------------------------------------------------------------------------
// Box distance helpers for conservative culling (body frame).
LD double box_dist(double3 l, double3 lo, double3 hi) {
  double dx = fmax(fmax(lo.x - l.x, l.x - hi.x), 0.0);
  double dy = fmax(fmax(lo.y - l.y, l.y - hi.y), 0.0);
  double dz = fmax(fmax(lo.z - l.z, l.z - hi.z), 0.0);
  return sqrt(dx * dx + dy * dy + dz * dz);
}
LD void grid_box(const double3 o, double invh, int3 gs, double3& lo, double3& hi) {
  lo = o;
  hi = d3(o.x + (gs.x - 1) / invh, o.y + (gs.y - 1) / invh, o.z + (gs.z - 1) / invh);
}

// True when no point within `reach` of l (wall frame) that lies in wall w's grid
// box can have phi <= 0, so that no node of a particle of that bounding radius can
// pass the wall's SDF test (sdf_eval rejects nodes outside the box, and inside it
// the interpolated phi is positive). q is l's grid position projected onto the
// box; for a node position p in the box |p - q| <= |p - l| (projection onto a
// convex set does not expand distances), the segment p-q stays in the box, and
// along it phi changes by at most the template's cell gradient-norm bound per
// grid unit (lip[2 sh + 1] spacings per spacing). phi(q) is the FP64 trilinear
// value of the grid, as the node test computes it, with a rounding margin.
LD bool wall_far(const StepArgs& a, int w, double3 l, double reach) {
  const int sh = a.W.shape[w];
  const int3 gs = a.S.gsize[sh];
  const double invh = a.W.invh[w];
  const double3 o = a.W.origin[w];
  const double qx = fmin(fmax((l.x - o.x) * invh, 0.0), (double)(gs.x - 1));
  const double qy = fmin(fmax((l.y - o.y) * invh, 0.0), (double)(gs.y - 1));
  const double qz = fmin(fmax((l.z - o.z) * invh, 0.0), (double)(gs.z - 1));
  const int i0 = min((int)qx, gs.x - 2), j0 = min((int)qy, gs.y - 2), k0 = min((int)qz, gs.z - 2);
  const double fx = qx - i0, fy = qy - j0, fz = qz - k0;
  const int sy = gs.x, sz = gs.x * gs.y;
  const double* b = a.S.sdf + a.S.sdf_off[sh] + ((size_t)k0 * sz + (size_t)j0 * sy + i0);
  const double sc = a.W.scale[w];
  double cmax = 0.0, acc = 0.0;
#pragma unroll 1
  for (int e = 0; e < 4; ++e) {  // the four x-edges of the cell
    const int dy = e & 1, dz = e >> 1;
    const double* be = b + dz * sz + dy * sy;
    const double v0 = __ldg(be), v1 = __ldg(be + 1);
    cmax = fmax(cmax, fmax(fabs(v0), fabs(v1)));
    acc += (v0 * (1.0 - fx) + v1 * fx) * (dy ? fy : 1.0 - fy) * (dz ? fz : 1.0 - fz);
  }
  const double phi = sc * acc;
  const double bound = (double)a.S.lip[2 * sh + 1] * reach * (1.0 + 1e-9) + 1e-12 * sc * cmax + 1e-300;
  return phi > bound;
}

// Appends this lane's entries A * cap + j, j < cnt, to a flat pair list, with
// one atomic per warp (all lanes of the warp call it).
LD void append_pairs(int* list, int* ctr, int A, int cap, int cnt) {
  const int lane = threadIdx.x & 31;
  int incl = cnt;
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += v;
  }
  const int tot = __shfl_sync(FULL, incl, 31);
  int base = 0;
  if (lane == 31 && tot > 0) base = atomicAdd(ctr, tot);
  base = __shfl_sync(FULL, base, 31) + incl - cnt;
  for (int j = 0; j < cnt; ++j) list[base + j] = A * cap + j;
}

// Centres and bounding radii in a sorted order (idx), FP32, for the candidate
// walks (the particle grid's, then the image search's).
__global__ void k_pack_cells(StepArgs a, const int* __restrict__ idx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.P.n) return;
  const int B = idx[k];
  const double3 x = a.P.pos[B];
  a.cell_pk[k] = make_float4((float)x.x, (float)x.y, (float)x.z, (float)a.P.radius[B]);
  if (a.pk_meta) {
    a.pk_meta[k] = make_int4(a.P.key[B], B, a.P.shape[B], __float_as_int((float)a.P.scale[B]));
    const Quat q = a.P.quat[B];
    a.pk_q[k] = make_float4((float)q.q0, (float)q.q1, (float)q.q2, (float)q.q3);
  }
}

// ---------------------------------------------------------------------------
// Support tables and the separation test of a candidate pair.
// The support of a point set P, h(w) = max over p in P of w . p, is convex and
// positively homogeneous in w. A direction u falls on one face of a cube map (the axis
// of its largest |component|, m = that |component|), where w = u / m = (+-1, p, q) in
// the face's coordinates (gnomonic square [-1, 1]^2, SUP_M x SUP_M cells). Restricted
// to the face's plane, h is convex in (p, q), so on each half of a cell (the triangles
// below and above its (p + 1, q) - (p, q + 1) diagonal) it lies below the linear
// interpolation of its values at the triangle's corners. The tables hold, per shape,
// those values at the cube map's vertices (rounded up), packed four per cell; the
// support along the unit direction u / |u| is h(w) m / |u|. Point sets: the template's
// surface nodes (sup_n) and points whose convex hull holds every point where B's
// trilinear phi can be <= 0 (sup_s; built by the host from the grid refined by two).

// Face coordinates of vertex (i, j) of face f as an unnormalised direction.
LD double3 sup_vertex(int f, int i, int j) {
  const double sg = (f & 1) ? -1.0 : 1.0;
  const double p = -1.0 + 2.0 * i / SUP_M, q = -1.0 + 2.0 * j / SUP_M;
  return f < 2 ? d3(sg, p, q) : (f < 4 ? d3(q, sg, p) : d3(p, q, sg));
}

// One warp per (shape, table, vertex): the largest projection, rounded up.
__global__ void k_support_vertices(int nshapes, const double3* __restrict__ node_pos, const int* __restrict__ node_off,
                                   const int* __restrict__ node_cnt, const double3* __restrict__ pts,
                                   const long long* __restrict__ pts_off, float* __restrict__ vtx,
                                   float* __restrict__ sup_r) {
  const int lane = threadIdx.x & 31;
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= 2LL * nshapes * SUP_VERTS) return;
  const int sh = (int)(w / (2 * SUP_VERTS)), tab = (int)((w / SUP_VERTS) & 1), v = (int)(w % SUP_VERTS);
  const int f = v / ((SUP_M + 1) * (SUP_M + 1)), j = (v / (SUP_M + 1)) % (SUP_M + 1), i = v % (SUP_M + 1);
  const double3 c = sup_vertex(f, i, j);
  double mx = -1e300;
  if (tab == 0) {
    for (int k = lane; k < node_cnt[sh]; k += 32) mx = fmax(mx, dot(c, node_pos[node_off[sh] + k]));
  } else {
    for (long long k = pts_off[sh] + lane; k < pts_off[sh + 1]; k += 32) mx = fmax(mx, dot(c, pts[k]));
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(FULL, mx, o));
  if (tab == 1 && v == 0) {  // the largest |p| of the solid's points
    double r = 0.;
    for (long long k = pts_off[sh] + lane; k < pts_off[sh + 1]; k += 32) r = fmax(r, sqrt(dot(pts[k], pts[k])));
    for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(FULL, r, o));
    if (lane == 0) sup_r[sh] = __double2float_ru(r * (1.0 + 1e-9));
  }
  // relative 1e-9 covers the rounding of the dot products and of the vertex coordinates
  if (lane == 0) vtx[w] = mx > -1e299 ? __double2float_ru(mx + 1e-9 * fabs(mx) + 1e-30) : -1e30f;
}

// One thread per (shape, table, cell): its four corner values in one float4.
__global__ void k_support_pack(int nshapes, const float* __restrict__ vtx, float4* __restrict__ sup_n,
                               float4* __restrict__ sup_s) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2LL * nshapes * SUP_CELLS) return;
  const int sh = (int)(t / (2 * SUP_CELLS)), tab = (int)((t / SUP_CELLS) & 1), cell = (int)(t % SUP_CELLS);
  const int f = cell / (SUP_M * SUP_M), j = (cell / SUP_M) % SUP_M, i = cell % SUP_M;
  const float* V = vtx + ((size_t)sh * 2 + tab) * SUP_VERTS + (size_t)f * (SUP_M + 1) * (SUP_M + 1);
  const float4 c = make_float4(V[j * (SUP_M + 1) + i], V[j * (SUP_M + 1) + i + 1], V[(j + 1) * (SUP_M + 1) + i],
                               V[(j + 1) * (SUP_M + 1) + i + 1]);
  (tab == 0 ? sup_n : sup_s)[(size_t)sh * SUP_CELLS + cell] = c;
}

void launch_support_tables(int nshapes, const double3* node_pos, const int* node_off, const int* node_cnt,
                           const double3* pts, const long long* pts_off, float* vtx, float4* sup_n, float4* sup_s,
                           float* sup_r, cudaStream_t s) {
  const long long warps = 2LL * nshapes * SUP_VERTS;
  if (warps <= 0) return;
  k_support_vertices<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(nshapes, node_pos, node_off, node_cnt, pts,
                                                                         pts_off, vtx, sup_r);
  const long long cells = 2LL * nshapes * SUP_CELLS;
  k_support_pack<<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(nshapes, vtx, sup_n, sup_s);
}

// The separation test runs in FP32 on the packed records of the candidate search, with
// explicitly rounded operations (the list filter and the walk of k_candidates inline it
// at two places; explicit rounding keeps them deciding every pair alike). Only the
// direction of the centre difference matters, so it is rotated into each body frame
// unnormalised.
LD float3 rot_inv_f(float3 v, float4 q) {
  const float w = q.x, a = -q.y, b = -q.z, c = -q.w;
  const float tx = __fmul_rn(2.0f, __fmaf_rn(b, v.z, -__fmul_rn(c, v.y)));
  const float ty = __fmul_rn(2.0f, __fmaf_rn(c, v.x, -__fmul_rn(a, v.z)));
  const float tz = __fmul_rn(2.0f, __fmaf_rn(a, v.y, -__fmul_rn(b, v.x)));
  return make_float3(__fadd_rn(__fmaf_rn(w, tx, v.x), __fmaf_rn(b, tz, -__fmul_rn(c, ty))),
                     __fadd_rn(__fmaf_rn(w, ty, v.y), __fmaf_rn(c, tx, -__fmul_rn(a, tz))),
                     __fadd_rn(__fmaf_rn(w, tz, v.z), __fmaf_rn(a, ty, -__fmul_rn(b, tx))));
}
// Upper bound of h(u / m) from the table tab of one shape; m = the largest |component|
// of u (0 when u = 0).
LD float sup_bound_f(const float4* __restrict__ tab, float3 u, float& m) {
  const float ax = fabsf(u.x), ay = fabsf(u.y), az = fabsf(u.z);
  int f;
  float p, q;
  if (ax >= ay && ax >= az) { f = u.x >= 0.f ? 0 : 1; m = ax; p = u.y; q = u.z; }
  else if (ay >= az) { f = u.y >= 0.f ? 2 : 3; m = ay; p = u.z; q = u.x; }
  else { f = u.z >= 0.f ? 4 : 5; m = az; p = u.x; q = u.y; }
  if (!(m > 0.f)) {
    m = 0.f;
    return 0.f;
  }
  const float r = __frcp_rn(m);
  const float x = __fmul_rn(__fmaf_rn(p, r, 1.0f), 0.5f * SUP_M);
  const float y = __fmul_rn(__fmaf_rn(q, r, 1.0f), 0.5f * SUP_M);
  const int i = min(max((int)floorf(x), 0), SUP_M - 1), j = min(max((int)floorf(y), 0), SUP_M - 1);
  const float s = fminf(fmaxf(__fsub_rn(x, (float)i), 0.f), 1.f), t = fminf(fmaxf(__fsub_rn(y, (float)j), 0.f), 1.f);
  const float4 c = __ldg(tab + (f * SUP_M + j) * SUP_M + i);
  if (__fadd_rn(s, t) <= 1.0f) return __fmaf_rn(s, __fsub_rn(c.y, c.x), __fmaf_rn(t, __fsub_rn(c.z, c.x), c.x));
  return __fmaf_rn(__fsub_rn(1.0f, s), __fsub_rn(c.z, c.w), __fmaf_rn(__fsub_rn(1.0f, t), __fsub_rn(c.y, c.w), c.w));
}

// Separating-axis test of the pair (A, B) along the line of centres u: every node of
// A projects onto u at most scale_A h_n(A, R_A^T u) beyond x_A, and every point where
// B's interpolated phi is <= 0 at least scale_B h_s(B, -R_B^T u) before x_B; if the two
// reaches sum to less than |x_B - x_A|, no node of A can be inside B and the pair has no
// contact. Margins: the FP32 centres differ from the FP64 ones by at most 2^-24 of each
// coordinate, so the distance by 1.2e-7 (n1 + D) and the direction by 3e-7 (n1 + D) / D;
// 2e-6 for the FP32 orientation and rotation, and 2e-6 for the rounding of the face
// coordinates and of the interpolation (the interpolated plane point moves by a few
// 1e-7, and the values, at most sqrt(3) times the set's largest |p|, round by a few
// ulps); a direction error e moves a support by at most e times the set's largest |p|
// (the bounding radius for A's nodes, scale_B sup_r for B's solid). The rotation keeps
// |R^T u| = |u| within 1e-6, covered by the relative 1e-5. Each margin is taken several
// times over.
LD bool pair_separated(const StepArgs& a, float4 pa, float n1a, float4 qa, float scA, int shA, float4 pb, float4 qb,
                       float scB, int shB) {
  const float dx = __fsub_rn(pb.x, pa.x), dy = __fsub_rn(pb.y, pa.y), dz = __fsub_rn(pb.z, pa.z);
  const float D2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
  if (!(D2 > 0.f)) return false;
  const float3 ua = rot_inv_f(make_float3(dx, dy, dz), qa);
  const float3 ub = rot_inv_f(make_float3(-dx, -dy, -dz), qb);
  float ma, mb;
  const float hA = sup_bound_f(a.S.sup_n + (size_t)shA * SUP_CELLS, ua, ma);
  const float hB = sup_bound_f(a.S.sup_s + (size_t)shB * SUP_CELLS, ub, mb);
  const float D = __fsqrt_rn(D2);
  const float reach = __fdiv_rn(__fmaf_rn(__fmul_rn(scA, ma), hA, __fmul_rn(__fmul_rn(scB, mb), hB)), D);
  const float n1 = __fadd_rn(n1a, __fadd_rn(__fadd_rn(fabsf(pb.x), fabsf(pb.y)), fabsf(pb.z)));
  const float eps = __fadd_rn(__fdiv_rn(__fmul_rn(4e-7f, __fadd_rn(n1, D)), D), 8e-6f);
  const float rho = __fadd_rn(pa.w, __fmul_rn(scB, __ldg(a.S.sup_r + shB)));
  const float slack = __fmaf_rn(eps, rho, __fmaf_rn(1e-6f, n1, __fmul_rn(1e-5f, D)));
  return __fmul_rn(__fadd_rn(reach, slack), 1.0f + 1e-5f) < D;
}

// Bounding-sphere test of the candidate search on the FP32 copies (centre and
// bounding radius): the reach carries a margin that covers their rounding
// (relative 1e-5 plus 1e-6 of the coordinates). Written with explicitly rounded
// operations so that every caller evaluates it to the same bits.
LD float reach_f(float4 pa, float n1a, float4 pb) {
  const float n1 = __fadd_rn(n1a, __fadd_rn(__fadd_rn(fabsf(pb.x), fabsf(pb.y)), fabsf(pb.z)));
  return __fmaf_rn(1e-6f, n1, __fmul_rn(__fadd_rn(pa.w, pb.w), 1.0f + 1e-5f));
}
LD float dist2_f(float4 pa, float4 pb) {
  const float dx = __fsub_rn(pb.x, pa.x), dy = __fsub_rn(pb.y, pa.y), dz = __fsub_rn(pb.z, pa.z);
  return __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
}

// Cell index along one axis of the point v, by floor and clamped to [0, n - 1]:
// monotone in v and equal to the key's int() cell for points inside the grid.
LD int ball_axis(double v, double mn, double inv, int n) {
  const double f = floor((v - mn) * inv);
  return f <= 0.0 ? 0 : (f >= (double)(n - 1) ? n - 1 : (int)f);
}
LD int3 ball_cell(double3 p, const GridP& g) {
  return make_int3(ball_axis(p.x, g.mn.x, g.inv.x, g.size.x), ball_axis(p.y, g.mn.y, g.inv.y, g.size.y),
                   ball_axis(p.z, g.mn.z, g.inv.z, g.size.z));
}

// Candidate partners of each particle A.
// Particle partners: B > A, visible (in a cell), bounding spheres within
// reach (|xA - xB| <= rA + rB is necessary for any node of A to pass the
// reference's |node - xB| <= rB test, which in turn implies B lies in the
// node's 27-cell window since cells are at least 2 max radius wide). The test
// runs on the FP32 copies (reach_f), so the candidates are a superset of the
// exact ones; the narrowphase decides every node exactly. A pair whose reaches along
// the line of centres fall short of the distance (pair_separated) has no node of A
// inside B and is dropped.
// Wall partners: visible walls whose SDF grid box the bounding sphere reaches and
// whose interpolated phi is not provably positive over it (wall_far).
// One thread per particle, threads in cell-sorted order: the lanes of a warp
// mostly share a cell, so they walk the same 27 cells (z, y, x order) in step
// and their occupant loads are broadcasts. Slots are filled in cell-walk then
// sorted-occupant order.
// The walk visits the cells of the window in ascending key order and the occupants
// of a cell in ascending index (stable sort), so its partners come in ascending
// (cell key, index) order.
//
// Neighbour lists: a step that sorts and rebuilds them (*reuse != 0) also keeps, per
// sorted position, the sorted positions k of the walk's partners within reach + skin
// (plus 1e-5 of the coordinates, beyond the FP32 rounding of either test). Until the
// next rebuild the sort is not run (thread t and position k keep their bodies) and
// every particle stays within sqrt(move2) = 0.4 skin of its position at the build, so
// a pair that passes the test now was within reach + skin then. A listed partner is a
// walk partner when its current cell is in the window of A's current clamped cell and
// it passes the same FP32 test; sorted by (current key, index) the listed partners
// are exactly the walk's, in the walk's order.
__global__ void __launch_bounds__(128) k_candidates(StepArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int n = 0, nw = 0, nl = 0;
  if (t < a.P.n) {
    const int A = a.cell_idx[t];
    const double3 xA = a.P.pos[A];
    const double rA = a.P.radius[A];
    const float4 pa = a.cell_pk[t];
    const float n1a = __fadd_rn(__fadd_rn(fabsf(pa.x), fabsf(pa.y)), fabsf(pa.z));
    const int cap = a.pp.cap;
    int* out = a.pp.id + (size_t)A * cap;
    const float4 qA = a.pk_q[t];
    const int4 mA = a.pk_meta[t];
    const float scA = __int_as_float(mA.w);
    const int shA = mA.z;
    const bool sep = a.S.sup_n != nullptr;
    const bool rebuild = a.nbr && *a.reuse != 0;
    if (t == 0 && rebuild) atomicAdd(&a.status->builds, 1);
    const int listed = a.nbr && !rebuild ? a.nbr_cnt[t] : -1;
    const int3 c = clamp_cell(cell_of(xA, a.pg), a.pg.size);
    if (listed >= 0) {
      const int sx = a.pg.size.x, sxy = a.pg.size.x * a.pg.size.y;
      int lk = -1, lb = -1;
      bool ordered = true;
      // four entries at a time: their list reads, then their key, centre and index
      // gathers, are issued together rather than one dependent chain per entry
      for (int j0 = 0; j0 < listed; j0 += 4) {
        int kk[4];
        int4 mb[4];
        float4 pb[4], qb[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) kk[u] = j0 + u < listed ? __ldg(a.nbr + (size_t)(j0 + u) * a.P.n + t) : -1;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (kk[u] >= 0) {
            mb[u] = a.pk_meta[kk[u]];
            pb[u] = __ldg(a.cell_pk + kk[u]);
            qb[u] = a.pk_q[kk[u]];
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (kk[u] < 0) continue;
          const int k = mb[u].x;
          if (k < 0 || k >= a.pg.ncells) continue;
          const int bx = k % sx, by = (k / sx) % a.pg.size.y, bz = k / sxy;
          if (abs(bx - c.x) > 1 || abs(by - c.y) > 1 || abs(bz - c.z) > 1) continue;
          const float R = reach_f(pa, n1a, pb[u]);
          if (dist2_f(pa, pb[u]) > __fmul_rn(R, R)) continue;
          const int B = mb[u].y;
          if (sep && pair_separated(a, pa, n1a, qA, scA, shA, pb[u], qb[u], __int_as_float(mb[u].w), mb[u].z)) continue;
          if (k < lk || (k == lk && B < lb)) ordered = false;
          lk = k;
          lb = B;
          if (n < cap) out[n] = B;
          ++n;
        }
      }
      if (!ordered && n <= cap) {
        // a partner changed cells since the build: restore the walk's order
        for (int u = 1; u < n; ++u) {
          const int B = out[u], kb = a.P.key[B];
          int v = u - 1;
          for (; v >= 0; --v) {
            const int C = out[v], kc = a.P.key[C];
            if (kc < kb || (kc == kb && C < B)) break;
            out[v + 1] = C;
          }
          out[v + 1] = B;
        }
      }
    } else {
      // the (up to) 3 cells of a row along x are contiguous in the sorted order
      const int x0 = c.x > 0 ? c.x - 1 : 0, x1 = c.x < a.pg.size.x - 1 ? c.x + 1 : a.pg.size.x - 1;
      // A rebuild lists every body within reach + skin of A, and that ball can reach
      // past the 27 cells (cells are only 2 rmax wide; reach + skin is up to 2.1 rmax):
      // it walks the cells the ball overlaps (at most two more per side), with a
      // rounding margin far beyond the FP32 list test's, and takes candidates only
      // from the 27-cell window, so the candidates and their order are the walk's.
      int3 lo = make_int3(x0, max(c.y - 1, 0), max(c.z - 1, 0));
      int3 hi = make_int3(x1, min(c.y + 1, a.pg.size.y - 1), min(c.z + 1, a.pg.size.z - 1));
      if (rebuild) {
        const double R = rA + a.rmax + (double)a.skin;
        const double ext = 1.001 * R + 1e-4 * (fabs(xA.x) + fabs(xA.y) + fabs(xA.z) + 4.0 * R);
        const int3 e0 = ball_cell(xA - d3(ext, ext, ext), a.pg), e1 = ball_cell(xA + d3(ext, ext, ext), a.pg);
        lo = make_int3(min(lo.x, e0.x), min(lo.y, e0.y), min(lo.z, e0.z));
        hi = make_int3(max(hi.x, e1.x), max(hi.y, e1.y), max(hi.z, e1.z));
      }
      for (int z = lo.z; z <= hi.z; ++z) {
        for (int y = lo.y; y <= hi.y; ++y) {
          const int h0 = lin3(make_int3(lo.x, y, z), a.pg.size);
          const int st = __ldg(a.cell_off + h0 + 1), en = __ldg(a.cell_off + h0 + (hi.x - lo.x) + 2);
          // sorted positions of the row's cells inside the 27-cell window
          int wst = 0, wen = 0;
          if (abs(z - c.z) <= 1 && abs(y - c.y) <= 1) {
            wst = __ldg(a.cell_off + h0 + (x0 - lo.x) + 1);
            wen = __ldg(a.cell_off + h0 + (x1 - lo.x) + 2);
          }
#pragma unroll 4
          for (int k = st; k < en; ++k) {
            const float4 pb = __ldg(a.cell_pk + k);  // read-only: loads may run ahead of the slot stores
            const float R = reach_f(pa, n1a, pb);
            const float d2 = dist2_f(pa, pb);
            if (rebuild) {
              const float n1 = __fadd_rn(n1a, __fadd_rn(__fadd_rn(fabsf(pb.x), fabsf(pb.y)), fabsf(pb.z)));
              const float Rs = __fmul_rn(__fmaf_rn(1e-5f, n1, __fadd_rn(R, a.skin)), 1.0f + 1e-4f);
              if (d2 > __fmul_rn(Rs, Rs)) continue;
              const int4 mb = a.pk_meta[k];
              const int B = mb.y;
              if (B <= A) continue;
              if (nl < a.nbr_cap) a.nbr[(size_t)nl * a.P.n + t] = k;
              ++nl;
              if (k < wst || k >= wen) continue;
              if (d2 > __fmul_rn(R, R)) continue;
              if (sep && pair_separated(a, pa, n1a, qA, scA, shA, pb, a.pk_q[k], __int_as_float(mb.w), mb.z)) continue;
              if (n < cap) out[n] = B;
              ++n;
            } else {
              if (k < wst || k >= wen) continue;
              if (d2 > __fmul_rn(R, R)) continue;
              const int4 mb = a.pk_meta[k];
              const int B = mb.y;
              if (B <= A) continue;
              if (sep && pair_separated(a, pa, n1a, qA, scA, shA, pb, a.pk_q[k], __int_as_float(mb.w), mb.z)) continue;
              if (n < cap) out[n] = B;
              ++n;
            }
          }
        }
      }
      if (rebuild) {
        // an overflowed list would need a walk on an unsorted step: the batch re-runs
        // with longer lists
        a.nbr_cnt[t] = nl <= a.nbr_cap ? nl : -1;
        if (nl > a.nbr_cap) atomicOr(&a.status->flags, OVF_NBR);
        a.xb[A] = xA;
      }
    }
    a.pp.cnt[A] = n < cap ? n : cap;
    if (n > cap) atomicOr(&a.status->flags, OVF_PP);
    // walls (few), in wall order
    const int capw = a.pw.cap;
    for (int w = 0; w < a.W.n; ++w) {
      if (a.W.key[w] < 0) continue;
      const double3 l = rotate_inv(xA - a.W.pos[w], a.W.quat[w]);
      double3 lo, hi;
      grid_box(a.W.origin[w], a.W.invh[w], a.S.gsize[a.W.shape[w]], lo, hi);
      const double reach = rA * (1.0 + 1e-9) + coord_slack(xA, a.W.pos[w]) + 1e-12 * len(hi - lo);
      if (box_dist(l, lo, hi) > reach) continue;
      if (wall_far(a, w, l, reach)) continue;
      if (nw < capw) a.pw.id[(size_t)A * capw + nw] = w;
      ++nw;
    }
    if (capw > 0) a.pw.cnt[A] = nw < capw ? nw : capw;
    if (nw > capw) atomicOr(&a.status->flags, OVF_WALL);
  }
  if (a.pl.ctr) {  // precision form: flat pair lists
    const int A = t < a.P.n ? a.cell_idx[t] : 0;
    append_pairs(a.pl.list[0], &a.pl.ctr[0], A, a.pp.cap, t < a.P.n ? a.pp.cnt[A] : 0);
    if (a.pw.cap > 0) append_pairs(a.pl.list[1], &a.pl.ctr[1], A, a.pw.cap, t < a.P.n ? min(nw, a.pw.cap) : 0);
  }
  // largest demand of the warp, one atomic per warp
  n = __reduce_max_sync(FULL, n);
  nw = __reduce_max_sync(FULL, nw);
  nl = __reduce_max_sync(FULL, nl);
  if ((threadIdx.x & 31) == 0) {
    if (n > 0) atomicMax(&a.status->need_pp, n);
    if (nw > 0) atomicMax(&a.status->need_wall, nw);
    if (nl > 0) atomicMax(&a.status->need_nbr, nl);
  }
}

void launch_candidates(const StepArgs& a, cudaStream_t s) {
  if (a.P.n <= 0) return;
  k_pack_cells<<<(a.P.n + 255) / 256, 256, 0, s>>>(a, a.cell_idx);
  k_candidates<<<(a.P.n + 127) / 128, 128, 0, s>>>(a);
}

// ---------------------------------------------------------------------------
// Narrowphase.
enum { KIND_PP = 0, KIND_WALL = 1, KIND_GHOST = 2 };

// The owner particle A of the warp.
struct SelfCtx {
  double3 x, v, w;
  Quat q;
  double sc;
  int n0, nn, cl0, ncl;
};

// Contact constants of one pair (contactKernel.cu:99-104 / :176-179 and the damping
// terms of LinearContact, contactKernel.cuh:50-58), evaluated once per pair.
struct PairK {
  double kn, ks, mu, cn, cs;
};

// The SDF side of a test.
struct Partner {
  double3 x;        // centre
  Quat q;
  double r;         // bounding radius (particle partners)
  double3 o;        // grid origin (body frame)
  double invh;
  int3 gs;
  const double* sdf;
  double sc;        // SDF value scale
  int key;          // cell key (walls: wall grid, ghosts: particle grid)
  int real;         // particle index receiving the reaction (-1: none)
  double3 v, w;     // velocity, angular velocity
  double invm, kn, ks, mu, res;
};

template <int KIND>
LD Partner load_partner(const StepArgs& a, int pid) {
  Partner P;
  if (KIND == KIND_WALL) {
    const BodyView& W = a.W;
    P.x = W.pos[pid]; P.q = W.quat[pid]; P.r = W.radius[pid];
    P.o = W.origin[pid]; P.invh = W.invh[pid];
    const int sh = W.shape[pid];
    P.gs = a.S.gsize[sh]; P.sdf = a.S.sdf + a.S.sdf_off[sh]; P.sc = W.scale[pid];
    P.key = W.key[pid]; P.real = -1;
    P.v = W.vel[pid]; P.w = W.angvel[pid];
    P.invm = 0.; P.kn = 0.; P.ks = 0.; P.mu = W.mu[pid]; P.res = W.res[pid];
  } else {
    const BodyView& B = a.P;
    int i = pid, set = 0;
    if (KIND == KIND_GHOST) { i = pid >> 3; set = pid & 7; }
    if (KIND == KIND_GHOST) {
      P.x = a.G.gpos[(size_t)set * B.n + i];
      P.key = a.G.gkey[(size_t)set * B.n + i];
    } else {
      P.x = B.pos[i];
      P.key = B.key[i];
    }
    P.q = B.quat[i]; P.r = B.radius[i];
    P.o = B.origin[i]; P.invh = B.invh[i];
    const int sh = B.shape[i];
    P.gs = a.S.gsize[sh]; P.sdf = a.S.sdf + a.S.sdf_off[sh]; P.sc = B.scale[i];
    P.real = i;
    P.v = B.vel[i]; P.w = B.angvel[i];
    if (KIND == KIND_GHOST && a.G.sector) {
      // rotated image: its own orientation and velocity; the angular velocity stays the
      // particle's (addGhostLevelSetParticleContactForceTorqueKernel, contactKernel.cu:240-242)
      P.q = a.G.gquat[(size_t)set * B.n + i];
      P.v = a.G.gvel[(size_t)set * B.n + i];
    }
    P.invm = B.invmass[i]; P.kn = B.kn[i]; P.ks = B.ks[i]; P.mu = B.mu[i]; P.res = B.res[i];
  }
  return P;
}

LD double3 node_world(const StepArgs& a, const SelfCtx& S, int ni) {
  const double3 nl = a.S.node_pos[S.n0 + ni] * S.sc;
  return rotate(S.q, nl) + S.x;
}

// Trilinear SDF evaluation at world point w (LSParticleContactDetectionKernel.cu:63-115,
// interpolateLevelSetFunctionValue .cuh:4-32). True when inside the grid with overlap >= 0.
LD bool sdf_eval(double3 w, const Partner& P, double& ov, double& fx, double& fy, double& fz, double* c) {
  const double3 l = rotate_inv(w - P.x, P.q);
  const double gx = (l.x - P.o.x) * P.invh;
  const double gy = (l.y - P.o.y) * P.invh;
  const double gz = (l.z - P.o.z) * P.invh;
  const int i0 = (int)floor(gx), j0 = (int)floor(gy), k0 = (int)floor(gz);
  if (i0 < 0 || j0 < 0 || k0 < 0) return false;
  if (i0 >= P.gs.x - 1 || j0 >= P.gs.y - 1 || k0 >= P.gs.z - 1) return false;
  fx = gx - (double)i0;
  fy = gy - (double)j0;
  fz = gz - (double)k0;
  const int sx = 1, sy = P.gs.x, sz = P.gs.x * P.gs.y;
  const double* b = P.sdf + (k0 * sz + j0 * sy + i0);
  c[0] = P.sc * __ldg(b);
  c[1] = P.sc * __ldg(b + sx);
  c[2] = P.sc * __ldg(b + sy);
  c[3] = P.sc * __ldg(b + sy + sx);
  c[4] = P.sc * __ldg(b + sz);
  c[5] = P.sc * __ldg(b + sz + sx);
  c[6] = P.sc * __ldg(b + sz + sy);
  c[7] = P.sc * __ldg(b + sz + sy + sx);
  const double wx0 = 1.0 - fx, wx1 = fx, wy0 = 1.0 - fy, wy1 = fy, wz0 = 1.0 - fz, wz1 = fz;
  const double phi = c[0] * wx0 * wy0 * wz0 + c[1] * wx1 * wy0 * wz0 + c[2] * wx0 * wy1 * wz0 +
                     c[3] * wx1 * wy1 * wz0 + c[4] * wx0 * wy0 * wz1 + c[5] * wx1 * wy0 * wz1 +
                     c[6] * wx0 * wy1 * wz1 + c[7] * wx1 * wy1 * wz1;
  ov = -phi;
  return ov >= 0.;
}

// Gradient in grid units (interpolateLevelSetFunctionGradient, .cuh:34-77).
LD double3 sdf_grad(double fx, double fy, double fz, const double* c, int flags) {
  const double x = (flags & FIX_GRADIENT) ? fx : (double)(int)fx;
  const double wx0 = 1.0 - x, wx1 = x, wy0 = 1.0 - fy, wy1 = fy, wz0 = 1.0 - fz, wz1 = fz;
  const double gx = (c[1] - c[0]) * wy0 * wz0 + (c[3] - c[2]) * wy1 * wz0 + (c[5] - c[4]) * wy0 * wz1 +
                    (c[7] - c[6]) * wy1 * wz1;
  const double gy = (c[2] - c[0]) * wx0 * wz0 + (c[3] - c[1]) * wx1 * wz0 + (c[6] - c[4]) * wx0 * wz1 +
                    (c[7] - c[5]) * wx1 * wz1;
  const double gz = (c[4] - c[0]) * wx0 * wy0 + (c[5] - c[1]) * wx1 * wy0 + (c[6] - c[2]) * wx0 * wy1 +
                    (c[7] - c[3]) * wx1 * wy1;
  return d3(gx, gy, gz);
}

// Exact per-node admission test of the reference for each partner kind.
template <int KIND>
LD bool node_admitted(const StepArgs& a, double3 w, const Partner& P) {
  if (KIND == KIND_PP) {
    const double3 r = w - P.x;
    return !(len2(r) > P.r * P.r);
  } else {
    int3 c, lo, hi;
    node_window(w, KIND == KIND_WALL ? a.wg : a.pg, c, lo, hi);
    return in_window(P.key, KIND == KIND_WALL ? a.wg : a.pg, c, lo, hi);
  }
}

// Conservative cluster cull: false only when no node of the cluster can pass.
template <int KIND>
LD bool cluster_may_hit(double3 wc, double rad, const Partner& P) {
  const double slack = coord_slack(wc, P.x);
  if (KIND == KIND_PP) {
    const double R = (P.r + rad) * (1.0 + 1e-9) + slack;
    return len2(wc - P.x) <= R * R;
  } else {
    const double3 l = rotate_inv(wc - P.x, P.q);
    double3 lo, hi;
    grid_box(P.o, P.invh, P.gs, lo, hi);
    return box_dist(l, lo, hi) <= rad * (1.0 + 1e-9) + slack + 1e-12 * len(hi - lo);
  }
}

LD double sqrt_damp(double v, int flags) { return (flags & FIX_SQRTF) ? sqrt(v) : (double)sqrtf((float)v); }

template <int KIND>
LD PairK pair_constants(const StepArgs& a, int A, const Partner& P) {
  const double invmA = a.P.invmass[A], knA = a.P.kn[A], ksA = a.P.ks[A], muA = a.P.mu[A], resA = a.P.res[A];
  double kn = 0., ks = 0., effM = 0., mu, res;
  if (KIND == KIND_WALL) {
    kn = knA; ks = ksA;
    if (invmA > 0.) effM = 1. / invmA;
    mu = fmin(muA, P.mu);
    res = fmin(resA, P.res);
  } else {
    if (knA > 0. && P.kn > 0.) kn = knA * P.kn / (knA + P.kn);
    if (ksA > 0. && P.ks > 0.) ks = ksA * P.ks / (ksA + P.ks);
    if (invmA > 0. || P.invm > 0.) effM = 1. / (invmA + P.invm);
    res = fmin(resA, P.res);
    mu = fmin(muA, P.mu);
  }
  const double logRes = log(res);
  const double diss = -logRes / sqrt_damp(logRes * logRes + M_PI * M_PI, a.flags);
  PairK k;
  k.kn = kn; k.ks = ks; k.mu = mu;
  k.cn = 2. * diss * sqrt_damp(effM * kn, a.flags);
  k.cs = 2. * diss * sqrt_damp(effM * ks, a.flags);
  return k;
}

// integrateSlidingSpring + LinearContact (contactKernel.cuh:4-77) with the pair constants.
LD void linear_contact(double3& F, double3& spring, double3 vc, double3 n, double delta, double dt, const PairK& k) {
  if (delta > 0.) {
    const double3 vn = dot(vc, n) * n;
    const double3 fn = k.kn * delta * n - k.cn * vn;
    const double3 vs = vc - vn;
    double3 s = d3(0., 0., 0.);
    if (k.mu > 0. && k.ks > 0.) {
      double3 p1 = spring - dot(spring, n) * n;
      const double a1 = len(p1);
      if (!is_zero(a1)) p1 *= len(spring) / a1;
      s = p1 + vs * dt;
      double3 fs = -k.ks * s - k.cs * vs;
      const double afs = len(fs), afn = len(fn);
      if (!is_zero(afs) && afs > k.mu * afn) {
        const double ratio = k.mu * afn / afs;
        fs *= ratio;
        s = -(fs + k.cs * vs) / k.ks;
      }
    }
    spring = s;
    const double3 fsl = -k.ks * spring - k.cs * vs;
    F = fn + fsl;
  } else {
    spring = d3(0., 0., 0.);
    F = d3(0., 0., 0.);
  }
}

template <int KIND>
LD const SlotView& slots_of(const StepArgs& a, bool old) {
  if (KIND == KIND_PP) return old ? a.pp_old : a.pp;
  if (KIND == KIND_WALL) return old ? a.pw_old : a.pw;
  return old ? a.pgh_old : a.pgh;
}

// The reference's per-node test in FP64: admission, then node inside the
// partner's SDF grid with phi <= 0.
template <int KIND>
LD bool node_hits(const StepArgs& a, const SelfCtx& S, const Partner& P, int ni) {
  const double3 w = node_world(a, S, ni);
  if (!node_admitted<KIND>(a, w, P)) return false;
  double ov, fx, fy, fz, cr[8];
  return sdf_eval(w, P, ov, fx, fy, fz, cr);
}

// Contact geometry, carried-over spring and linear contact force of one
// admitted node (LSParticleContactDetectionKernel.cu:63-115, contactKernel.cu:75-117 /
// :155-190 / :225-270); writes the contact at pos.
template <int KIND>
LD void contact_node(const StepArgs& a, const SelfCtx& S, const Partner& P, const PairK& K, int ni, int ostart,
                     int ocnt, bool staged, const int* s_old, int pos, bool can_write, double3& FA, double3& TA,
                     double3& FB, double3& TB) {
  const double3 w = node_world(a, S, ni);
  double ov, fx, fy, fz, cr[8];
  sdf_eval(w, P, ov, fx, fy, fz, cr);
  double3 n = sdf_grad(fx, fy, fz, cr, a.flags);
  n = rotate(P.q, n);
  n = normalize_dev(n);
  const double3 pc = w + 0.5 * ov * n;
  // carried-over spring: binary search of node ni in the old segment (sorted by node)
  double3 spring = d3(0., 0., 0.);
  int lo = 0, hi = ocnt - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int v = staged ? s_old[mid] : a.C_old.node[ostart + mid];
    if (v == ni) { spring = a.C_old.spring[ostart + mid]; break; }
    if (v < ni) lo = mid + 1; else hi = mid - 1;
  }
  const double3 vc = S.v + cross(S.w, pc - S.x) - (P.v + cross(P.w, pc - P.x));
  double3 F;
  linear_contact(F, spring, vc, n, ov, a.dt, K);
  if (can_write) {
    a.C.node[pos] = ni;
    a.C.spring[pos] = spring;
    if (a.C.point) {
      a.C.point[pos] = pc;
      a.C.normal[pos] = n;
      a.C.overlap[pos] = ov;
      a.C.en_n[pos] = 0.5 * ov * ov * K.kn;
      a.C.en_s[pos] = 0.5 * len2(spring) * K.ks;
    }
  }
  FA += F;
  TA += cross(pc - S.x, F);
  FB -= F;
  TB += cross(pc - P.x, -F);
}

// Second half of a pair, shared by both arithmetic forms: given the ballots of
// admitted nodes per chunk of 32 (s_mask; node_at(k) is this lane's node of
// chunk k, chunks in ascending node order), one
// atomic reserves a contiguous segment ordered by node, the previous step's
// segment of the same pair is located, and the contacts are evaluated and
// written in FP64. The partner's reaction is reduced over the warp and added
// with one atomic per component.
template <int KIND, class NodeAt>
LD void finish_pair(const StepArgs& a, int A, int slot, int pid, const SelfCtx& S, const Partner& P,
                    NodeAt node_at, const unsigned* s_mask, int* s_old, int nsurv, int total, double3& FA,
                    double3& TA) {
  const int lane = threadIdx.x & 31;
  const SlotView& cur = slots_of<KIND>(a, false);
  const size_t sidx = (size_t)A * cur.cap + slot;
  int base = 0;
  if (lane == 0 && total > 0) base = atomicAdd(a.C.count, total);
  base = __shfl_sync(FULL, base, 0);
  const bool can_write = (base + total <= a.C.cap);
  if (lane == 0) {
    cur.seg_start[sidx] = base;
    cur.seg_cnt[sidx] = can_write ? total : 0;
    if (!can_write) atomicOr(&a.status->flags, OVF_CONTACT);
  }
  if (total == 0) return;
  // previous segment of the same pair
  const SlotView& old = slots_of<KIND>(a, true);
  int ostart = 0, ocnt = 0;
  if (old.cnt != nullptr) {
    const int on = old.cnt[A] < old.cap ? old.cnt[A] : old.cap;
    for (int j0 = 0; j0 < on; j0 += 32) {
      const int j = j0 + lane;
      const bool match = j < on && old.id[(size_t)A * old.cap + j] == pid;
      const unsigned m = __ballot_sync(FULL, match);
      if (m) {
        const int src = j0 + __ffs(m) - 1;
        ostart = old.seg_start[(size_t)A * old.cap + src];
        ocnt = old.seg_cnt[(size_t)A * old.cap + src];
        break;
      }
    }
  }
  // the previous segment's node ids in shared memory (binary-searched by every contact)
  const bool staged = ocnt <= OLDCAP;
  if (staged)
    for (int j = lane; j < ocnt; j += 32) s_old[j] = a.C_old.node[ostart + j];
  __syncwarp();
  const PairK K = pair_constants<KIND>(a, A, P);
  double3 FB = d3(0., 0., 0.), TB = d3(0., 0., 0.);
  int off = 0;
  for (int k = 0; k < nsurv; ++k) {
    const unsigned m = s_mask[k];
    if (m == 0) continue;
    if ((m >> lane) & 1u)
      contact_node<KIND>(a, S, P, K, node_at(k), ostart, ocnt, staged, s_old,
                         base + off + __popc(m & lanemask_lt()), can_write, FA, TA, FB, TB);
    off += __popc(m);
  }
  if (KIND != KIND_WALL && !(KIND == KIND_GHOST && P.real == A)) {
    FB = warp_sum3(FB);
    TB = warp_sum3(TB);
    if (lane == 0) {
      atomic_add3(a.P.force, P.real, FB);
      atomic_add3(a.P.torque, P.real, TB);
    }
  }
}

// Processes one (A, partner) pair with the whole warp in FP64: cluster culling,
// then a first sweep over the surviving clusters that ballots the admitted
// nodes, then finish_pair.
template <int KIND>
LD void do_pair(const StepArgs& a, int A, int slot, int pid, const SelfCtx& S, int* s_cl, unsigned* s_mask,
                int* s_old, double3& FA, double3& TA) {
  const int lane = threadIdx.x & 31;
  __syncwarp();  // the previous pair's second sweep may still read s_cl / s_mask
  const Partner P = load_partner<KIND>(a, pid);
  // cluster culling
  int nsurv = 0;
  for (int c0 = 0; c0 < S.ncl; c0 += 32) {
    const int c = c0 + lane;
    bool keep = false;
    if (c < S.ncl) {
      const double4 sp = a.S.cl_sphere[S.cl0 + c];
      const double3 wc = rotate(S.q, d3(sp.x, sp.y, sp.z) * S.sc) + S.x;
      keep = cluster_may_hit<KIND>(wc, sp.w * S.sc, P);
    }
    const unsigned m = __ballot_sync(FULL, keep);
    if (keep) s_cl[nsurv + __popc(m & lanemask_lt())] = c;
    nsurv += __popc(m);
  }
  __syncwarp();
  // sweep 1: admission + SDF test
  int total = 0;
  for (int k = 0; k < nsurv; ++k) {
    const int ni = s_cl[k] * 32 + lane;
    const bool hit = ni < S.nn && node_hits<KIND>(a, S, P, ni);
    const unsigned m = __ballot_sync(FULL, hit);
    if (lane == 0) s_mask[k] = m;
    total += __popc(m);
  }
  __syncwarp();
  finish_pair<KIND>(a, A, slot, pid, S, P, [&](int k) { return s_cl[k] * 32 + lane; }, s_mask, s_old, nsurv, total,
                    FA, TA);
}

template <int KINDS>
__global__ void __launch_bounds__(NP_WARPS * 32, 2) k_narrowphase(StepArgs a) {
  __shared__ int s_cl[NP_WARPS][MAXCL];
  __shared__ unsigned s_mask[NP_WARPS][MAXCL];
  __shared__ int s_old[NP_WARPS][OLDCAP];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int ng_max = 0;
  for (int A = blockIdx.x * NP_WARPS + warp; A < a.P.n; A += gridDim.x * NP_WARPS) {
    const int npp = (KINDS & 1) ? a.pp.cnt[A] : 0;
    const int nw = (KINDS & 2) ? (a.pw.cap > 0 ? a.pw.cnt[A] : 0) : 0;
    const int ng = (KINDS & 4) ? a.pgh.cnt[A] : 0;
    ng_max = ng > ng_max ? ng : ng_max;
    const int ngc = ng < a.pgh.cap ? ng : a.pgh.cap;
    if (npp + nw + ngc == 0) continue;
    SelfCtx S;
    S.x = a.P.pos[A]; S.v = a.P.vel[A]; S.w = a.P.angvel[A]; S.q = a.P.quat[A];
    S.sc = a.P.scale[A];
    const int sh = a.P.shape[A];
    S.n0 = a.S.node_off[sh]; S.nn = a.S.node_cnt[sh];
    S.cl0 = a.S.cl_off[sh]; S.ncl = a.S.cl_cnt[sh];
    double3 FA = d3(0., 0., 0.), TA = d3(0., 0., 0.);
    for (int j = 0; j < npp; ++j)
      do_pair<KIND_PP>(a, A, j, a.pp.id[(size_t)A * a.pp.cap + j], S, s_cl[warp], s_mask[warp], s_old[warp], FA, TA);
    for (int j = 0; j < nw; ++j)
      do_pair<KIND_WALL>(a, A, j, a.pw.id[(size_t)A * a.pw.cap + j], S, s_cl[warp], s_mask[warp], s_old[warp], FA, TA);
    for (int j = 0; j < ngc; ++j)
      do_pair<KIND_GHOST>(a, A, j, a.pgh.id[(size_t)A * a.pgh.cap + j], S, s_cl[warp], s_mask[warp], s_old[warp], FA, TA);
    FA = warp_sum3(FA);
    TA = warp_sum3(TA);
    if (lane == 0) {
      atomic_add3(a.P.force, A, FA);
      atomic_add3(a.P.torque, A, TA);
    }
  }
  if ((KINDS & 4) && lane == 0 && ng_max > 0) atomicMax(&a.status->need_ghost, ng_max);
}

// ---------------------------------------------------------------------------
// Precision form: certified FP32 screening on 16-bit SDF templates.
//
// Almost every node the narrowphase visits is rejected (outside the partner's
// bounding sphere or cell window, or phi > 0). The precision form makes those
// rejections in FP32 against SDF templates stored as phi / h in FP16 or BF16,
// and rejects a node only when error bounds prove that the FP64 test
// (node_hits) rejects it too. Every node it cannot reject is decided by
// node_hits itself, and every contact is evaluated by the FP64 code of
// finish_pair. Pair lists, contact segments and forces are therefore those of
// the FP64 form; the 16-bit store and FP32 arithmetic only make the rejections
// cheaper.
//
// Per pair, the owner's node offsets n (template units) map to the partner's
// frame by l = M n + dB, M = R_B^T R_A scale_A, dB = R_B^T (xA - xB), and to its
// grid by g = l invh + cg, cg = -origin invh. M and dB are formed in FP32 from the
// step's FP32 rotation matrices (each entry rounded once from FP64) and from
// xA - xB rounded from FP64.
//
// Error bounds (unit roundoff u = 2^-24; |.|_1 norms bound the Euclidean ones):
// l carries at most ~10u (N1 + |d|_1) of rounding, N1 = sqrt(3) x the largest
// node distance x scale_A, and g adds u |g|_1 + invh u |origin|_1; EPS_F = 1.6e-5
// (~270u) bounds all of it with a wide margin: el = EPS_F (N1 + 2 |d|_1) in
// length, eg = invh (el + EPS_F |origin|_1) + EPS_F (sizes summed) in grid units
// per axis. The 16-bit corners c differ from the FP64 values v by at most
// Q |v| (Q = 2^-11 for FP16, 2^-8 for BF16, round to nearest, plus the FP32
// rounding of phi / h and of the interpolation); an error eg in the grid point
// moves the piecewise-trilinear phi / h by at most 3 L eg, L = the largest
// difference of neighbouring grid values of the partner's template in spacings;
// and every corner of the cell lies within 3 L of the interpolated value. So
// with Q' = Q / (1 - Q), the FP64 phi at the FP64 point is positive whenever the
// interpolated 16-bit value exceeds
//   T = (3 L Q' + 3 L eg + 1e-7) / (1 - Q'),
// a constant of the pair: a node is rejected by one comparison.
LD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
LD float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
LD float3 tof(double3 v) { return f3((float)v.x, (float)v.y, (float)v.z); }
LD double3 tod(float3 v) { return d3(v.x, v.y, v.z); }

static constexpr float EPS_F = 1.6e-5f;

// relative bound of the 16-bit store and FP32 interpolation error (with margin)
template <int SDFK>
LD constexpr float quant16() { return SDFK == PREC_FP32_BF16 ? 3.95e-3f + 1e-6f : 4.95e-4f + 1e-6f; }

// Constants of one screened pair.
struct PairF {
  float M[9];        // R_B^T R_A scale_A, row-major
  float3 dB;         // R_B^T (xA - xB)
  float3 cg;         // -origin invh
  float invh;
  float ux, uy, uz;  // grid size - 1 per axis
  float R2;          // particle partners: admission radius (with margin), squared
  float rB;          // particle partners: bounding radius
  float el;          // position error bound in the partner frame (length)
  float eg;          // grid-point error bound per axis (grid units)
  float T;           // rejection threshold of phi / h
  float Tq;          // 1 / (1 - Q')
  float gmax;        // gradient-norm bound of phi / h per grid unit
  int sy, sz;        // cell strides
  const uint4* cells;
  int key;           // walls and images: the partner's cell key
  float RA[9];       // walls and images: R_A scale_A (world offsets of the nodes)
  float n1w;         // walls and images: error bound of the world node offset
  // learned SDF: u = l * ms - mc (network input), phi / h = y * mtoh, threshold Tn
  float ms, mtoh, Tn;
  float3 mc;
  int pshape;
};

// Rotation matrix columns of q (the images of the unit axes under rotate()).
LD void rot_cols(Quat q, double3 c[3]) {
  c[0] = rotate(q, d3(1., 0., 0.));
  c[1] = rotate(q, d3(0., 1., 0.));
  c[2] = rotate(q, d3(0., 0., 1.));
}

template <int KIND, int SDFK>
LD PairF make_pair_f(const StepArgs& a, int A, const Partner& P, int pshape, int pidx) {
  PairF F;
  // rows of R_A (FP32, from the step's matrices) and of R_B (particles likewise;
  // walls from their quaternion)
  float ra[9], rb[9];
  {
    const float4 r0 = __ldg(a.P.rotm + 3 * A), r1 = __ldg(a.P.rotm + 3 * A + 1), r2 = __ldg(a.P.rotm + 3 * A + 2);
    ra[0] = r0.x; ra[1] = r0.y; ra[2] = r0.z; ra[3] = r1.x; ra[4] = r1.y; ra[5] = r1.z;
    ra[6] = r2.x; ra[7] = r2.y; ra[8] = r2.z;
  }
  if (KIND == KIND_WALL || (KIND == KIND_GHOST && a.G.sector)) {
    double3 cb[3];
    rot_cols(P.q, cb);
    for (int j = 0; j < 3; ++j) {
      rb[j] = (float)cb[j].x; rb[3 + j] = (float)cb[j].y; rb[6 + j] = (float)cb[j].z;
    }
  } else {
    const float4 r0 = __ldg(a.P.rotm + 3 * pidx), r1 = __ldg(a.P.rotm + 3 * pidx + 1), r2 = __ldg(a.P.rotm + 3 * pidx + 2);
    rb[0] = r0.x; rb[1] = r0.y; rb[2] = r0.z; rb[3] = r1.x; rb[4] = r1.y; rb[5] = r1.z;
    rb[6] = r2.x; rb[7] = r2.y; rb[8] = r2.z;
  }
  const int shA = a.P.shape[A];
  const float scA = (float)a.P.scale[A];
  // M = R_B^T R_A scale_A
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      F.M[3 * i + j] = fmaf(rb[i], ra[j], fmaf(rb[3 + i], ra[3 + j], rb[6 + i] * ra[6 + j])) * scA;
  const double3 d = a.P.pos[A] - P.x;
  const float3 df = tof(d);
  F.dB = f3(fmaf(rb[0], df.x, fmaf(rb[3], df.y, rb[6] * df.z)), fmaf(rb[1], df.x, fmaf(rb[4], df.y, rb[7] * df.z)),
            fmaf(rb[2], df.x, fmaf(rb[5], df.y, rb[8] * df.z)));
  F.invh = (float)P.invh;
  F.cg = tof(-1.0 * P.o * P.invh);
  F.ux = (float)(P.gs.x - 1); F.uy = (float)(P.gs.y - 1); F.uz = (float)(P.gs.z - 1);
  const float N1 = 1.7320508f * (float)a.S.node_box[8 * shA + 6] * scA;
  const float n1d = fabsf(df.x) + fabsf(df.y) + fabsf(df.z);
  const float el = EPS_F * (N1 + 2.0f * n1d);
  F.el = el;
  F.rB = (float)P.r;
  const float R = F.rB * (1.0f + 1e-6f) + el;
  F.R2 = R * R * (1.0f + 1e-6f);
  const float eg = F.invh * (el + EPS_F * (fabsf(F.cg.x) + fabsf(F.cg.y) + fabsf(F.cg.z)) / F.invh) +
                   EPS_F * (float)(P.gs.x + P.gs.y + P.gs.z);
  F.eg = eg;
  const float L = a.S.lip[2 * pshape];
  const float Q = quant16<SDFK>();
  const float Qp = Q / (1.0f - Q);
  F.Tq = 1.0f / (1.0f - Qp);
  F.T = (3.0f * L * Qp + 3.0f * L * eg + 1e-7f) * F.Tq * (1.0f + 1e-5f);
  F.gmax = a.S.lip[2 * pshape + 1];
  F.sy = P.gs.x - 1;
  F.sz = (P.gs.x - 1) * (P.gs.y - 1);
  F.cells = a.S.cell16 + a.S.cell_off[pshape];
  F.key = P.key;
  if (KIND != KIND_PP) {
    for (int k = 0; k < 9; ++k) F.RA[k] = ra[k] * scA;
    F.n1w = EPS_F * N1;
  }
  F.pshape = pshape;
  if (a.mlp_inf) {
    // partner frame (length) -> template units (/ scale) -> network input
    const MlpNorm nm = a.mlp_norm[pshape];
    const double ht = 1.0 / (P.invh * P.sc);  // template spacing
    F.ms = (float)(1.0 / (P.sc * nm.R));
    F.mc = f3(nm.cx / nm.R, nm.cy / nm.R, nm.cz / nm.R);
    F.mtoh = (float)(nm.R / ht);
    F.Tn = a.mlp_band[pshape];
  }
  return F;
}

LD float3 mulf(const float* M, float x, float y, float z) {
  return f3(fmaf(M[0], x, fmaf(M[1], y, M[2] * z)), fmaf(M[3], x, fmaf(M[4], y, M[5] * z)),
            fmaf(M[6], x, fmaf(M[7], y, M[8] * z)));
}

// Interpolated phi / h of the 16-bit store at grid point g, which must lie in
// [0, size - 1) on every axis: one 16-byte load of the cell's corners.
template <int SDFK>
LD float2 unpack16(unsigned w) {
  if (SDFK == PREC_FP32_BF16) return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
  return __half22float2(*reinterpret_cast<const __half2*>(&w));
}
template <int SDFK>
LD float phi16_interp(uint4 w, float gx, float gy, float gz) {
  const float fx = gx - floorf(gx), fy = gy - floorf(gy), fz = gz - floorf(gz);
  const float2 c01 = unpack16<SDFK>(w.x), c23 = unpack16<SDFK>(w.y);
  const float2 c45 = unpack16<SDFK>(w.z), c67 = unpack16<SDFK>(w.w);
  const float x0 = fmaf(fx, c01.y - c01.x, c01.x), x1 = fmaf(fx, c23.y - c23.x, c23.x);
  const float x2 = fmaf(fx, c45.y - c45.x, c45.x), x3 = fmaf(fx, c67.y - c67.x, c67.x);
  const float y0 = fmaf(fy, x1 - x0, x0), y1 = fmaf(fy, x3 - x2, x2);
  return fmaf(fz, y1 - y0, y0);
}
// The cell's corners (one 16-byte load) and the interpolation, split so that the load
// can be issued early.
LD uint4 phi16_cell(const uint4* cells, int sy, int sz, float gx, float gy, float gz) {
  const int i0 = __float2int_rd(gx), j0 = __float2int_rd(gy), k0 = __float2int_rd(gz);
  return __ldg(cells + (k0 * sz + j0 * sy + i0));
}
template <int SDFK>
LD float phi16_at(const uint4* cells, int sy, int sz, float gx, float gy, float gz) {
  return phi16_interp<SDFK>(phi16_cell(cells, sy, sz, gx, gy, gz), gx, gy, gz);
}
template <int SDFK>
LD float phi16(const PairF& F, float gx, float gy, float gz) {
  return phi16_at<SDFK>(F.cells, F.sy, F.sz, gx, gy, gz);
}

// Cell-window admission of walls and images from the FP32 world node offset ra
// (error bound e): 0 = certainly rejected, 1 = certainly admitted, 2 = the FP64
// node may lie in a neighbouring cell (within e of a cell boundary).
template <int KIND>
LD int window_state(const StepArgs& a, double3 x, float3 ra, float e0, int key) {
  const GridP& g = KIND == KIND_WALL ? a.wg : a.pg;
  const double3 w = x + tod(ra);
  const double e = (double)e0 + 1e-14 * (fabs(w.x) + fabs(w.y) + fabs(w.z));
  const double ux = (w.x - g.mn.x) * g.inv.x, uy = (w.y - g.mn.y) * g.inv.y, uz = (w.z - g.mn.z) * g.inv.z;
  if (fabs(ux - rint(ux)) <= e * g.inv.x + 1e-9 || fabs(uy - rint(uy)) <= e * g.inv.y + 1e-9 ||
      fabs(uz - rint(uz)) <= e * g.inv.z + 1e-9)
    return 2;
  int3 c, lo, hi;
  node_window(w, g, c, lo, hi);
  return in_window(key, g, c, lo, hi) ? 1 : 0;
}

// FP32 screen of one node (offset nd, template units): false only when the
// FP64 test (node_hits) certainly rejects it.
template <int KIND, int SDFK>
LD bool node_may_hit_f(const StepArgs& a, double3 xA, const PairF& F, float4 nd, bool& looked) {
  const float3 l = mulf(F.M, nd.x, nd.y, nd.z) + F.dB;
  if (KIND == KIND_PP) {
    if (l.x * l.x + l.y * l.y + l.z * l.z > F.R2) return false;
  } else {
    if (window_state<KIND>(a, xA, mulf(F.RA, nd.x, nd.y, nd.z), F.n1w, F.key) == 0) return false;
  }
  const float gx = fmaf(l.x, F.invh, F.cg.x), gy = fmaf(l.y, F.invh, F.cg.y), gz = fmaf(l.z, F.invh, F.cg.z);
  // the FP64 test rejects g < 0 or g >= size - 1 on any axis
  const float lo = fminf(gx, fminf(gy, gz));
  const float hi = fmaxf(gx - F.ux, fmaxf(gy - F.uy, gz - F.uz));
  if (lo < -F.eg || hi >= F.eg) return false;
  if (lo < F.eg || hi >= -F.eg) return true;  // within the error of the grid boundary
  looked = true;
  return !(phi16<SDFK>(F, gx, gy, gz) > F.T);  // NaN never rejects
}

// Cluster cull (sphere of radius rad about the cluster centre cn, template
// units): false only when no node of the cluster can pass node_hits.
//  - particle partners: the sphere misses the partner's bounding sphere;
//  - the sphere misses the partner's grid box (nodes outside it fail the SDF test);
//  - phi / h at q, the centre projected into the box shrunk by m >= eg, exceeds
//    the cluster's reach: for a node p inside the box, |p - q| <= |p - c| +
//    sqrt(3) m (projection onto a convex set does not expand distances), the
//    segment p-q lies in the box, and along it phi / h changes by at most gmax
//    per grid unit, so phi(q) - gmax (rad + sqrt(3) m) > 0 proves phi > 0 at
//    every node of the cluster.
//  With up != nullptr (learned form), *up receives an estimate of the largest phi / h
//  over the cluster's nodes (phi at q plus gmax times the reach; +inf when phi at q is
//  not looked up): where it is below the network's rejection threshold the network would
//  reject a node only by overestimating phi there, so the nodes are not sent to it (an
//  efficiency choice only: every node the network does not see takes the grid test).
template <int KIND, int SDFK>
LD bool cluster_may_hit_f(const PairF& F, float4 cn, float scA, float* up = nullptr) {
  if (up) *up = INFINITY;
  const float3 l = mulf(F.M, cn.x, cn.y, cn.z) + F.dB;
  const float rad = cn.w * scA * (1.0f + 1e-6f);
  if (KIND == KIND_PP) {
    const float R = F.rB * (1.0f + 1e-6f) + rad + F.el;
    if (l.x * l.x + l.y * l.y + l.z * l.z > R * R * (1.0f + 1e-6f)) return false;
  }
  const float gx = fmaf(l.x, F.invh, F.cg.x), gy = fmaf(l.y, F.invh, F.cg.y), gz = fmaf(l.z, F.invh, F.cg.z);
  const float radh = rad * F.invh;
  const float dx = fmaxf(fmaxf(-gx, gx - F.ux), 0.f), dy = fmaxf(fmaxf(-gy, gy - F.uy), 0.f),
              dz = fmaxf(fmaxf(-gz, gz - F.uz), 0.f);
  const float Rb = (radh + F.eg) * (1.0f + 1e-6f);
  if (dx * dx + dy * dy + dz * dz > Rb * Rb) return false;
  const float m = fmaxf(F.eg, 1e-3f);  // > 0: q stays below size - 1, so its cell is in the grid
  if (F.ux < 4.f * m || F.uy < 4.f * m || F.uz < 4.f * m) return true;
  const float qx = fminf(fmaxf(gx, m), F.ux - m), qy = fminf(fmaxf(gy, m), F.uy - m),
              qz = fminf(fmaxf(gz, m), F.uz - m);
  const float reach = (F.gmax * (radh + 2.8f * m) + 1e-6f) * F.Tq * (1.0f + 1e-6f);
  const float ph = phi16<SDFK>(F, qx, qy, qz);
  if (up) *up = ph + reach;
  return !(ph > F.T + reach);
}

LD SelfCtx self_ctx(const StepArgs& a, int A) {
  SelfCtx S;
  S.x = a.P.pos[A]; S.v = a.P.vel[A]; S.w = a.P.angvel[A]; S.q = a.P.quat[A];
  S.sc = a.P.scale[A];
  const int sh = a.P.shape[A];
  S.n0 = a.S.node_off[sh]; S.nn = a.S.node_cnt[sh];
  S.cl0 = a.S.cl_off[sh]; S.ncl = a.S.cl_cnt[sh];
  return S;
}

template <int KIND>
LD int partner_shape(const StepArgs& a, int pid) {
  if (KIND == KIND_WALL) return a.W.shape[pid];
  return a.P.shape[KIND == KIND_GHOST ? (pid >> 3) : pid];
}

// Screens one (A, partner) pair: cluster cull, then the node screen over the
// surviving clusters. The nodes the screen cannot reject are written, in node
// order, to the precision-form node buffer and the pair is queued for
// k_contacts_f; a pair without such nodes gets its empty contact segment here.
template <int KIND, int SDFK, bool LRN>
LD void screen_pair_f(const StepArgs& a, int A, int slot, int pid, int li, int* s_cl, unsigned short* s_sub,
                      unsigned* s_mask, unsigned (&cnt)[8]) {
  const int lane = threadIdx.x & 31;
  __syncwarp();  // the previous pair's write pass may still read s_cl / s_mask
  const int shA = a.P.shape[A];
  const int n0 = a.S.node_off[shA], nn = a.S.node_cnt[shA], cl0 = a.S.cl_off[shA], ncl = a.S.cl_cnt[shA];
  const float scA = (float)a.P.scale[A];
  const double3 xA = a.P.pos[A];
  PairF F;
  {
    const Partner P = load_partner<KIND>(a, pid);
    F = make_pair_f<KIND, SDFK>(a, A, P, partner_shape<KIND>(a, pid), KIND == KIND_GHOST ? (pid >> 3) : pid);
  }
  int nsurv = 0;
  for (int c0 = 0; c0 < ncl; c0 += 32) {
    const int c = c0 + lane;
    bool keep = false;
    if (c < ncl) keep = cluster_may_hit_f<KIND, SDFK>(F, __ldg(a.S.cl_sphere_f + cl0 + c), scA);
    const unsigned m = __ballot_sync(FULL, keep);
    if (keep) s_cl[nsurv + __popc(m & lanemask_lt())] = c;
    nsurv += __popc(m);
  }
  __syncwarp();
  // second level: sub-clusters of 8 nodes of the surviving clusters, compacted in
  // ascending order; chunk k of the node loop is sub-clusters 4k .. 4k + 3. Learned
  // form: bit 15 marks a sub-cluster whose phi / h estimate is below the network's
  // threshold; its nodes take the grid test here instead of the network.
  int nsub = 0;
  for (int j0 = 0; j0 < 4 * nsurv; j0 += 32) {
    const int j = j0 + lane;
    bool keep = false;
    int sid = 0;
    if (j < 4 * nsurv) {
      sid = s_cl[j >> 2] * 4 + (j & 3);
      const float4 sp = __ldg(a.S.sub_sphere + 4 * cl0 + sid);
      float up = INFINITY;
      keep = sp.w >= 0.f && cluster_may_hit_f<KIND, SDFK>(F, sp, scA, LRN ? &up : nullptr);
      if (LRN && up <= F.Tn) sid |= 0x8000;
    }
    const unsigned m = __ballot_sync(FULL, keep);
    if (keep) s_sub[nsub + __popc(m & lanemask_lt())] = (unsigned short)sid;
    nsub += __popc(m);
  }
  const int nch = (nsub + 3) >> 2;
  cnt[0] += 1; cnt[1] += ncl; cnt[2] += nsurv; cnt[7] += nsub;
  __syncwarp();
  // this lane's node in chunk k (nn when none)
  auto node_of = [&](int k) {
    const int j = 4 * k + (lane >> 3);
    if (j >= nsub) return nn;
    const int ni = (s_sub[j] & 0x7fff) * 8 + (lane & 7);
    return ni < nn ? ni : nn;
  };
  int total = 0;
  if (LRN) {
    // Learned form: the nodes the partner's bounds cannot reject go to the network of the
    // partner's shape (k_net_screen, tensor cores), which decides with the grid test of
    // the nodes it keeps, unless their sub-cluster is marked (then the grid test runs
    // here). A pair with network nodes records all its remaining nodes in node order as
    // pending (the marked ones with a passing verdict already; k_net_compact queues the
    // survivors for the FP64 pass); a pair without takes the plain screen's tail.
    const NetView& Q = a.net[li];
    unsigned* s_dir = reinterpret_cast<unsigned*>(s_cl);  // the cluster list is spent
    int tnet = 0, tdir = 0;
    for (int k = 0; k < nch; ++k) {
      const int ni = node_of(k);
      const int j = 4 * k + (lane >> 3);
      const bool marked = j < nsub && (s_sub[j] & 0x8000);
      cnt[4] += __popc(__ballot_sync(FULL, ni < nn));
      bool need = false, may = false, looked = false;
      if (ni < nn) {
        const float4 nd = __ldg(a.S.node_pos_f + n0 + ni);
        if (marked) {
          may = node_may_hit_f<KIND, SDFK>(a, xA, F, nd, looked);
        } else {
          const float3 l = mulf(F.M, nd.x, nd.y, nd.z) + F.dB;
          bool adm;
          if (KIND == KIND_PP) adm = !(l.x * l.x + l.y * l.y + l.z * l.z > F.R2);
          else adm = window_state<KIND>(a, xA, mulf(F.RA, nd.x, nd.y, nd.z), F.n1w, F.key) != 0;
          const float gx = fmaf(l.x, F.invh, F.cg.x), gy = fmaf(l.y, F.invh, F.cg.y), gz = fmaf(l.z, F.invh, F.cg.z);
          const float lo = fminf(gx, fminf(gy, gz));
          const float hi = fmaxf(gx - F.ux, fmaxf(gy - F.uy, gz - F.uz));
          need = adm && !(lo < -F.eg || hi >= F.eg);
        }
      }
      cnt[3] += __popc(__ballot_sync(FULL, looked));
      const unsigned mn = __ballot_sync(FULL, need), md = __ballot_sync(FULL, may);
      if (lane == 0) {
        s_mask[k] = mn;
        s_dir[k] = md;
      }
      tnet += __popc(mn);
      tdir += __popc(md);
    }
    __syncwarp();
    if (tnet == 0) {
      // no node for the network: the marked nodes that passed go to the FP64 pass as in
      // the plain screen
      for (int k = lane; k < nch; k += 32) s_mask[k] = s_dir[k];
      total = tdir;
      __syncwarp();
    } else {
      const SlotView& cur = slots_of<KIND>(a, false);
      const size_t sidx = (size_t)A * cur.cap + slot;
      if (lane == 0) {  // set here; k_contacts_f writes the segment of a pair with contacts
        cur.seg_start[sidx] = 0;
        cur.seg_cnt[sidx] = 0;
      }
      const int tot = tnet + tdir;
      int pstart = 0, pi = 0;
      bool ok = false;
      if (lane == 0) {
        pstart = atomicAdd(&Q.ctr[0], tot);
        pi = atomicAdd(&Q.ctr[1], 1);
        ok = pstart + tot <= Q.pcap && pi < Q.paircap;
        if (!ok) {
          atomicOr(&a.status->flags, OVF_NET);
          const long long need = (long long)pstart + tot;
          atomicMax(&a.status->need_pend, (int)(need < 0x7fffffff ? need : 0x7fffffff));
        }
      }
      pstart = __shfl_sync(FULL, pstart, 0);
      pi = __shfl_sync(FULL, pi, 0);
      ok = __shfl_sync(FULL, ok, 0);
      if (!ok) return;
      const int sh = F.pshape;
      int off = 0;
      for (int k = 0; k < nch; ++k) {
        const unsigned mn = s_mask[k], md = s_dir[k], m = mn | md;
        if (m == 0u) continue;
        const int ni = node_of(k);
        int base = 0;
        if (lane == 0 && mn) base = atomicAdd(&Q.cnt[sh], __popc(mn));
        base = __shfl_sync(FULL, base, 0);
        if ((m >> lane) & 1u) {
          const int idx = pstart + off + __popc(m & lanemask_lt());
          Q.pend_n[idx] = ni;
          if ((md >> lane) & 1u) {
            Q.pend_v[idx] = 1;
          } else {
            const float4 nd = __ldg(a.S.node_pos_f + n0 + ni);
            const float3 l = mulf(F.M, nd.x, nd.y, nd.z) + F.dB;
            const float gx = fmaf(l.x, F.invh, F.cg.x), gy = fmaf(l.y, F.invh, F.cg.y),
                        gz = fmaf(l.z, F.invh, F.cg.z);
            const float lo = fminf(gx, fminf(gy, gz));
            const float hi = fmaxf(gx - F.ux, fmaxf(gy - F.uy, gz - F.uz));
            const bool edge = lo < F.eg || hi >= -F.eg;
            const int r = base + __popc(mn & lanemask_lt());
            if (r < Q.qcap) {
              float4* row = Q.row + 2 * ((size_t)sh * Q.qcap + r);
              row[0] = make_float4(fmaf(l.x, F.ms, -F.mc.x), fmaf(l.y, F.ms, -F.mc.y), fmaf(l.z, F.ms, -F.mc.z),
                                   __int_as_float(idx | (edge ? (int)0x80000000u : 0)));
              row[1] = make_float4(gx, gy, gz, F.T);
            } else {
              atomicOr(&a.status->flags, OVF_NET);
              atomicMax(&a.status->need_netq, r + 1);
            }
          }
        }
        off += __popc(m);
      }
      if (lane == 0) Q.pair[pi] = make_int4(A, (KIND << 24) | slot, pstart, tot);
      return;
    }
  } else {
    for (int k = 0; k < nch; ++k) {
      const int ni = node_of(k);
      cnt[4] += __popc(__ballot_sync(FULL, ni < nn));
      bool may = false, looked = false;
      if (ni < nn) may = node_may_hit_f<KIND, SDFK>(a, xA, F, __ldg(a.S.node_pos_f + n0 + ni), looked);
      cnt[3] += __popc(__ballot_sync(FULL, looked));
      const unsigned m = __ballot_sync(FULL, may);
      if (lane == 0) s_mask[k] = m;
      total += __popc(m);
    }
  }
  cnt[5] += total;
  __syncwarp();
  const SlotView& cur = slots_of<KIND>(a, false);
  const size_t sidx = (size_t)A * cur.cap + slot;
  if (total == 0) {
    if (lane == 0) {
      cur.seg_start[sidx] = 0;
      cur.seg_cnt[sidx] = 0;
    }
    return;
  }
  int start = 0;
  bool ok = false;
  if (lane == 0) {
    start = atomicAdd(&a.mb.ctr[0], total);
    const int pi = atomicAdd(&a.mb.ctr[1 + li], 1);
    ok = start + total <= a.mb.cap && pi < a.mb.pcap;
    if (ok) {
      a.mb.pair[(size_t)li * a.mb.pcap + pi] = make_int4(A, (KIND << 24) | slot, start, total);
    } else {
      // the pair index is reserved: mark its entry empty so that the contact pass skips it
      // (the node queue is full; the batch re-runs with grown capacities)
      if (pi < a.mb.pcap) a.mb.pair[(size_t)li * a.mb.pcap + pi] = make_int4(-1, 0, 0, 0);
      atomicOr(&a.status->flags, OVF_CONTACT);
      const long long need = start + total > 2LL * (pi + 1) ? start + total : 2LL * (pi + 1);
      atomicMax(&a.status->need_contact, (int)(need < 0x7fffffff ? need : 0x7fffffff));
    }
    cur.seg_start[sidx] = 0;
    cur.seg_cnt[sidx] = 0;
  }
  start = __shfl_sync(FULL, start, 0);
  ok = __shfl_sync(FULL, ok, 0);
  if (!ok) return;
  int off = 0;
  for (int k = 0; k < nch; ++k) {
    const unsigned m = s_mask[k];
    if ((m >> lane) & 1u) a.mb.node[start + off + __popc(m & lanemask_lt())] = node_of(k);
    off += __popc(m);
  }
}

// One warp per listed pair: the flat pair lists of the kinds in KINDS, in
// particle, wall, image order.
// Particle-only screens fit 64 registers (8 blocks per SM); walls and images
// need the window test's FP64 registers.
template <int KINDS, int SDFK, bool LRN>
__global__ void __launch_bounds__(NP_WARPS * 32, KINDS == 1 ? 8 : 5) k_screen_f(StepArgs a, int li) {
  __shared__ int s_cl[NP_WARPS][MAXCL];
  __shared__ unsigned short s_sub[NP_WARPS][4 * MAXCL];
  __shared__ unsigned s_mask[NP_WARPS][MAXCL];
  const int warp = threadIdx.x >> 5;
  const int n0 = (KINDS & 1) ? min(a.pl.ctr[0], a.P.n * a.pp.cap) : 0;
  const int n1 = (KINDS & 2) && a.pw.cap > 0 ? min(a.pl.ctr[1], a.P.n * a.pw.cap) : 0;
  const int n2 = (KINDS & 4) ? min(a.pl.ctr[2], a.P.n * a.pgh.cap) : 0;
  const int tot = n0 + n1 + n2;
  unsigned cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // warp-uniform screen counters
  for (int e = blockIdx.x * NP_WARPS + warp; e < tot; e += gridDim.x * NP_WARPS) {
    if ((KINDS & 1) && e < n0) {
      const int idx = __ldg(a.pl.list[0] + e);
      const int A = idx / a.pp.cap;
      screen_pair_f<KIND_PP, SDFK, LRN>(a, A, idx - A * a.pp.cap, __ldg(a.pp.id + idx), li, s_cl[warp], s_sub[warp],
                                        s_mask[warp], cnt);
    } else if ((KINDS & 2) && e < n0 + n1) {
      const int idx = a.pl.list[1][e - n0];
      const int A = idx / a.pw.cap;
      screen_pair_f<KIND_WALL, SDFK, LRN>(a, A, idx - A * a.pw.cap, a.pw.id[idx], li, s_cl[warp], s_sub[warp],
                                          s_mask[warp], cnt);
    } else if (KINDS & 4) {
      const int idx = __ldg(a.pl.list[2] + e - n0 - n1);
      const int A = idx / a.pgh.cap;
      screen_pair_f<KIND_GHOST, SDFK, LRN>(a, A, idx - A * a.pgh.cap, __ldg(a.pgh.id + idx), li, s_cl[warp], s_sub[warp],
                                           s_mask[warp], cnt);
    }
  }
  if (a.screen_stats && (threadIdx.x & 31) == 0) {
    for (int k = 0; k < 8; ++k)
      if (cnt[k]) atomicAdd(&a.screen_stats[k], (unsigned long long)cnt[k]);
    // grid screen: nodes queued for the FP64 test by partner kind (one kind per launch)
    if (!LRN && cnt[5]) atomicAdd(&a.screen_stats[8 + (KINDS == 1 ? 0 : (KINDS == 2 ? 1 : 2))], (unsigned long long)cnt[5]);
  }
}

// Queued pairs of the screen, one warp each, in FP64: the reference's node test
// on the screened nodes, then finish_pair (segment, history, forces).
template <int KIND>
LD void contacts_pair(const StepArgs& a, int A, int slot, int start, int cnt, unsigned* s_mask, int* s_old) {
  const int lane = threadIdx.x & 31;
  const int pid = slots_of<KIND>(a, false).id[(size_t)A * slots_of<KIND>(a, false).cap + slot];
  const SelfCtx S = self_ctx(a, A);
  const Partner P = load_partner<KIND>(a, pid);
  const int* nodes = a.mb.node + start;
  const int nch = (cnt + 31) >> 5;
  __syncwarp();  // the previous pair may still read s_mask / s_old
  int total = 0;
  for (int k = 0; k < nch; ++k) {
    const int j = k * 32 + lane;
    const bool hit = j < cnt && node_hits<KIND>(a, S, P, nodes[j]);
    const unsigned m = __ballot_sync(FULL, hit);
    if (lane == 0) s_mask[k] = m;
    total += __popc(m);
  }
  __syncwarp();
  double3 FA = d3(0., 0., 0.), TA = d3(0., 0., 0.);
  finish_pair<KIND>(a, A, slot, pid, S, P, [&](int k) { return nodes[k * 32 + lane]; }, s_mask, s_old, nch, total,
                    FA, TA);
  FA = warp_sum3(FA);
  TA = warp_sum3(TA);
  if (lane == 0 && total > 0) {
    atomic_add3(a.P.force, A, FA);
    atomic_add3(a.P.torque, A, TA);
  }
}

__global__ void __launch_bounds__(NP_WARPS * 32) k_contacts_f(StepArgs a, int li) {
  __shared__ unsigned s_mask[NP_WARPS][MAXCL];
  __shared__ int s_old[NP_WARPS][OLDCAP];
  const int warp = threadIdx.x >> 5;
  const int np = min(a.mb.ctr[1 + li], a.mb.pcap);
  for (int p = blockIdx.x * NP_WARPS + warp; p < np; p += gridDim.x * NP_WARPS) {
    const int4 e = a.mb.pair[(size_t)li * a.mb.pcap + p];
    if (e.x < 0) continue;  // reserved by a pair whose nodes did not fit the queue
    const int kind = e.y >> 24, slot = e.y & 0xffffff;
    if (kind == KIND_PP) contacts_pair<KIND_PP>(a, e.x, slot, e.z, e.w, s_mask[warp], s_old[warp]);
    else if (kind == KIND_WALL) contacts_pair<KIND_WALL>(a, e.x, slot, e.z, e.w, s_mask[warp], s_old[warp]);
    else contacts_pair<KIND_GHOST>(a, e.x, slot, e.z, e.w, s_mask[warp], s_old[warp]);
  }
}

// Learned form, the network pass of launch li: the queued nodes of each partner shape
// in 128-row tiles on the tensor cores (mlp.cuh), one tile per CTA at a time over a
// persistent grid. A node is kept when phi_net does not exceed the shape's network
// threshold (trust band plus the measured one-sided error, in spacings); a kept node
// then takes the 16-bit grid test of the plain screen (skipped within the error of the
// grid boundary), and its verdict goes to the pair's pending list. If a tensor-core wait
// gives up, the tile's nodes are passed on (no rejection) and the batch reports an error.
template <int SDFK>
__global__ void __launch_bounds__(MLP_TILE) k_net_screen(StepArgs a, int li) {
  extern __shared__ unsigned char dyn[];
  MlpTcSmem* T = mlp_tc_smem(dyn);
  int* s_pre = reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(T) + sizeof(MlpTcSmem));
  const NetView& Q = a.net[li];
  const int ns = a.nshapes;
  if (threadIdx.x == 0) {
    int t = 0, mx = 0;
    for (int s = 0; s < ns; ++s) {
      const int c = Q.cnt[s];
      mx = max(mx, c);
      s_pre[s] = t;
      t += (min(c, Q.qcap) + MLP_TILE - 1) / MLP_TILE;
    }
    s_pre[ns] = t;
    if (blockIdx.x == 0) {  // this step's demands, for the capacity planning
      atomicMax(&a.status->need_netq, mx);
      atomicMax(&a.status->need_pend, Q.ctr[0]);
    }
  }
  __syncthreads();
  const int tiles = s_pre[ns];
  if ((int)blockIdx.x >= tiles) return;  // no tensor memory taken
  mlp_tc_setup(T);
  unsigned evals = 0, looks = 0;
  bool ok = true;
  // tile t's shape and this thread's row; the row of the CTA's next tile is loaded while
  // the current one runs
  auto shape_of = [&](int t) {
    int sh = 0;
    while (s_pre[sh + 1] <= t) ++sh;
    return sh;
  };
  auto load_row = [&](int t, int sh, float4& u, float4& g) {
    const int r = (t - s_pre[sh]) * MLP_TILE + threadIdx.x;
    if (t < tiles && r < min(Q.cnt[sh], Q.qcap)) {
      const float4* row = Q.row + 2 * ((size_t)sh * Q.qcap + r);
      u = row[0];
      g = row[1];
    } else {
      u = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
      g = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  int t = blockIdx.x, sh = shape_of(t);
  float4 u, g;
  load_row(t, sh, u, g);
  while (t < tiles && ok) {
    if (T->staged != sh) mlp_tc_stage(T, a.mlp_inf[sh], sh);
    const int tag = __float_as_int(u.w);
    const bool act = tag != -1;
    const bool edge = act && tag < 0;
    const int idx = tag & 0x7fffffff;
    // the grid test's 16-byte cell load is in flight during layer 1 and the MMA; the
    // test is applied only to the nodes the network keeps
    uint4 cell = make_uint4(0u, 0u, 0u, 0u);
    if (act && !edge) {
      const int3 gs = a.S.gsize[sh];
      cell = phi16_cell(a.S.cell16 + a.S.cell_off[sh], gs.x - 1, (gs.x - 1) * (gs.y - 1), g.x, g.y, g.z);
    }
    mlp_tc_layer1(T, u.x, u.y, u.z);
    const float4 gc = g;
    const int tn = t + gridDim.x;
    const int shn = tn < tiles ? shape_of(tn) : sh;
    load_row(tn, shn, u, g);
    ok = mlp_tc_mma(T);
    const float y = mlp_tc_output(T);
    if (act) {
      unsigned char may = 1;
      if (ok && !(y * __ldg(&a.mlp_norm[sh].r_over_h) > __ldg(&a.mlp_band[sh]))) {
        // kept by the network: the plain screen's grid test decides (not within the error
        // of the grid boundary, where the FP64 test decides)
        if (!edge) {
          may = !(phi16_interp<SDFK>(cell, gc.x, gc.y, gc.z) > gc.w);
          ++looks;
        }
      } else if (ok) {
        may = 0;
      }
      Q.pend_v[idx] = may;
      ++evals;
    }
    t = tn;
    sh = shn;
  }
  if (!ok && threadIdx.x == 0) atomicAdd(&a.status->errors, 1);
  if (a.screen_stats) {
    evals = __reduce_add_sync(FULL, evals);
    looks = __reduce_add_sync(FULL, looks);
    if ((threadIdx.x & 31) == 0) {
      if (evals) atomicAdd(&a.screen_stats[6], (unsigned long long)evals);
      if (looks) atomicAdd(&a.screen_stats[3], (unsigned long long)looks);
    }
  }
  mlp_tc_teardown(T, ok);
}

// Learned form, after the network pass of launch li: one warp per pair record, its
// pending nodes with a passing verdict compacted in node order into the FP64 pass's
// node queue, and the pair queued for k_contacts_f (the screen's tail for the plain
// screen).
__global__ void __launch_bounds__(NP_WARPS * 32) k_net_compact(StepArgs a, int li) {
  __shared__ unsigned s_mask[NP_WARPS][MAXCL];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const NetView& Q = a.net[li];
  const int np = min(Q.ctr[1], Q.paircap);
  unsigned queued = 0;
  for (int p = blockIdx.x * NP_WARPS + warp; p < np; p += gridDim.x * NP_WARPS) {
    const int4 e = Q.pair[p];
    const int nch = (e.w + 31) >> 5;
    __syncwarp();  // the previous pair may still read s_mask
    int total = 0;
    for (int k = 0; k < nch; ++k) {
      const int j = k * 32 + lane;
      const bool may = j < e.w && Q.pend_v[e.z + j] != 0;
      const unsigned m = __ballot_sync(FULL, may);
      if (lane == 0) s_mask[warp][k] = m;
      total += __popc(m);
    }
    __syncwarp();
    if (total == 0) continue;
    queued += total;
    int start = 0;
    bool ok = false;
    if (lane == 0) {
      start = atomicAdd(&a.mb.ctr[0], total);
      const int pi = atomicAdd(&a.mb.ctr[1 + li], 1);
      ok = start + total <= a.mb.cap && pi < a.mb.pcap;
      if (ok) {
        a.mb.pair[(size_t)li * a.mb.pcap + pi] = make_int4(e.x, e.y, start, total);
      } else {
        if (pi < a.mb.pcap) a.mb.pair[(size_t)li * a.mb.pcap + pi] = make_int4(-1, 0, 0, 0);
        atomicOr(&a.status->flags, OVF_CONTACT);
        const long long need = start + total > 2LL * (pi + 1) ? start + total : 2LL * (pi + 1);
        atomicMax(&a.status->need_contact, (int)(need < 0x7fffffff ? need : 0x7fffffff));
      }
    }
    start = __shfl_sync(FULL, start, 0);
    ok = __shfl_sync(FULL, ok, 0);
    if (!ok) continue;
    int off = 0;
    for (int k = 0; k < nch; ++k) {
      const unsigned m = s_mask[warp][k];
      if ((m >> lane) & 1u) a.mb.node[start + off + __popc(m & lanemask_lt())] = Q.pend_n[e.z + k * 32 + lane] & 0x7fffffff;
      off += __popc(m);
    }
  }
  if (a.screen_stats && lane == 0 && queued) atomicAdd(&a.screen_stats[5], (unsigned long long)queued);
}

static int g_num_sms = 0;
static int num_sms() {
  if (g_num_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

template <int KINDS, int SDFK, bool LRN>
void launch_screen_k(const StepArgs& a, int li, dim3 g, dim3 b, cudaStream_t s) {
  k_screen_f<KINDS, SDFK, LRN><<<g, b, 0, s>>>(a, li);
}

// Learned form: the network pass and the compaction after the screen of launch li.
template <int SDFK>
void launch_net_k(const StepArgs& a, int li, cudaStream_t s) {
  const int smem = (int)(MLP_TC_SMEM + sizeof(int) * (a.nshapes + 1));
  static int attr = 0;  // per kernel instance: the largest dynamic shared memory set so far
  if (smem > attr) {
    cudaFuncSetAttribute(k_net_screen<SDFK>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    attr = smem;
  }
  // eight CTAs per SM (8 x 64 = all 512 tensor-memory columns, 8 x 27 KB of shared
  // memory): a CTA that finds no free columns (the other launch's pass beside it) waits
  // in tcgen05.alloc until a CTA on its SM has finished
  k_net_screen<SDFK><<<num_sms() * 8, MLP_TILE, smem, s>>>(a, li);
}
void launch_net_screen(const StepArgs& a, int li, cudaStream_t s) {
  if (!a.mlp_inf || a.P.n <= 0) return;
  if (a.precision == PREC_FP32_FP16) launch_net_k<PREC_FP32_FP16>(a, li, s);
  else launch_net_k<PREC_FP32_BF16>(a, li, s);
}
void launch_net_compact(const StepArgs& a, int li, cudaStream_t s) {
  if (!a.mlp_inf || a.P.n <= 0) return;
  k_net_compact<<<num_sms() * 16, NP_WARPS * 32, 0, s>>>(a, li);
}

template <bool LRN>
// Particle and wall pairs in two launches: the particle-only screen fits 64 registers
// (8 blocks per SM); the wall pairs (few) take the window test's FP64 registers.
void launch_screen(const StepArgs& a, int kinds, int li, dim3 g, dim3 b, cudaStream_t s) {
  if (a.precision == PREC_FP32_FP16) {
    if (kinds & 1) launch_screen_k<1, PREC_FP32_FP16, LRN>(a, li, g, b, s);
    if (kinds & 2) launch_screen_k<2, PREC_FP32_FP16, LRN>(a, li, g, b, s);
    if (kinds & 4) launch_screen_k<4, PREC_FP32_FP16, LRN>(a, li, g, b, s);
  } else {
    if (kinds & 1) launch_screen_k<1, PREC_FP32_BF16, LRN>(a, li, g, b, s);
    if (kinds & 2) launch_screen_k<2, PREC_FP32_BF16, LRN>(a, li, g, b, s);
    if (kinds & 4) launch_screen_k<4, PREC_FP32_BF16, LRN>(a, li, g, b, s);
  }
}

void launch_narrowphase(const StepArgs& a, int kinds, cudaStream_t s) {
  if (a.P.n <= 0) return;
  int want = (a.P.n + NP_WARPS - 1) / NP_WARPS;
  int cap = num_sms() * 16;
  int blocks = want < cap ? want : cap;
  const dim3 g(blocks), b(NP_WARPS * 32);
  if (a.precision == PREC_FP64) {
    if (kinds == 3) k_narrowphase<3><<<g, b, 0, s>>>(a);
    else if (kinds == 1) k_narrowphase<1><<<g, b, 0, s>>>(a);
    else if (kinds == 4) k_narrowphase<4><<<g, b, 0, s>>>(a);
    else k_narrowphase<7><<<g, b, 0, s>>>(a);
    return;
  }
  // precision form: the screen over the flat pair lists (launch_contact_pass
  // follows it); the grid is sized for the device, the list length is on it
  const int li = kinds == 4 ? 1 : 0;
  if (a.mlp_inf) launch_screen<true>(a, kinds, li, g, b, s);  // launch_net_screen and _compact follow
  else launch_screen<false>(a, kinds, li, g, b, s);
}

void launch_contact_pass(const StepArgs& a, int li, cudaStream_t s) {
  if (a.P.n <= 0 || a.precision == PREC_FP64) return;
  k_contacts_f<<<num_sms() * 4, NP_WARPS * 32, 0, s>>>(a, li);
}

// ---------------------------------------------------------------------------
// Periodic boundary: wrap along each periodic axis in x, y, z order, each
// single-axis image set taken right after its own axis is wrapped, the
// multi-axis sets after all wraps (mySpatialGrid.cu:28-56, 87-152 and the order
// of PeriodicBoundaryXY2D::updateGhostSpatialGrid, PeriodicBoundary.h:215-288).
// Ghost keys follow calculateGhostHashKernel (mySpatialGrid.cu:214-240),
// including its z-upper test against the y bound.
LD void ghost_image(double3 p, const GridP& g, int mask, double3& out) {
  const int3 c = cell_of(p, g);
  bool hit = true;
  if (mask & 1) hit = hit && c.x == 0;
  if (mask & 2) hit = hit && c.y == 0;
  if (mask & 4) hit = hit && c.z == 0;
  out = p;
  if (hit) {
    double3 off = d3(0., 0., 0.);
    if (mask & 1) off = off + d3(g.mx.x - g.mn.x, 0., 0.);
    if (mask & 2) off = off + d3(0., g.mx.y - g.mn.y, 0.);
    if (mask & 4) off = off + d3(0., 0., g.mx.z - g.mn.z);
    out += off;
  }
}
LD int ghost_key(double3 p, const GridP& g) {
  int3 c = cell_of(p, g);
  bool out = false;
  if (p.x < g.mn.x) { c.x = 0; out = true; } else if (p.x >= g.mx.x) { c.x = g.size.x - 1; out = true; }
  if (p.y < g.mn.y) { c.y = 0; out = true; } else if (p.y >= g.mx.y) { c.y = g.size.y - 1; out = true; }
  if (p.z < g.mn.z) { c.z = 0; out = true; } else if (p.z >= g.mx.y) { c.z = g.size.z - 1; out = true; }
  return out ? lin3(c, g.size) : -1;
}

// Sector periodicity about the z axis through the domain minimum m: a particle
// left of x = m.x (with y >= m.y) is turned by -90 degrees about that axis, one
// below y = m.y (with x >= m.x) by +90 degrees: position about m, velocity and
// orientation (updateVelocityPositionOrientationOutOfSectorKernel, mySpatialGrid.cu:58-85;
// the angular velocity is left as it is, as there). The particle and wall forces of
// the step were evaluated before the wrap with the pre-wrap state, so its force and
// torque turn with it (the reference evaluates them after the wrap, which mixes the
// frames as for translations). Images: a copy per set, turned by 90 degrees when the
// particle is in the first cell row along y, by 270 (-90) degrees when in the first
// cell column along x, and by 180 degrees when in both
// (calculateSectorGhostVelocityPositionOrientationKernel, mySpatialGrid.cu:154-212).
LD void sector_wrap_images(const StepArgs& a, int i, double3& p) {
  const GridP& g = a.pg;
  const int n = a.P.n;
  const double hp = 0.5 * 3.14159265358979323846;
  double3 v = a.P.vel[i];
  Quat q = a.P.quat[i];
  bool turned = false;
  double3 om = d3(0., 0., 0.);
  if (p.x < g.mn.x && p.y >= g.mn.y) {
    om = d3(0., 0., -hp);
    v = rotate_vector_dev(v, om);
    p = g.mn + rotate_vector_dev(p - g.mn, om);
    q = rotate_quaternion_dev(q, om);
    a.P.force[i] = rotate_vector_dev(a.P.force[i], om);
    a.P.torque[i] = rotate_vector_dev(a.P.torque[i], om);
    turned = true;
  }
  if (p.y < g.mn.y && p.x >= g.mn.x) {
    om = d3(0., 0., hp);
    v = rotate_vector_dev(v, om);
    p = g.mn + rotate_vector_dev(p - g.mn, om);
    q = rotate_quaternion_dev(q, om);
    a.P.force[i] = rotate_vector_dev(a.P.force[i], om);
    a.P.torque[i] = rotate_vector_dev(a.P.torque[i], om);
    turned = true;
  }
  if (turned) {
    a.P.vel[i] = v;
    a.P.quat[i] = q;
    if (a.P.rotm) {
      const double3 c0 = rotate(q, d3(1., 0., 0.)), c1 = rotate(q, d3(0., 1., 0.)), c2 = rotate(q, d3(0., 0., 1.));
      a.P.rotm[3 * i] = make_float4((float)c0.x, (float)c1.x, (float)c2.x, 0.f);
      a.P.rotm[3 * i + 1] = make_float4((float)c0.y, (float)c1.y, (float)c2.y, 0.f);
      a.P.rotm[3 * i + 2] = make_float4((float)c0.z, (float)c1.z, (float)c2.z, 0.f);
    }
  }
  double3 gp[3] = {p, p, p}, gv[3] = {v, v, v};
  Quat gq[3] = {q, q, q};
  const double ang[3] = {hp, 2.0 * hp, -hp};  // sets R90, R180, R270
  const int3 c = cell_of(p, g);
  const bool row = c.y == 0, col = c.x == 0;
  for (int s = 0; s < 3; ++s) {
    const bool on = s == 0 ? row : (s == 1 ? row && col : col);
    if (!on) continue;
    const double3 o = d3(0., 0., ang[s]);
    gv[s] = rotate_vector_dev(v, o);
    gp[s] = g.mn + rotate_vector_dev(p - g.mn, o);
    gq[s] = rotate_quaternion_dev(q, o);
  }
  for (int s = 0; s < 3; ++s) {
    a.G.gpos[(size_t)s * n + i] = gp[s];
    a.G.gvel[(size_t)s * n + i] = gv[s];
    a.G.gquat[(size_t)s * n + i] = gq[s];
  }
}

__global__ void k_periodic(StepArgs a, int axes, double3* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.P.n) return;
  const GridP& g = a.pg;
  double3 p = a.P.pos[i];
  const int n = a.P.n;
  for (int ax = 0; ax < 3; ++ax) {
    if (!((axes >> ax) & 1)) continue;
    if (ax == 0) { const double L = g.mx.x - g.mn.x; if (p.x < g.mn.x) p.x += L; else if (p.x >= g.mx.x) p.x -= L; }
    if (ax == 1) { const double L = g.mx.y - g.mn.y; if (p.y < g.mn.y) p.y += L; else if (p.y >= g.mx.y) p.y -= L; }
    if (ax == 2) { const double L = g.mx.z - g.mn.z; if (p.z < g.mn.z) p.z += L; else if (p.z >= g.mx.z) p.z -= L; }
    for (int s = 0; s < a.G.nsets; ++s)
      if (a.G.mask[s] == (1 << ax)) ghost_image(p, g, a.G.mask[s], a.G.gpos[(size_t)s * n + i]);
  }
  if (a.G.sector) {
    sector_wrap_images(a, i, p);
  } else {
    for (int s = 0; s < a.G.nsets; ++s)
      if (__popc(a.G.mask[s]) >= 2) ghost_image(p, g, a.G.mask[s], a.G.gpos[(size_t)s * n + i]);
  }
  for (int s = 0; s < a.G.nsets; ++s) a.G.gkey[(size_t)s * n + i] = ghost_key(a.G.gpos[(size_t)s * n + i], g);
  out[i] = p;
}

// out: where the wrapped positions go (the particles' own positions, or a separate array
// when the images run beside the particle narrowphase, which still reads the pre-wrap ones)
void launch_periodic(const StepArgs& a, int axes, double3* out, cudaStream_t s) {
  if (a.P.n > 0) k_periodic<<<(a.P.n + 255) / 256, 256, 0, s>>>(a, axes, out);
}

// Clamped cell of every particle after the wrap (search grid for ghost partners).
__global__ void k_clamped_keys(StepArgs a, int* key2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.P.n) return;
  key2[i] = lin3(clamp_cell(cell_of(a.P.pos[i], a.pg), a.pg.size), a.pg.size);
}
void launch_clamped_keys(const StepArgs& a, int* key2, cudaStream_t s) {
  if (a.P.n > 0) k_clamped_keys<<<(a.P.n + 255) / 256, 256, 0, s>>>(a, key2);
}

// Visible images (ghost key >= 0) are compacted into a list first: only a
// few percent of (set, particle) pairs are images, so a thread per pair would
// leave almost every lane idle.
__global__ void k_ghost_compact(StepArgs a) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool vis = t < (long long)a.G.nsets * a.P.n && a.G.gkey[t] >= 0;
  const unsigned m = __ballot_sync(FULL, vis);
  if (m == 0) return;
  int base = 0;
  const int lane = threadIdx.x & 31;
  if (lane == __ffs(m) - 1) base = atomicAdd(a.G.count, __popc(m));
  base = __shfl_sync(FULL, base, __ffs(m) - 1);
  if (vis) a.G.list[base + __popc(m & lanemask_lt())] = (int)t;
}

// Cell range along one axis of a ball (centre p, radius r) on the clamped grid,
// intersected with [c - 2, c + 2].
LD int axis_lo(double p, double mn, double inv, int size, double r, int c) {
  int v = (int)floor((p - mn - r) * inv);
  v = v < 0 ? 0 : (v > size - 1 ? size - 1 : v);
  return v > c - 2 ? v : c - 2;
}
LD int axis_hi(double p, double mn, double inv, int size, double r, int c) {
  int v = (int)floor((p - mn + r) * inv);
  v = v < 0 ? 0 : (v > size - 1 ? size - 1 : v);
  return v < c + 2 ? v : c + 2;
}

// Ghost partners, searched with one warp per visible image G: a node of A can
// only reach G's cell window when A's clamped cell is within 2 cells of G's
// cell, and only when A's bounding sphere reaches G's SDF grid box. The lanes
// walk the occupants of those cells.
__global__ void k_ghost_candidates(StepArgs a, const int* __restrict__ g2_idx, const int* __restrict__ g2_off) {
  const int lane = threadIdx.x & 31;
  const int nvis = *a.G.count;
  const int n = a.P.n;
  const GridP& g = a.pg;
  int need = 0;  // largest per-particle image count seen by this lane
  for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < nvis; v += (gridDim.x * blockDim.x) >> 5) {
    const int t = a.G.list[v];
    const int s = t / n, i = t % n;
    const int gk = a.G.gkey[t];
    const double3 xg = a.G.gpos[t];
    const int cx = gk % g.size.x, cy = (gk / g.size.x) % g.size.y, cz = gk / (g.size.x * g.size.y);
    // circumradius of the image's SDF grid box about its centre
    double3 lo, hi;
    grid_box(a.P.origin[i], a.P.invh[i], a.S.gsize[a.P.shape[i]], lo, hi);
    const double3 far = d3(fmax(fabs(lo.x), fabs(hi.x)), fmax(fabs(lo.y), fabs(hi.y)), fmax(fabs(lo.z), fabs(hi.z)));
    const double Rg = len(far);
    const int pid = (i << 3) | s;
    // A candidate lies within rmax + Rg of the image, so its clamped cell lies in
    // the per-axis cell range of that ball (edge cells are open outward: they
    // also hold clamped bodies outside the domain), intersected with the 2-cell
    // window.
    const double reach = (a.rmax + Rg) * (1.0 + 1e-6) + coord_slack(xg, xg);
    const int x0 = axis_lo(xg.x, g.mn.x, g.inv.x, g.size.x, reach, cx), x1 = axis_hi(xg.x, g.mn.x, g.inv.x, g.size.x, reach, cx);
    const int y0 = axis_lo(xg.y, g.mn.y, g.inv.y, g.size.y, reach, cy), y1 = axis_hi(xg.y, g.mn.y, g.inv.y, g.size.y, reach, cy);
    const int z0 = axis_lo(xg.z, g.mn.z, g.inv.z, g.size.z, reach, cz), z1 = axis_hi(xg.z, g.mn.z, g.inv.z, g.size.z, reach, cz);
    const float3 xgf = make_float3((float)xg.x, (float)xg.y, (float)xg.z);
    const float Rgf = (float)Rg, n1g = fabsf(xgf.x) + fabsf(xgf.y) + fabsf(xgf.z);
    // separation test of the pair (owner A, image) along the line of centres, as for
    // particle pairs: a translated image has the particle's orientation, shape and scale
    // (turned sector images are not tested)
    const bool sep = a.S.sup_n != nullptr && !a.G.sector;
    const Quat qi = a.P.quat[i];
    const float4 qbf = make_float4((float)qi.q0, (float)qi.q1, (float)qi.q2, (float)qi.q3);
    const float4 pbf = make_float4(xgf.x, xgf.y, xgf.z, 0.f);
    const int shB = a.P.shape[i];
    const float scB = (float)a.P.scale[i];
    for (int z = z0; z <= z1; ++z) {
      for (int y = y0; y <= y1; ++y) {
        // the cells x0..x1 of a row are contiguous in the sorted order
        const int h0 = lin3(make_int3(x0, y, z), g.size);
        const int st = g2_off[h0 + 1], en = g2_off[h0 + (x1 - x0) + 2];
        {
          for (int k0 = st; k0 < en; k0 += 32) {
            const int k = k0 + lane;
            int slot = -1, A = 0;
            if (k < en) {
              // superset test on the FP32 copies (margin covers their rounding)
              const float4 pa = __ldg(a.cell_pk + k);
              const float dx = pa.x - xgf.x, dy = pa.y - xgf.y, dz = pa.z - xgf.z;
              const float R = (pa.w + Rgf) * (1.0f + 1e-5f) + 1e-6f * (n1g + fabsf(pa.x) + fabsf(pa.y) + fabsf(pa.z));
              bool cand = !(dx * dx + dy * dy + dz * dz > R * R);
              if (cand) A = __ldg(g2_idx + k);
              if (cand && sep) {
                const Quat qa = a.P.quat[A];
                const float4 qaf = make_float4((float)qa.q0, (float)qa.q1, (float)qa.q2, (float)qa.q3);
                const float n1a = __fadd_rn(__fadd_rn(fabsf(pa.x), fabsf(pa.y)), fabsf(pa.z));
                cand = !pair_separated(a, pa, n1a, qaf, (float)a.P.scale[A], a.P.shape[A], pbf, qbf, scB, shB);
              }
              if (cand) {
                slot = atomicAdd(&a.pgh.cnt[A], 1);
                if (slot < a.pgh.cap) a.pgh.id[(size_t)A * a.pgh.cap + slot] = pid;
                else atomicOr(&a.status->flags, OVF_GHOST);
              }
            }
            need = max(need, slot + 1);
            if (a.pl.ctr) {  // precision form: flat pair list
              const bool ok = slot >= 0 && slot < a.pgh.cap;
              const unsigned m = __ballot_sync(FULL, ok);
              int base = 0;
              if (lane == 0 && m) base = atomicAdd(&a.pl.ctr[2], __popc(m));
              base = __shfl_sync(FULL, base, 0);
              if (ok) a.pl.list[2][base + __popc(m & lanemask_lt())] = A * a.pgh.cap + slot;
            }
          }
        }
      }
    }
  }
  need = __reduce_max_sync(FULL, need);
  if (lane == 0 && need > 0) atomicMax(&a.status->need_ghost, need);
}

void launch_ghost_candidates(const StepArgs& a, const int* g2_idx, const int* g2_off, cudaStream_t s) {
  long long n = (long long)a.G.nsets * a.P.n;
  if (n <= 0) return;
  k_ghost_compact<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a);
  StepArgs g = a;
  g.pk_meta = nullptr;  // the particle records stay in the particle grid's order
  k_pack_cells<<<(a.P.n + 255) / 256, 256, 0, s>>>(g, g2_idx);  // the candidate walk's copy is spent
  int blocks = num_sms() * 16;
  k_ghost_candidates<<<blocks, 128, 0, s>>>(a, g2_idx, g2_off);
}

// ---------------------------------------------------------------------------
// V-bond forces, one thread per bond.
__global__ void k_bonds(StepArgs a, BondView b) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= b.n) return;
  double* st = b.state + 9 * (size_t)k;
  if (b.bonded[k] == 0) {
    for (int q = 0; q < 6; ++q) st[q] = 0.;
    return;
  }
  const int i = b.ids[2 * k], j = b.ids[2 * k + 1];
  const Quat qi = a.P.quat[i], qj = a.P.quat[j];
  const double3* fr = b.frames + 8 * (size_t)k;
  const double3 n1i = rotate(qi, fr[0]), n2i = rotate(qi, fr[1]), n3i = rotate(qi, fr[2]);
  const double3 n1j = rotate(qj, fr[4]), n2j = rotate(qj, fr[5]), n3j = rotate(qj, fr[6]);
  const double3 ri = a.P.pos[i], rj = a.P.pos[j];
  const double3 rbi = rotate(qi, fr[3]) + ri;
  const double3 rbj = rotate(qj, fr[7]) + rj;
  const double3 bp = 0.5 * (rbi + rbj);
  st[6] = bp.x; st[7] = bp.y; st[8] = bp.z;
  const double B1 = b.B[4 * k], B2 = b.B[4 * k + 1], B3 = b.B[4 * k + 2], B4 = b.B[4 * k + 3];
  const double Rb = b.geo[5 * k], D0 = b.geo[5 * k + 1], ten = b.geo[5 * k + 2], coh = b.geo[5 * k + 3],
               fmu = b.geo[5 * k + 4];
  double3 F = d3(0., 0., 0.), Mij = d3(0., 0., 0.), Mji = d3(0., 0., 0.);
  int ok = 1;
  const double3 rbij = rbi - rbj;
  const double D = len(rbij);
  if (!is_zero(D)) {
    const double3 nij = normalize_dev(rbij);
    const double3 e = -nij;
    st[0] = 0.5 * B1 * (D - D0) * (D - D0);
    st[1] = B2 * (0.5 * dot((n1j - n1i), e) - 0.25 * dot(n1i, n1j) + 0.75);
    st[2] = (0.25 * B2 + B3 + 0.5 * B4) * (dot(n1i, n1j) + 1.);
    st[3] = -0.5 * B4 * (dot(n1i, n1j) + dot(n2i, n2j) + dot(n3i, n3j) - 1);
    F = B1 * (D - D0) * e + B2 / (2 * D) * ((n1j - n1i) - dot((n1j - n1i), e) * e);
    const double3 MTB = B3 * cross(n1j, n1i) - 0.5 * B4 * (cross(n2j, n2i) + cross(n3j, n3i));
    Mij = -0.5 * B2 * cross(e, n1i) + MTB;
    Mji = 0.5 * B2 * cross(e, n1j) - MTB;
    const double fnb = dot(F, nij);
    const double3 fsb = F - fnb * nij;
    const double tt = dot(MTB, nij);
    const double3 tb = MTB - tt * nij;
    const double Ab = Rb * Rb * M_PI;
    const double Ib = Ab * Rb * Rb / 4.;
    const double Jb = 2 * Ib;
    st[4] = -fnb / Ab + len(tb) / Ib * Rb;
    st[5] = len(fsb) / Ab + fabs(tt) / Jb * Rb;
    if (ten > 0. && st[4] > ten) ok = 0;
    else if (coh > 0. && st[5] > coh - fmu * st[4]) ok = 0;
  }
  b.bonded[k] = ok;
  atomic_add3(a.P.force, i, F);
  atomic_add3(a.P.torque, i, Mij + cross(rbi - ri, F));
  atomic_add3(a.P.force, j, -F);
  atomic_add3(a.P.torque, j, Mji + cross(rbj - rj, -F));
}

void launch_bonds(const StepArgs& a, const BondView& b, cudaStream_t s) {
  if (b.n > 0) k_bonds<<<(b.n + 127) / 128, 128, 0, s>>>(a, b);
}

}  // namespace lsdem
