// Bonds from the recorded particle-particle contacts, built on the device
// (LSSolver::createBondsFromContacts, LSSolver.h:385-418, over VBondedInteraction::add,
// VBondedInteraction.h:74-195): one bond per contact, owner -> partner, in the order of
// the contact list (owner particle, candidate slot, node), with the bond's local frames
// and points computed from the particles' current pose. The file is compiled without
// fused multiply-add contraction and every expression keeps the operation order of the
// host routine that adds one bond (add_bond_impl), so each bond is bit-identical to the
// one that routine would add for the same contact.
#include "kernels.h"

namespace lsdem {
namespace {

struct H3 { double x, y, z; };
__device__ __forceinline__ H3 h3(double3 v) { return H3{v.x, v.y, v.z}; }
__device__ __forceinline__ H3 hcross(H3 a, H3 b) {
  return H3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// rotation of v by q (scalar first), the host's t = 2 (qv x v), v + q0 t + qv x t
__device__ __forceinline__ H3 hrot(const double q[4], H3 v) {
  const H3 qv{q[1], q[2], q[3]};
  H3 t = hcross(qv, v);
  t = H3{t.x * 2.0, t.y * 2.0, t.z * 2.0};
  const H3 u = hcross(qv, t);
  const H3 a{v.x + t.x * q[0], v.y + t.y * q[0], v.z + t.z * q[0]};
  return H3{a.x + u.x, a.y + u.y, a.z + u.z};
}
__device__ __forceinline__ H3 hrot_inv(H3 v, Quat q) {
  const double c[4] = {q.q0, -q.q1, -q.q2, -q.q3};
  return hrot(c, v);
}
__device__ __forceinline__ H3 hnorm(H3 v) {
  const double l2 = v.x * v.x + v.y * v.y + v.z * v.z;
  if (fabs(l2) <= 1.0e-20) return H3{0., 0., 0.};
  const double inv = 1.0 / sqrt(l2);
  return H3{v.x * inv, v.y * inv, v.z * inv};
}

// Contacts per owner particle (sum of its slots' segment lengths).
__global__ void k_bond_count(SlotView pp, int n, int* __restrict__ cnt) {
  const int A = blockIdx.x * blockDim.x + threadIdx.x;
  if (A >= n) return;
  const int m = min(pp.cnt[A], pp.cap);
  int c = 0;
  for (int j = 0; j < m; ++j) c += pp.seg_cnt[(size_t)A * pp.cap + j];
  cnt[A] = c;
}

// One thread per owner particle: its contacts in slot, then node order, each a bond at
// offs[A] + k. frames: master n1, n2, n3, local point, slave n1, n2, n3, local point.
__global__ void k_bond_make(SlotView pp, int n, const int* __restrict__ offs, const double3* __restrict__ point,
                            const double3* __restrict__ normal, const double3* __restrict__ pos,
                            const Quat* __restrict__ quat, double Lb, int* __restrict__ ids, double3* __restrict__ frames,
                            double3* __restrict__ bpoint, int* __restrict__ bad) {
  const int A = blockIdx.x * blockDim.x + threadIdx.x;
  if (A >= n) return;
  const int m = min(pp.cnt[A], pp.cap);
  int out = offs[A];
  const H3 pi = h3(pos[A]);
  const Quat qi = quat[A];
  for (int j = 0; j < m; ++j) {
    const size_t sl = (size_t)A * pp.cap + j;
    const int B = pp.id[sl];
    const H3 pj = h3(pos[B]);
    const Quat qj = quat[B];
    const int c0 = pp.seg_start[sl], nc = pp.seg_cnt[sl];
    for (int k = 0; k < nc; ++k, ++out) {
      const H3 gn = h3(normal[c0 + k]);
      if (fabs(gn.x * gn.x + gn.y * gn.y + gn.z * gn.z) <= 1.0e-20) atomicOr(bad, 1);
      const double inv_len = 1.0 / sqrt(gn.x * gn.x + gn.y * gn.y + gn.z * gn.z);
      const H3 nv{gn.x * inv_len, gn.y * inv_len, gn.z * inv_len};
      const H3 c = h3(point[c0 + k]);
      const H3 gpi{c.x + 0.5 * Lb * nv.x, c.y + 0.5 * Lb * nv.y, c.z + 0.5 * Lb * nv.z};
      const H3 gpj{c.x - 0.5 * Lb * nv.x, c.y - 0.5 * Lb * nv.y, c.z - 0.5 * Lb * nv.z};
      const H3 lpi = hrot_inv(H3{gpi.x - pi.x, gpi.y - pi.y, gpi.z - pi.z}, qi);
      const H3 lpj = hrot_inv(H3{gpj.x - pj.x, gpj.y - pj.y, gpj.z - pj.z}, qj);
      const H3 n1i{-nv.x, -nv.y, -nv.z};
      const H3 ref = (fabs(n1i.x) < 0.9) ? H3{1., 0., 0.} : H3{0., 1., 0.};
      const H3 n2i = hnorm(hcross(ref, n1i));
      const H3 n3i = hnorm(hcross(n1i, n2i));
      const H3 n1j{-n1i.x, -n1i.y, -n1i.z};
      const H3 loc[8] = {hnorm(hrot_inv(n1i, qi)), hnorm(hrot_inv(n2i, qi)), hnorm(hrot_inv(n3i, qi)), lpi,
                         hnorm(hrot_inv(n1j, qj)), hnorm(hrot_inv(n2i, qj)), hnorm(hrot_inv(n3i, qj)), lpj};
      ids[2 * (size_t)out] = A;
      ids[2 * (size_t)out + 1] = B;
      for (int f = 0; f < 8; ++f) frames[8 * (size_t)out + f] = make_double3(loc[f].x, loc[f].y, loc[f].z);
      bpoint[out] = make_double3(c.x, c.y, c.z);
    }
  }
}

}  // namespace

void bonds_from_contacts_count(const SlotView& pp, int n, int* cnt, cudaStream_t s) {
  if (n > 0) k_bond_count<<<(n + 255) / 256, 256, 0, s>>>(pp, n, cnt);
}

void bonds_from_contacts_make(const SlotView& pp, int n, const int* offs, const double3* point, const double3* normal,
                              const double3* pos, const Quat* quat, double Lb, int* ids, double3* frames,
                              double3* bpoint, int* bad, cudaStream_t s) {
  if (n > 0)
    k_bond_make<<<(n + 127) / 128, 128, 0, s>>>(pp, n, offs, point, normal, pos, quat, Lb, ids, frames, bpoint, bad);
}

}  // namespace lsdem
