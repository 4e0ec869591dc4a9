// Host-array driver around the reference solver's own CUDA launchers —
// TEST INFRASTRUCTURE ONLY (golden-vector generation).
//
// Built by oracle/build_ref.sh together with the reference's kernel sources,
// where they lie in the reference tree, into oracle/_ref/libfundem_ref.so.
// Each fref_* entry point uploads host arrays in the reference's own data
// layout (per-particle SDF copies addressed by an inclusive prefix sum, one
// node list with a particle id per node), calls the reference launcher(s)
// named in its comment, and copies the results back. Nothing here is part of
// the product path.
#include <cuda_runtime.h>
#include <cstdio>
#include <vector>
#include "CUDAKernelFunction/LSParticleContactDetectionKernel.cuh"
#include "CUDAKernelFunction/contactKernel.cuh"
#include "CUDAKernelFunction/particleIntegrationKernel.cuh"
#include "CUDAKernelFunction/myUtility/mySpatialGrid.h"
#include "CUDAKernelFunction/myUtility/buildHashStartEnd.h"

namespace {

struct Dev {
  std::vector<void*> ptrs;
  ~Dev() { for (void* p : ptrs) cudaFree(p); }
  template <class T> T* up(const T* h, size_t n) {
    T* d = nullptr;
    cudaMalloc(&d, (n ? n : 1) * sizeof(T));
    if (n && h) cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
    else cudaMemset(d, 0, (n ? n : 1) * sizeof(T));
    ptrs.push_back(d);
    return d;
  }
  template <class T> T* zeros(size_t n) { return up<T>(nullptr, n); }
};

template <class T> void down(T* h, const T* d, size_t n) {
  if (n) cudaMemcpy(h, d, n * sizeof(T), cudaMemcpyDeviceToHost);
}

inline double3 D3(const double* p) { return make_double3(p[0], p[1], p[2]); }
inline int3 I3(const int* p) { return make_int3(p[0], p[1], p[2]); }
inline size_t blk(size_t n) { return n < 256 ? (n ? n : 1) : 256; }
inline size_t grd(size_t n) { size_t b = blk(n); return (n + b - 1) / b; }

int finish() {
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { fprintf(stderr, "fref: %s\n", cudaGetErrorString(e)); return 1; }
  return 0;
}

}  // namespace

extern "C" {

// launchUpdateSpatialGridHashStartEnd (ghost=0) or
// launchUpdateGhostSpatialGridHashStartEnd (ghost=1).
int fref_hash_sort(int ghost, int n, const double* pos, const double* mn, const double* mx, const double* inv,
                   const int* size, int ncells, int* key, int* idx, int* start, int* end) {
  Dev d;
  double3* dp = d.up((const double3*)pos, n);
  int* dk = d.zeros<int>(n);
  int* di = d.zeros<int>(n);
  int* ds = d.zeros<int>(ncells);
  int* de = d.zeros<int>(ncells);
  if (ghost)
    launchUpdateGhostSpatialGridHashStartEnd(di, dk, dp, ds, de, D3(mn), D3(mx), D3(inv), I3(size), ncells, n, grd(n),
                                             blk(n), 0);
  else
    launchUpdateSpatialGridHashStartEnd(di, dk, dp, ds, de, D3(mn), D3(mx), D3(inv), I3(size), ncells, n, grd(n),
                                        blk(n), 0);
  if (finish()) return 1;
  down(key, dk, n); down(idx, di, n); down(start, ds, ncells); down(end, de, ncells);
  return 0;
}

// Narrowphase count + inclusive scan + write, mode 0:
// launchBuildLevelSetBoundaryNodeInteractions1st/2nd (particle-particle),
// mode 1: launchBuildLevelSetBoundaryNodeFixedParticleInteractions1st/2nd (walls, ghosts).
// bodies: SDF side (for mode 0 the particles themselves). prefix_b is the
// inclusive SDF prefix sum per body. The caller provides the previous
// step's prefix sum and contact partner/spring arrays (may be empty).
int fref_detect(int mode, int nn, const double* node_local, const int* node_pid, int np, const double* ppos,
                const double* pquat, int nb, const double* bpos, const double* bquat, const double* brad,
                const double* binvh, const double* borigin, const int* bsize, const int* bprefix, long long nsdf,
                const double* sdf, const double* mn, const double* inv, const int* size, int ncells, const int* hidx,
                const int* hstart, const int* hend, const int* prefix_old, int nold, const int* partner_old,
                const double* spring_old, int cap, int* count, int* prefix, int* ncontact, double* spring,
                double* point, double* normal, double* overlap, int* node_out, int* partner_out) {
  Dev d;
  double3* dnl = d.up((const double3*)node_local, nn);
  int* dnp = d.up(node_pid, nn);
  double3* dpp = d.up((const double3*)ppos, np);
  quaternion* dpq = d.up((const quaternion*)pquat, np);
  double3* dbp = d.up((const double3*)bpos, nb);
  quaternion* dbq = d.up((const quaternion*)bquat, nb);
  double* dbr = d.up(brad, nb);
  double* dbi = d.up(binvh, nb);
  double3* dbo = d.up((const double3*)borigin, nb);
  int3* dbs = d.up((const int3*)bsize, nb);
  int* dbx = d.up(bprefix, nb);
  double* dsdf = d.up(sdf, (size_t)nsdf);
  int* dhi = d.up(hidx, nb);
  int* dhs = d.up(hstart, ncells);
  int* dhe = d.up(hend, ncells);
  int* dpo = d.up(prefix_old, nn);
  int* dpa_old = d.up(partner_old, nold);
  double3* dsp_old = d.up((const double3*)spring_old, nold);
  int* dcnt = d.zeros<int>(nn);
  int* dpre = d.zeros<int>(nn);
  if (mode == 0)
    launchBuildLevelSetBoundaryNodeInteractions1st(dcnt, dnl, dnp, dsdf, dpp, dpq, dbr, dbi, dbo, dbs, dbx, dhi, dhs,
                                                   dhe, D3(mn), D3(inv), I3(size), nn, grd(nn), blk(nn), 0);
  else
    launchBuildLevelSetBoundaryNodeFixedParticleInteractions1st(dcnt, dnl, dnp, dsdf, dpp, dpq, dbp, dbq, dbi, dbo,
                                                                dbs, dbx, dhi, dhs, dhe, D3(mn), D3(inv), I3(size), nn,
                                                                grd(nn), blk(nn), 0);
  buildPrefixSum(dpre, dcnt, nn, 0);
  if (finish()) return 1;
  down(count, dcnt, nn);
  down(prefix, dpre, nn);
  const int nc = nn ? prefix[nn - 1] : 0;
  *ncontact = nc;
  if (nc > cap) return 2;
  double3* dsp = d.zeros<double3>(nc);
  double3* dpt = d.zeros<double3>(nc);
  double3* dnm = d.zeros<double3>(nc);
  double* dov = d.zeros<double>(nc);
  int* dno = d.zeros<int>(nc);
  int* dpa = d.zeros<int>(nc);
  if (mode == 0)
    launchBuildLevelSetBoundaryNodeInteractions2nd(dsp, dpt, dnm, dov, dno, dpa, dsp_old, dpa_old, dnl, dnp, dpre, dpo,
                                                   dsdf, dpp, dpq, dbr, dbi, dbo, dbs, dbx, dhi, dhs, dhe, D3(mn),
                                                   D3(inv), I3(size), nn, grd(nn), blk(nn), 0);
  else
    launchBuildLevelSetBoundaryNodeFixedParticleInteractions2nd(dsp, dpt, dnm, dov, dno, dpa, dsp_old, dpa_old, dnl,
                                                                dnp, dpre, dpo, dsdf, dpp, dpq, dbp, dbq, dbi, dbo, dbs,
                                                                dbx, dhi, dhs, dhe, D3(mn), D3(inv), I3(size), nn,
                                                                grd(nn), blk(nn), 0);
  if (finish()) return 1;
  down((double3*)spring, dsp, nc); down((double3*)point, dpt, nc); down((double3*)normal, dnm, nc);
  down(overlap, dov, nc); down(node_out, dno, nc); down(partner_out, dpa, nc);
  return 0;
}

// kind 0: launchAddLevelSetParticleContactForceTorque, 1: launchAddFixedLevelSetParticleContactForceTorque,
// 2: launchAddGhostLevelSetParticleContactForceTorque. jpos/jvel/jangvel/jmu/jres describe the partner
// set (walls, or ghost images with the real particles' parameters). force/torque are in/out.
int fref_force(int kind, int nc, double* spring, double* en_n, double* en_s, const double* point, const double* normal,
               const double* overlap, const int* node, const int* partner, int nn, const int* node_pid, int np,
               const double* pos, const double* vel, const double* angvel, const double* invm, const double* kn,
               const double* ks, const double* mu, const double* res, int nj, const double* jpos, const double* jvel,
               const double* jangvel, const double* jmu, const double* jres, double dt, double* force,
               double* torque) {
  Dev d;
  double3* dsp = d.up((const double3*)spring, nc);
  double* den = d.zeros<double>(nc);
  double* des = d.zeros<double>(nc);
  double3* dpt = d.up((const double3*)point, nc);
  double3* dnm = d.up((const double3*)normal, nc);
  double* dov = d.up(overlap, nc);
  int* dno = d.up(node, nc);
  int* dpa = d.up(partner, nc);
  int* dnp = d.up(node_pid, nn);
  double3* dF = d.up((const double3*)force, np);
  double3* dT = d.up((const double3*)torque, np);
  double3* dp = d.up((const double3*)pos, np);
  double3* dv = d.up((const double3*)vel, np);
  double3* dw = d.up((const double3*)angvel, np);
  double* dim = d.up(invm, np);
  double* dkn = d.up(kn, np);
  double* dks = d.up(ks, np);
  double* dmu = d.up(mu, np);
  double* dre = d.up(res, np);
  if (nc > 0) {
    if (kind == 0) {
      launchAddLevelSetParticleContactForceTorque(dsp, den, des, dpt, dnm, dov, dno, dpa, dnp, dF, dT, dp, dv, dw, dim,
                                                  dkn, dks, dmu, dre, dt, nc, grd(nc), blk(nc), 0);
    } else if (kind == 1) {
      double3* djp = d.up((const double3*)jpos, nj);
      double3* djv = d.up((const double3*)jvel, nj);
      double3* djw = d.up((const double3*)jangvel, nj);
      double* djm = d.up(jmu, nj);
      double* djr = d.up(jres, nj);
      launchAddFixedLevelSetParticleContactForceTorque(dsp, den, des, dpt, dnm, dov, dno, dpa, dnp, dF, dT, dp, dv, dw,
                                                       dim, dkn, dks, dmu, dre, djp, djv, djw, djm, djr, dt, nc,
                                                       grd(nc), blk(nc), 0);
    } else {
      double3* djp = d.up((const double3*)jpos, nj);
      double3* djv = d.up((const double3*)jvel, nj);
      launchAddGhostLevelSetParticleContactForceTorque(dsp, den, des, dpt, dnm, dov, dno, dpa, dnp, dF, dT, dp, dv,
                                                       dw, dim, dkn, dks, dmu, dre, djp, djv, dt, nc, grd(nc),
                                                       blk(nc), 0);
    }
  }
  if (finish()) return 1;
  down((double3*)spring, dsp, nc); down(en_n, den, nc); down(en_s, des, nc);
  down((double3*)force, dF, np); down((double3*)torque, dT, np);
  return 0;
}

// launchAddBondedForceTorque. frames: per bond master n1,n2,n3,pos then slave n1,n2,n3,pos (24 doubles).
// geo: per bond radius, L0, tensile, cohesion, mu. Bk: B1..B4. state out: Un,Us,Ub,Ut,sigma,tau,point(3).
int fref_bond(int nb, const int* ids, const double* Bk, const double* geo, const double* frames, int* bonded,
              double* state, int np, const double* pos, const double* quat, double* force, double* torque) {
  std::vector<double> B[4], g[5];
  std::vector<double3> fr[8];
  std::vector<int> mi(nb), si(nb);
  for (int k = 0; k < nb; ++k) {
    for (int a = 0; a < 4; ++a) B[a].push_back(Bk[4 * k + a]);
    for (int a = 0; a < 5; ++a) g[a].push_back(geo[5 * k + a]);
    for (int a = 0; a < 8; ++a) fr[a].push_back(D3(frames + 24 * k + 3 * a));
    mi[k] = ids[2 * k];
    si[k] = ids[2 * k + 1];
  }
  Dev d;
  double3* dpt = d.zeros<double3>(nb);
  double* ds[6];
  for (int a = 0; a < 6; ++a) {
    std::vector<double> h(nb);
    for (int k = 0; k < nb; ++k) h[k] = state[9 * k + a];
    ds[a] = d.up(h.data(), nb);
  }
  int* dbd = d.up(bonded, nb);
  double* dB[4];
  for (int a = 0; a < 4; ++a) dB[a] = d.up(B[a].data(), nb);
  double* dg[5];
  for (int a = 0; a < 5; ++a) dg[a] = d.up(g[a].data(), nb);
  double3* dfr[8];
  for (int a = 0; a < 8; ++a) dfr[a] = d.up(fr[a].data(), nb);
  int* dmi = d.up(mi.data(), nb);
  int* dsi = d.up(si.data(), nb);
  double3* dF = d.up((const double3*)force, np);
  double3* dT = d.up((const double3*)torque, np);
  double3* dp = d.up((const double3*)pos, np);
  quaternion* dq = d.up((const quaternion*)quat, np);
  launchAddBondedForceTorque(dpt, ds[4], ds[5], ds[0], ds[1], ds[2], ds[3], dbd, dB[0], dB[1], dB[2], dB[3], dg[0],
                             dg[1], dg[2], dg[3], dg[4], dfr[0], dfr[1], dfr[2], dfr[3], dfr[4], dfr[5], dfr[6],
                             dfr[7], dmi, dsi, dF, dT, dp, dq, nb, grd(nb), blk(nb), 0);
  if (finish()) return 1;
  std::vector<double3> hp(nb);
  down(hp.data(), dpt, nb);
  for (int a = 0; a < 6; ++a) {
    std::vector<double> h(nb);
    down(h.data(), ds[a], nb);
    for (int k = 0; k < nb; ++k) state[9 * k + a] = h[k];
  }
  for (int k = 0; k < nb; ++k) { state[9 * k + 6] = hp[k].x; state[9 * k + 7] = hp[k].y; state[9 * k + 8] = hp[k].z; }
  down(bonded, dbd, nb);
  down((double3*)force, dF, np); down((double3*)torque, dT, np);
  return 0;
}

// launchParticleVelocityAngularVelocityIntegration (half kick h).
int fref_kick(int n, double* vel, double* angvel, const double* force, const double* torque, const double* invm,
              const double* quat, const double* invI, const double* g, double h) {
  Dev d;
  double3* dv = d.up((const double3*)vel, n);
  double3* dw = d.up((const double3*)angvel, n);
  double3* dF = d.up((const double3*)force, n);
  double3* dT = d.up((const double3*)torque, n);
  double* dim = d.up(invm, n);
  quaternion* dq = d.up((const quaternion*)quat, n);
  symMatrix* dI = d.up((const symMatrix*)invI, n);
  launchParticleVelocityAngularVelocityIntegration(dv, dw, dF, dT, dim, dq, dI, D3(g), h, n, grd(n), blk(n), 0);
  if (finish()) return 1;
  down((double3*)vel, dv, n); down((double3*)angvel, dw, n);
  return 0;
}

// launchParticlePositionOrientationIntegration.
int fref_drift(int n, double* pos, double* quat, const double* vel, const double* angvel, double dt) {
  Dev d;
  double3* dp = d.up((const double3*)pos, n);
  quaternion* dq = d.up((const quaternion*)quat, n);
  double3* dv = d.up((const double3*)vel, n);
  double3* dw = d.up((const double3*)angvel, n);
  launchParticlePositionOrientationIntegration(dp, dq, dv, dw, dt, n, grd(n), blk(n), 0);
  if (finish()) return 1;
  down((double3*)pos, dp, n); down((quaternion*)quat, dq, n);
  return 0;
}

// launchUpdatePositionOutOfBoundary{XD,YD} (axis 0/1).
int fref_wrap(int n, double* pos, const double* mn, const double* mx, int axis) {
  Dev d;
  double3* dp = d.up((const double3*)pos, n);
  if (axis == 0) launchUpdatePositionOutOfBoundaryXD(dp, D3(mn), D3(mx), n, grd(n), blk(n), 0);
  else launchUpdatePositionOutOfBoundaryYD(dp, D3(mn), D3(mx), n, grd(n), blk(n), 0);
  if (finish()) return 1;
  down((double3*)pos, dp, n);
  return 0;
}

// launchCalculateGhostPosition{XD,YD,XYD} (mask 1, 2, 3).
int fref_ghost_pos(int n, const double* pos, const double* mn, const double* mx, const double* inv, const int* size,
                   int mask, double* gpos) {
  Dev d;
  double3* dp = d.up((const double3*)pos, n);
  double3* dg = d.zeros<double3>(n);
  if (mask == 1) launchCalculateGhostPositionXD(dg, dp, D3(mn), D3(mx), D3(inv), I3(size), n, grd(n), blk(n), 0);
  else if (mask == 2) launchCalculateGhostPositionYD(dg, dp, D3(mn), D3(mx), D3(inv), I3(size), n, grd(n), blk(n), 0);
  else launchCalculateGhostPositionXYD(dg, dp, D3(mn), D3(mx), D3(inv), I3(size), n, grd(n), blk(n), 0);
  if (finish()) return 1;
  down((double3*)gpos, dg, n);
  return 0;
}

}  // extern "C"
