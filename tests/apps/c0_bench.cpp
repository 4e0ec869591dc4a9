// Config-0 workload (identical ellipsoids above a floor wall) written against the
// app-facing LSSolver API only, so the same source builds against the reference
// solver (FunDEM/kernel/LSSolver.h with its kernel sources) and against this
// repository's drop-in include/kernel/LSSolver.h.
//
//   c0_bench SCENE OUTDIR RESULT
//
// SCENE is the binary scene written by tests/test_fundem_same_gpu.py; OUTDIR is an
// absolute output directory (the solver writes its frames there); RESULT receives
// the device time of steps (k0, k1] (CUDA events recorded on stream 0 from the
// external-force hook, which both solvers call every step between the forces and
// the second half kick) and the particle velocities at step k1.
#include "kernel/LSSolver.h"

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

namespace {

template <class T>
void rd(std::ifstream& f, T* p, size_t n) {
  f.read(reinterpret_cast<char*>(p), (std::streamsize)(n * sizeof(T)));
}
template <class T>
T rd1(std::ifstream& f) {
  T v;
  rd(f, &v, 1);
  return v;
}
std::vector<double3> rd3(std::ifstream& f, size_t n) {
  std::vector<double> a(3 * n);
  rd(f, a.data(), a.size());
  std::vector<double3> out(n);
  for (size_t i = 0; i < n; ++i) out[i] = make_double3(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
  return out;
}

class Bench : public LSSolver {
 public:
  Bench(const std::string& dir, int k0, int k1) : LSSolver(dir), k0_(k0), k1_(k1) {
    cudaEventCreate(&a_);
    cudaEventCreate(&b_);
  }
  int k0_, k1_, k_ = 0;
  cudaEvent_t a_, b_;
  std::vector<double3> vel_;

 protected:
  void addExternalForceTorque(const double) override {
    ++k_;
    if (k_ == k0_) cudaEventRecord(a_, 0);
    if (k_ == k1_) {
      cudaEventRecord(b_, 0);
      const int n = (int)getLSParticle().num_device();
      vel_.resize(n);
      cudaMemcpy(vel_.data(), getLSParticle().velocity(), sizeof(double3) * n, cudaMemcpyDeviceToHost);
    }
  }
};

}  // namespace

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s SCENE OUTDIR RESULT\n", argv[0]);
    return 2;
  }
  std::ifstream f(argv[1], std::ios::binary);
  char magic[8];
  f.read(magic, 8);
  if (!f || std::string(magic, 7) != "LSDEMC0") {
    std::fprintf(stderr, "bad scene file\n");
    return 2;
  }
  const int nn = rd1<int32_t>(f), gx = rd1<int32_t>(f), gy = rd1<int32_t>(f), gz = rd1<int32_t>(f);
  const int np = rd1<int32_t>(f);
  const double h = rd1<double>(f);
  double o[3];
  rd(f, o, 3);
  const std::vector<double3> nodes = rd3(f, (size_t)nn);
  std::vector<double> sdf((size_t)gx * gy * gz);
  rd(f, sdf.data(), sdf.size());
  const std::vector<double3> pos = rd3(f, (size_t)np);
  std::vector<double> q(4 * (size_t)np);
  rd(f, q.data(), q.size());
  const std::vector<double3> vel = rd3(f, (size_t)np);
  double mat[5];  // kn, ks, mu, e, density
  rd(f, mat, 5);
  const int wx = rd1<int32_t>(f), wy = rd1<int32_t>(f), wz = rd1<int32_t>(f);
  const double wh = rd1<double>(f);
  double wo[3], wp[3], wq[4], wm[2];
  rd(f, wo, 3);
  std::vector<double> wsdf((size_t)wx * wy * wz);
  rd(f, wsdf.data(), wsdf.size());
  rd(f, wp, 3);
  rd(f, wq, 4);
  rd(f, wm, 2);
  const int nv = rd1<int32_t>(f), nt = rd1<int32_t>(f);
  const std::vector<double3> verts = rd3(f, (size_t)nv);
  std::vector<int32_t> tri(3 * (size_t)nt);
  rd(f, tri.data(), tri.size());
  std::vector<int3> tris((size_t)nt);
  for (int i = 0; i < nt; ++i) tris[i] = make_int3(tri[3 * i], tri[3 * i + 1], tri[3 * i + 2]);
  double dt, dmin[3], dmax[3], g[3];
  dt = rd1<double>(f);
  rd(f, dmin, 3);
  rd(f, dmax, 3);
  rd(f, g, 3);
  const int nsteps = rd1<int32_t>(f), k0 = rd1<int32_t>(f), k1 = rd1<int32_t>(f);
  if (!f) {
    std::fprintf(stderr, "truncated scene file\n");
    return 2;
  }
  // optional second phase: its step count and the floor's angular velocity about z
  // (set between the phases with setFixedAngularVelocityToWall, as tutorial 2 does)
  int32_t nsteps2 = 0;
  double floor_w = 0.;
  f.read(reinterpret_cast<char*>(&nsteps2), 4);
  if (f) f.read(reinterpret_cast<char*>(&floor_w), 8);
  if (!f) nsteps2 = 0;

  Bench s(argv[2], k0, k1);
  for (int i = 0; i < np; ++i)
    s.addLSParticle(nodes, sdf, make_double3(o[0], o[1], o[2]), make_int3(gx, gy, gz), h, pos[i], vel[i],
                    make_double3(0., 0., 0.), make_quaternion(q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]),
                    mat[0], mat[1], mat[2], mat[3], mat[4]);
  s.addWall(verts, tris, wsdf, make_double3(wo[0], wo[1], wo[2]), make_int3(wx, wy, wz), wh,
            make_double3(wp[0], wp[1], wp[2]), make_quaternion(wq[0], wq[1], wq[2], wq[3]), wm[0], wm[1]);
  // numStep = floor(T / dt) + 1 and numStep + 1 steps: T = (nsteps - 1.5) dt gives nsteps steps
  s.solve(make_double3(dmin[0], dmin[1], dmin[2]), make_double3(dmax[0], dmax[1], dmax[2]),
          make_double3(g[0], g[1], g[2]), dt, (nsteps - 1.5) * dt, 1, argc, argv);
  if (nsteps2 > 0) {
    s.setFixedAngularVelocityToWall(0, make_double3(0., 0., floor_w));
    s.solve(make_double3(dmin[0], dmin[1], dmin[2]), make_double3(dmax[0], dmax[1], dmax[2]),
            make_double3(g[0], g[1], g[2]), dt, (nsteps2 - 1.5) * dt, 1, argc, argv);
  }
  cudaDeviceSynchronize();
  float ms = -1.f;
  if (s.k_ >= k1) cudaEventElapsedTime(&ms, s.a_, s.b_);
  std::ofstream r(argv[3], std::ios::binary);
  const int32_t hdr[3] = {s.k_, k1 - k0, (int32_t)s.vel_.size()};
  r.write(reinterpret_cast<const char*>(hdr), sizeof(hdr));
  const double msd = ms;
  r.write(reinterpret_cast<const char*>(&msd), sizeof(msd));
  r.write(reinterpret_cast<const char*>(s.vel_.data()), (std::streamsize)(sizeof(double3) * s.vel_.size()));
  std::printf("steps %d window %d ms %.6f ms_per_step %.6f\n", s.k_, k1 - k0, ms, ms / (k1 - k0));
  return 0;
}
