// Bonded workload (config 2: ellipsoids on an HCP lattice joined by V-bonds, a floor
// and a top wall moving down) written against the app-facing LSSolver API only, so
// the same source builds against the reference solver (FunDEM/kernel/LSSolver.h with
// its kernel sources) and against this repository's drop-in include/kernel/LSSolver.h.
//
//   c2_bench SCENE OUTDIR RESULT
//
// SCENE is the binary scene written by tests/test_fundem_same_gpu.py (one shape,
// particles added with a density, walls with a prescribed velocity, bonds); OUTDIR
// is an absolute output directory (the solver writes its frames there); RESULT
// receives the device time of steps (k0, k1] (CUDA events recorded on stream 0 from
// the external-force hook, which both solvers call every step between the forces and
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
double3 v3(const double* p) { return make_double3(p[0], p[1], p[2]); }

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
  if (!f || std::string(magic, 7) != "LSDEMC2") {
    std::fprintf(stderr, "bad scene file\n");
    return 2;
  }
  // shape
  const int nn = rd1<int32_t>(f), gx = rd1<int32_t>(f), gy = rd1<int32_t>(f), gz = rd1<int32_t>(f);
  const double h = rd1<double>(f);
  double o[3];
  rd(f, o, 3);
  const std::vector<double3> nodes = rd3(f, (size_t)nn);
  std::vector<double> sdf((size_t)gx * gy * gz);
  rd(f, sdf.data(), sdf.size());
  // particles
  const int np = rd1<int32_t>(f);
  const std::vector<double3> pos = rd3(f, (size_t)np);
  std::vector<double> q(4 * (size_t)np);
  rd(f, q.data(), q.size());
  const std::vector<double3> vel = rd3(f, (size_t)np);
  double mat[5];  // kn, ks, mu, e, density
  rd(f, mat, 5);
  // walls
  struct Wall {
    int size[3];
    double h, o[3], p[4 + 3], m[2], v[3];
    std::vector<double> sdf;
    std::vector<double3> verts;
    std::vector<int3> tris;
  };
  const int nw = rd1<int32_t>(f);
  std::vector<Wall> walls((size_t)nw);
  for (Wall& w : walls) {
    rd(f, w.size, 3);
    w.h = rd1<double>(f);
    rd(f, w.o, 3);
    w.sdf.resize((size_t)w.size[0] * w.size[1] * w.size[2]);
    rd(f, w.sdf.data(), w.sdf.size());
    rd(f, w.p, 7);  // position, quaternion
    rd(f, w.m, 2);  // mu, e
    rd(f, w.v, 3);  // fixed velocity
    const int nv = rd1<int32_t>(f), nt = rd1<int32_t>(f);
    w.verts = rd3(f, (size_t)nv);
    std::vector<int32_t> tri(3 * (size_t)nt);
    rd(f, tri.data(), tri.size());
    w.tris.resize((size_t)nt);
    for (int i = 0; i < nt; ++i) w.tris[i] = make_int3(tri[3 * i], tri[3 * i + 1], tri[3 * i + 2]);
  }
  // bonds
  const int nb = rd1<int32_t>(f);
  std::vector<int32_t> ids(2 * (size_t)nb);
  rd(f, ids.data(), ids.size());
  std::vector<double> bp(3 * (size_t)nb), bn(3 * (size_t)nb), br((size_t)nb), bl((size_t)nb), bt((size_t)nb),
      bc((size_t)nb);
  rd(f, bp.data(), bp.size());
  rd(f, bn.data(), bn.size());
  rd(f, br.data(), br.size());
  rd(f, bl.data(), bl.size());
  rd(f, bt.data(), bt.size());
  rd(f, bc.data(), bc.size());
  double bmat[3];  // Young's modulus, Poisson ratio, bond friction
  rd(f, bmat, 3);
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

  Bench s(argv[2], k0, k1);
  for (int i = 0; i < np; ++i)
    s.addLSParticle(nodes, sdf, make_double3(o[0], o[1], o[2]), make_int3(gx, gy, gz), h, pos[i], vel[i],
                    make_double3(0., 0., 0.), make_quaternion(q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]),
                    mat[0], mat[1], mat[2], mat[3], mat[4]);
  for (int k = 0; k < nw; ++k) {
    const Wall& w = walls[k];
    s.addWall(w.verts, w.tris, w.sdf, v3(w.o), make_int3(w.size[0], w.size[1], w.size[2]), w.h, v3(w.p),
              make_quaternion(w.p[3], w.p[4], w.p[5], w.p[6]), w.m[0], w.m[1]);
    if (w.v[0] != 0. || w.v[1] != 0. || w.v[2] != 0.) s.setFixedVelocityToWall(k, v3(w.v));
  }
  for (int b = 0; b < nb; ++b)
    s.addBondedInteraction(ids[2 * b], ids[2 * b + 1], v3(&bp[3 * (size_t)b]), v3(&bn[3 * (size_t)b]), br[b], bl[b],
                           bmat[0], bmat[1], bt[b], bc[b], bmat[2]);
  // numStep = floor(T / dt) + 1 and numStep + 1 steps: T = (nsteps - 1.5) dt gives nsteps steps
  s.solve(make_double3(dmin[0], dmin[1], dmin[2]), make_double3(dmax[0], dmax[1], dmax[2]),
          make_double3(g[0], g[1], g[2]), dt, (nsteps - 1.5) * dt, 1, argc, argv);
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
