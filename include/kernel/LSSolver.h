// Drop-in app-facing solver: the class, constructor, methods and protected
// hooks of the reference's LSSolver (FunDEM/kernel/LSSolver.h:11-518), built
// on the lsdem_b200 C ABI. Apps written for the reference (a subclass that
// overrides addExternalForceTorque and launches kernels on
// getLSParticle().force() etc.) compile against this header unchanged.
//
// Output: each frame writes the reference's VTU files (surface-node mesh and
// particle centres, contacts, bonds, walls, wall contacts) under <dir>_phase<k>/,
// produced on the GPU by lsdem_write_vtu.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../lsdem_b200.h"
#include "CUDAKernelFunction/myUtility/myMat.h"

// Device view of a body set, as handed to external-force kernels
// (the device getters of the reference's LSParticle, LSParticle.h:660-685).
class LSParticle {
 public:
  double3* position() { return (double3*)pos_; }
  double3* velocity() { return (double3*)vel_; }
  double3* angularVelocity() { return (double3*)angvel_; }
  double3* force() { return (double3*)force_; }
  double3* torque() { return (double3*)torque_; }
  quaternion* orientation() { return (quaternion*)quat_; }
  size_t num() const { return n_; }
  size_t num_device() const { return n_; }
  const size_t& gridDim() const { return grid_; }
  const size_t& blockDim() const { return block_; }

 private:
  friend class LSSolver;
  void* pos_ = nullptr;
  void* vel_ = nullptr;
  void* angvel_ = nullptr;
  void* force_ = nullptr;
  void* torque_ = nullptr;
  void* quat_ = nullptr;
  size_t n_ = 0, grid_ = 1, block_ = 1;
};

class LSSolver {
 public:
  LSSolver(const std::string dir = "Problem", cudaStream_t stream = 0, const size_t maxGPUThread = 256,
           const int device = 0)
      : dir_(dir), stream_(stream), maxGPUThread_(maxGPUThread), device_(device) {
    if (lsdem_create(device, (void*)stream, &h_) != LSDEM_OK) h_ = nullptr;
  }
  virtual ~LSSolver() { lsdem_destroy(h_); }
  LSSolver(const LSSolver&) = delete;
  LSSolver& operator=(const LSSolver&) = delete;

  // Density overload: mass, centroid and inertia from the SDF (LSSolver.h:51-163).
  void addLSParticle(const std::vector<double3>& boundaryNodeLocalPosition,
                     const std::vector<double>& gridNodeSignedDistance, const double3 gridNodeLocalOrigin,
                     const int3 gridNodeSize, const double gridNodeSpacing, const double3 position,
                     const double3 velocity, const double3 angularVelocity, const quaternion orientation,
                     const double normalStiffness, const double shearStiffness, const double frictionCoefficient,
                     const double restitutionCoefficient, const double density,
                     const std::vector<int3>& boundaryNodeConnectivity = {}) {
    const int sz[3] = {gridNodeSize.x, gridNodeSize.y, gridNodeSize.z};
    const double o[3] = {gridNodeLocalOrigin.x, gridNodeLocalOrigin.y, gridNodeLocalOrigin.z};
    const double p[3] = {position.x, position.y, position.z};
    const double v[3] = {velocity.x, velocity.y, velocity.z};
    const double w[3] = {angularVelocity.x, angularVelocity.y, angularVelocity.z};
    const double q[4] = {orientation.q0, orientation.q1, orientation.q2, orientation.q3};
    int index = -1;
    if (report(lsdem_add_ls_particle(h_, (const double*)boundaryNodeLocalPosition.data(),
                                     (int)boundaryNodeLocalPosition.size(), gridNodeSignedDistance.data(), sz, o,
                                     gridNodeSpacing, p, v, w, q, normalStiffness, shearStiffness, frictionCoefficient,
                                     restitutionCoefficient, density, &index),
               "[LSParticle] "))
      return;
    setTriangles(0, index, boundaryNodeConnectivity);
  }

  // Explicit mass and inertia overload (LSSolver.h:190-223).
  void addLSParticle(const std::vector<double3>& boundaryNodeLocalPosition,
                     const std::vector<double>& gridNodeSignedDistance, const double3 gridNodeLocalOrigin,
                     const int3 gridNodeSize, const double gridNodeSpacing, const double3 position,
                     const double3 velocity, const double3 angularVelocity, const quaternion orientation,
                     const double mass, const symMatrix inertiaTensor, const double normalStiffness,
                     const double shearStiffness, const double frictionCoefficient,
                     const double restitutionCoefficient, const std::vector<int3>& boundaryNodeConnectivity = {}) {
    const int sz[3] = {gridNodeSize.x, gridNodeSize.y, gridNodeSize.z};
    const double o[3] = {gridNodeLocalOrigin.x, gridNodeLocalOrigin.y, gridNodeLocalOrigin.z};
    int shape = -1;
    if (report(lsdem_add_shape(h_, (const double*)boundaryNodeLocalPosition.data(),
                               (int)boundaryNodeLocalPosition.size(), gridNodeSignedDistance.data(), sz, o,
                               gridNodeSpacing, &shape),
               "[LSParticle] "))
      return;
    const symMatrix inv = mass > 0. ? inverse(inertiaTensor) : make_symMatrix(0., 0., 0., 0., 0., 0.);
    const double invm = mass > 0. ? 1. / mass : 0.;
    const double I6[6] = {inv.xx, inv.yy, inv.zz, inv.xy, inv.xz, inv.yz};
    const double p[3] = {position.x, position.y, position.z};
    const double v[3] = {velocity.x, velocity.y, velocity.z};
    const double w[3] = {angularVelocity.x, angularVelocity.y, angularVelocity.z};
    const double q[4] = {orientation.q0, orientation.q1, orientation.q2, orientation.q3};
    int index = -1;
    if (report(lsdem_add_particles(h_, 1, &shape, nullptr, p, v, w, q, &invm, I6, &normalStiffness, &shearStiffness,
                                   &frictionCoefficient, &restitutionCoefficient, &index),
               "[LSParticle] "))
      return;
    setTriangles(0, index, boundaryNodeConnectivity);
  }

  // Fixed level-set wall (LSSolver.h:245-272).
  void addWall(const std::vector<double3>& objVertexLocalPosition, const std::vector<int3>& objTriangleVertexID,
               const std::vector<double>& gridNodeSignedDistance, const double3 gridNodeLocalOrigin,
               const int3 gridNodeSize, const double gridNodeSpacing, const double3 position,
               const quaternion orientation, const double frictionCoefficient,
               const double restitutionCoefficient = 1.) {
    const int sz[3] = {gridNodeSize.x, gridNodeSize.y, gridNodeSize.z};
    const double o[3] = {gridNodeLocalOrigin.x, gridNodeLocalOrigin.y, gridNodeLocalOrigin.z};
    const double p[3] = {position.x, position.y, position.z};
    const double q[4] = {orientation.q0, orientation.q1, orientation.q2, orientation.q3};
    int index = -1;
    if (report(lsdem_add_wall(h_, (const double*)objVertexLocalPosition.data(), (int)objVertexLocalPosition.size(),
                              gridNodeSignedDistance.data(), sz, o, gridNodeSpacing, p, q, frictionCoefficient,
                              restitutionCoefficient, &index),
               "[LSParticle] "))
      return;
    setTriangles(1, index, objTriangleVertexID);
  }

  void moveLSParticle(const size_t index, const double3 offSet) {
    const double o[3] = {offSet.x, offSet.y, offSet.z};
    lsdem_move_particle(h_, (int)index, o);
  }
  void moveWall(const size_t index, const double3 offset) {
    const double o[3] = {offset.x, offset.y, offset.z};
    lsdem_move_wall(h_, (int)index, o);
  }
  void setFixedVelocityToWall(const size_t index, const double3 velocity) {
    const double v[3] = {velocity.x, velocity.y, velocity.z};
    lsdem_set_wall_velocity(h_, (int)index, v);
  }
  void setFixedAngularVelocityToWall(const size_t index, const double3 angularVelocity) {
    const double w[3] = {angularVelocity.x, angularVelocity.y, angularVelocity.z};
    lsdem_set_wall_angular_velocity(h_, (int)index, w);
  }

  // V-bond (LSSolver.h:344-379).
  void addBondedInteraction(const int masterObjectID, const int slaveObjectID, const double3 bondPoint,
                            const double3 bondNormal, const double radius, const double initialLength,
                            const double YoungsModulus, const double poissonRatio, const double tensileStrength = 0.,
                            const double cohesion = 0., const double frictionCoefficient = 0.) {
    const double p[3] = {bondPoint.x, bondPoint.y, bondPoint.z};
    const double n[3] = {bondNormal.x, bondNormal.y, bondNormal.z};
    report(lsdem_add_bond(h_, masterObjectID, slaveObjectID, p, n, radius, initialLength, YoungsModulus,
                          poissonRatio, tensileStrength, cohesion, frictionCoefficient),
           "[VBondedInteraction] ");
  }
  // Bonds at the current particle-particle contacts (LSSolver.h:385-418).
  void createBondsFromContacts(const double radius, const double initialLength, const double YoungsModulus,
                               const double poissonRatio, const double tensileStrength = 0.,
                               const double cohesion = 0., const double frictionCoefficient = 0.) {
    report(lsdem_create_bonds_from_contacts(h_, radius, initialLength, YoungsModulus, poissonRatio, tensileStrength,
                                            cohesion, frictionCoefficient),
           "[VBondedInteraction] ");
  }

  void addPeriodicBoundaryXD() { periodic_ |= 1; lsdem_set_periodic(h_, periodic_); }
  void addPeriodicBoundaryYD() { periodic_ |= 2; lsdem_set_periodic(h_, periodic_); }
  // Extension: the same image rule along z.
  void addPeriodicBoundaryZD() { periodic_ |= 4; lsdem_set_periodic(h_, periodic_); }
  void addPeriodicBoundarySector() { periodic_ = LSDEM_PERIODIC_SECTOR; lsdem_set_periodic(h_, periodic_); }
  void removePeriodicBoundary() { periodic_ = 0; lsdem_set_periodic(h_, 0); }

  // Extension: arithmetic form of the narrowphase (LSDEM_PREC_FP64, the reference's,
  // by default; LSDEM_PREC_FP32_FP16 / LSDEM_PREC_FP32_BF16: certified FP32 screening on
  // 16-bit SDF templates with FP64 contacts). Takes effect at the next solve().
  void setPrecision(const int mode) { report(lsdem_set_precision(h_, mode), "[Solver] "); }

  // Runs the step loop for maximumTime (numStep = floor(T/dt) + 1, numStep + 1 steps,
  // an output every numStep / numFrame steps), as LSSolver::solve (LSSolver.h:478-505, 994-1022).
  void solve(const double3 minDomain, const double3 maxDomain, const double3 gravity, const double timeStep,
             const double maximumTime, const size_t numFrame, const int argc, char** argv) {
    const double3 L = maxDomain - minDomain;
    if (L.x <= 0.0 || L.y <= 0.0 || L.z <= 0.0) {
      std::cerr << "[Solver] Invalid simulation domain size: (" << L.x << ", " << L.y << ", " << L.z << ")."
                << std::endl;
      return;
    }
    if (timeStep <= 0.0) { std::cerr << "[Solver] Invalid timeStep: " << timeStep << "." << std::endl; return; }
    if (maximumTime < 0.0) { std::cerr << "[Solver] Invalid maximumTime: " << maximumTime << "." << std::endl; return; }
    phase_ += 1;
    resolveDir(argc, argv);
    const double mn[3] = {minDomain.x, minDomain.y, minDomain.z};
    const double mx[3] = {maxDomain.x, maxDomain.y, maxDomain.z};
    const double g[3] = {gravity.x, gravity.y, gravity.z};
    std::cout << "[Solver] Uploading..." << std::endl;
    const int rc = lsdem_initialize(h_, mn, mx, g);
    if (rc == LSDEM_ERR_NODEVICE) {
      std::cout << "cudaSetDevice( " << device_ << " ) failed! Do you have a CUDA-capable GPU installed?"
                << std::endl;
      exit(1);
    }
    if (report(rc, "[Solver] ")) return;
    bindView();
    lsdem_set_record_contacts(h_, 1);
    clearOutput();
    std::cout << "[Solver] Upload Completed" << std::endl;
    const size_t numStep = size_t(maximumTime / timeStep) + 1;
    size_t frameInterval = numStep;
    if (numFrame > 0) frameInterval = numStep / numFrame;
    if (frameInterval < 1) frameInterval = 1;
    size_t iStep = 0, iFrame = 0;
    output(iFrame, iStep, lsdem_time(h_));
    while (iStep <= numStep) {
      const size_t next = std::min(numStep + 1, (iStep / frameInterval + 1) * frameInterval);
      const long long n = (long long)(next - iStep);
      if (report(lsdem_step(h_, timeStep, n, &LSSolver::hookTrampoline, this), "[Solver] ")) return;
      iStep = next;
      if (iStep % frameInterval == 0) output(++iFrame, iStep, lsdem_time(h_));
    }
    output(++iFrame, iStep, lsdem_time(h_));
    std::cout << "[Solver] Computation Completed" << std::endl;
  }

 protected:
  virtual void addExternalForceTorque(const double time) { (void)time; }
  LSParticle& getLSParticle() { return particles_; }
  LSParticle& getWall() { return walls_; }
  lsdem_solver* handle() { return h_; }

 private:
  static void hookTrampoline(void* self, double time) { static_cast<LSSolver*>(self)->addExternalForceTorque(time); }

  bool report(int rc, const char* who) {
    if (rc == LSDEM_OK) return false;
    std::cerr << who << lsdem_last_error(h_) << std::endl;
    return true;
  }

  void bindView() {
    LSParticle& v = particles_;
    lsdem_device_pointers(h_, &v.force_, &v.torque_, &v.vel_, &v.angvel_, &v.pos_, &v.quat_);
    v.n_ = (size_t)lsdem_num(h_, 0);
    v.block_ = maxGPUThread_ > 0 ? maxGPUThread_ : 1;
    if (v.n_ < v.block_) v.block_ = v.n_ ? v.n_ : 1;
    v.grid_ = (v.n_ + v.block_ - 1) / v.block_;
    walls_.n_ = (size_t)lsdem_num(h_, 1);
  }

  // Relative output directories are placed under the executable's "build" ancestor
  // (LSSolver.h:535-564).
  void resolveDir(int argc, char** argv) {
    std::filesystem::path p(dir_);
    if (p.is_absolute()) return;
    std::filesystem::path exe = (argc > 0 && argv && argv[0]) ? std::filesystem::path(argv[0])
                                                              : std::filesystem::current_path();
    if (exe.is_relative()) exe = std::filesystem::absolute(exe);
    exe = std::filesystem::weakly_canonical(exe);
    std::filesystem::path d = exe.parent_path();
    while (!d.empty() && d.filename() != "build" && d.parent_path() != d) d = d.parent_path();
    if (d.empty() || d.filename() != "build") d = exe.parent_path();
    dir_ = (d / p).string();
  }

  // Triangles of a body's nodes, kept for the mesh files (LSParticle::add, LSParticle.h:165-172).
  void setTriangles(int kind, int index, const std::vector<int3>& tris) {
    if (tris.empty() || index < 0) return;
    report(lsdem_set_triangles(h_, kind, index, (const int*)tris.data(), (int)tris.size()), "[LSParticle] ");
  }

  std::string phaseDir() const { return dir_ + "_phase" + std::to_string(phase_); }

  // removeVtuFiles of the four output directories at the start of a phase (LSSolver.h:600-612).
  void clearOutput() {
    for (const char* sub : {"LSParticle", "LSParticleInteraction", "Wall", "LSParticle-WallInteraction"}) {
      const std::filesystem::path d = std::filesystem::path(phaseDir()) / sub;
      std::error_code ec;
      if (!std::filesystem::is_directory(d, ec)) continue;
      for (const auto& e : std::filesystem::directory_iterator(d, ec))
        if (e.path().extension() == ".vtu") std::filesystem::remove(e.path(), ec);
    }
  }

  // One frame: the reference's six VTU files (LSSolver::output, LSSolver.h:637-665), written by
  // the library from device state (lsdem_write_vtu).
  void output(size_t iFrame, size_t iStep, double time) {
    std::cout << "[Solver] Phase " << phase_ << ": ------ Frame " << iFrame << " at Time " << time << " ------ "
              << std::endl;
    report(lsdem_write_vtu(h_, phaseDir().c_str(), iFrame, iStep, time), "[Solver] ");
  }

  lsdem_solver* h_ = nullptr;
  std::string dir_;
  cudaStream_t stream_;
  size_t maxGPUThread_;
  int device_;
  size_t phase_ = 0;
  int periodic_ = 0;
  LSParticle particles_, walls_;
};
