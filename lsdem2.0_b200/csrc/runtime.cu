// Host runtime and C ABI of the B200 level-set DEM step.
//
// Owns the model (shape templates, particles, walls, bonds), the device
// buffers and the step loop. The step loop runs in batches: the state at the
// start of a batch is copied aside, the batch is launched without any host
// synchronisation, and one status word is read back at the end. If a
// capacity (candidate slots, contact list) overflowed anywhere in the batch,
// buffers grow to the recorded need and the batch is re-run from the copy.
// This replaces the reference's per-list device-to-host count read and
// stream synchronisation every step (FunDEM/kernel/SolidInteraction.h:104-121).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>
#include "../../include/lsdem_b200.h"
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include "kernels.h"

using namespace lsdem;

namespace {

// ---------------------------------------------------------------------------
// Device array owner.
template <class T>
struct DArr {
  T* p = nullptr;
  size_t n = 0;
  DArr() = default;
  DArr(const DArr&) = delete;
  DArr& operator=(const DArr&) = delete;
  ~DArr() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t m) {
    release();
    if (m == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc((void**)&p, m * sizeof(T));
    if (e == cudaSuccess) n = m;
    else p = nullptr;
    return e;
  }
  cudaError_t upload(const T* h, size_t m, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    if (m != n || !p) e = alloc(m);
    if (e != cudaSuccess || m == 0) return e;
    return cudaMemcpyAsync(p, h, m * sizeof(T), cudaMemcpyHostToDevice, s);
  }
  cudaError_t zero(cudaStream_t s) { return n ? cudaMemsetAsync(p, 0, n * sizeof(T), s) : cudaSuccess; }
};

struct Fail {
  int code;
  std::string msg;
};
#define CK(x)                                                                                    \
  do {                                                                                           \
    cudaError_t e_ = (x);                                                                        \
    if (e_ != cudaSuccess)                                                                       \
      throw Fail{e_ == cudaErrorMemoryAllocation ? LSDEM_ERR_NOMEM : LSDEM_ERR_CUDA,             \
                 std::string(#x) + ": " + cudaGetErrorString(e_)};                               \
  } while (0)

// ---------------------------------------------------------------------------
// Host-side helpers (same arithmetic as the reference host code).
struct V3 { double x, y, z; };
inline V3 v3(const double* p) { return V3{p[0], p[1], p[2]}; }
inline double hlen(V3 v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
inline void qnormalize(const double* q, double* out) {
  double l2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  if (std::fabs(l2) <= 1.0e-20) { for (int a = 0; a < 4; ++a) out[a] = q[a]; return; }
  double inv = 1.0 / std::sqrt(l2);
  for (int a = 0; a < 4; ++a) out[a] = q[a] * inv;
}
inline V3 hrotate(const double* q, V3 v) {  // rotateVectorByQuaternion
  V3 qv{q[1], q[2], q[3]};
  auto cr = [](V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; };
  V3 t = cr(qv, v);
  t = V3{t.x * 2.0, t.y * 2.0, t.z * 2.0};
  V3 u = cr(qv, t);
  V3 a{v.x + t.x * q[0], v.y + t.y * q[0], v.z + t.z * q[0]};
  return V3{a.x + u.x, a.y + u.y, a.z + u.z};
}
inline V3 hrotate_inv(V3 v, const double* q) {  // reverseRotateVectorByQuaternion
  double c[4] = {q[0], -q[1], -q[2], -q[3]};
  return hrotate(c, v);
}
inline V3 hnormalize(V3 v) {
  double l2 = v.x * v.x + v.y * v.y + v.z * v.z;
  if (std::fabs(l2) <= 1.0e-20) return V3{0, 0, 0};
  double inv = 1.0 / std::sqrt(l2);
  return V3{v.x * inv, v.y * inv, v.z * inv};
}
inline V3 hcross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

inline int lin3h(int x, int y, int z, int nx, int ny) { return z * ny * nx + y * nx + x; }

// Mass properties by smoothed Heaviside integration (LSSolver.h:66-135). The loops, their
// x / y / z order and the smoothed Heaviside are the reference's on purpose: the sums are
// then taken in the reference's order and the masses and inertias equal its values bit for
// bit (the GPU routine in massprops.cu sums in parallel and agrees to rounding).
void mass_props(const double* sdf, const int* sz, const double* o, double h, double density, double* out) {
  auto H = [](double phi, double eps) -> double {
    if (eps <= 0.0) return (phi > 0.0) ? 0.0 : 1.0;
    if (phi < -eps) return 1.0;
    if (phi > eps) return 0.0;
    const double x = -phi / eps;
    return 0.5 * (1.0 + x + std::sin(M_PI * x) / M_PI);
  };
  const int nx = sz[0], ny = sz[1], nz = sz[2];
  double mass = 0.;
  const double mg = density * h * h * h;
  for (int x = 0; x < nx; x++)
    for (int y = 0; y < ny; y++)
      for (int z = 0; z < nz; z++) mass += H(sdf[lin3h(x, y, z, nx, ny)] / h, 1.5);
  mass *= mg;
  double c[3] = {0, 0, 0};
  double I[6] = {0, 0, 0, 0, 0, 0};
  if (mass > 0.) {
    for (int x = 0; x < nx; x++)
      for (int y = 0; y < ny; y++)
        for (int z = 0; z < nz; z++) {
          const double Hv = H(sdf[lin3h(x, y, z, nx, ny)] / h, 1.5);
          c[0] += Hv * (o[0] + double(x) * h);
          c[1] += Hv * (o[1] + double(y) * h);
          c[2] += Hv * (o[2] + double(z) * h);
        }
    const double f = mg / mass;
    c[0] *= f; c[1] *= f; c[2] *= f;
    for (int x = 0; x < nx; x++)
      for (int y = 0; y < ny; y++)
        for (int z = 0; z < nz; z++) {
          const double Hv = H(sdf[lin3h(x, y, z, nx, ny)] / h, 1.5);
          const double rx = o[0] + h * double(x) - c[0];
          const double ry = o[1] + h * double(y) - c[1];
          const double rz = o[2] + h * double(z) - c[2];
          I[0] += Hv * (ry * ry + rz * rz) * mg;
          I[1] += Hv * (rx * rx + rz * rz) * mg;
          I[2] += Hv * (ry * ry + rx * rx) * mg;
          I[3] -= Hv * rx * ry * mg;
          I[4] -= Hv * rx * rz * mg;
          I[5] -= Hv * ry * rz * mg;
        }
  }
  // inverse (myMat.h:163-195)
  double inv[6] = {0, 0, 0, 0, 0, 0};
  if (mass > 0.) {
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
  out[0] = mass;
  for (int a = 0; a < 3; ++a) out[1 + a] = c[a];
  for (int a = 0; a < 6; ++a) out[4 + a] = I[a];
  for (int a = 0; a < 6; ++a) out[10 + a] = inv[a];
}

void sym_inverse(const double* A, double* inv) {
  const double xx = A[0], yy = A[1], zz = A[2], xy = A[3], xz = A[4], yz = A[5];
  const double det = xx * (yy * zz - yz * yz) + xy * (yz * xz - xy * zz) + xz * (xy * yz - yy * xz);
  for (int a = 0; a < 6; ++a) inv[a] = 0.;
  if (std::fabs(det) < 1e-30) return;
  const double di = 1.0 / det;
  inv[0] = (yy * zz - yz * yz) * di;
  inv[1] = (xx * zz - xz * xz) * di;
  inv[2] = (xx * yy - xy * xy) * di;
  inv[3] = -(xy * zz - xz * yz) * di;
  inv[4] = (xy * yz - xz * yy) * di;
  inv[5] = -(xx * yz - xz * xy) * di;
}

uint64_t fnv(const void* data, size_t bytes, uint64_t h = 1469598103934665603ull) {
  const unsigned char* p = (const unsigned char*)data;
  for (size_t i = 0; i < bytes; ++i) { h ^= p[i]; h *= 1099511628211ull; }
  return h;
}

// ---------------------------------------------------------------------------
struct ShapeHost {
  std::vector<double> nodes;  // caller order, 3 per node
  std::vector<double> sdf;
  int size[3];
  double origin[3];
  double h;
  std::vector<int> perm;      // cluster position -> caller index
  std::vector<double> cl;     // 4 per cluster
  std::vector<double> sub;    // 4 per sub-cluster of 8 nodes (4 sub-clusters per cluster)
  uint64_t hash;
};

// Orders nodes along a Morton curve so that runs of 32 consecutive nodes are
// spatially compact, and bounds each run by a sphere.
void build_clusters(ShapeHost& s) {
  const int M = (int)(s.nodes.size() / 3);
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < M; ++i)
    for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], s.nodes[3 * i + a]); hi[a] = std::max(hi[a], s.nodes[3 * i + a]); }
  auto spread = [](uint32_t v) {
    uint64_t x = v & 0x1fffff;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
  };
  std::vector<std::pair<uint64_t, int>> key(M);
  for (int i = 0; i < M; ++i) {
    uint64_t code = 0;
    for (int a = 0; a < 3; ++a) {
      double ext = hi[a] - lo[a];
      double t = ext > 0 ? (s.nodes[3 * i + a] - lo[a]) / ext : 0.0;
      uint32_t q = (uint32_t)std::min(1023.0, std::max(0.0, t * 1023.0));
      code |= spread(q) << a;
    }
    key[i] = {code, i};
  }
  std::stable_sort(key.begin(), key.end());
  s.perm.resize(M);
  for (int i = 0; i < M; ++i) s.perm[i] = key[i].second;
  const int ncl = (M + 31) / 32;
  s.cl.assign(4 * (size_t)ncl, 0.0);
  for (int c = 0; c < ncl; ++c) {
    const int b = c * 32, e = std::min(M, b + 32);
    double m[3] = {0, 0, 0};
    for (int k = b; k < e; ++k)
      for (int a = 0; a < 3; ++a) m[a] += s.nodes[3 * s.perm[k] + a];
    for (int a = 0; a < 3; ++a) m[a] /= (e - b);
    double r = 0;
    for (int k = b; k < e; ++k) {
      const double* p = &s.nodes[3 * s.perm[k]];
      r = std::max(r, std::sqrt((p[0] - m[0]) * (p[0] - m[0]) + (p[1] - m[1]) * (p[1] - m[1]) +
                                (p[2] - m[2]) * (p[2] - m[2])));
    }
    s.cl[4 * c] = m[0]; s.cl[4 * c + 1] = m[1]; s.cl[4 * c + 2] = m[2];
    s.cl[4 * c + 3] = r * (1.0 + 1e-12) + 1e-300;
  }
  // sub-clusters: 8 consecutive nodes each, 4 per cluster (a missing one has radius -1)
  s.sub.assign(16 * (size_t)ncl, 0.0);
  for (int q = 0; q < 4 * ncl; ++q) {
    const int b = q * 8, e = std::min(M, b + 8);
    if (b >= M) { s.sub[4 * q + 3] = -1.0; continue; }
    double m[3] = {0, 0, 0};
    for (int k = b; k < e; ++k)
      for (int a = 0; a < 3; ++a) m[a] += s.nodes[3 * s.perm[k] + a];
    for (int a = 0; a < 3; ++a) m[a] /= (e - b);
    double r = 0;
    for (int k = b; k < e; ++k) {
      const double* p = &s.nodes[3 * s.perm[k]];
      r = std::max(r, std::sqrt((p[0] - m[0]) * (p[0] - m[0]) + (p[1] - m[1]) * (p[1] - m[1]) +
                                (p[2] - m[2]) * (p[2] - m[2])));
    }
    s.sub[4 * q] = m[0]; s.sub[4 * q + 1] = m[1]; s.sub[4 * q + 2] = m[2];
    s.sub[4 * q + 3] = r * (1.0 + 1e-12) + 1e-300;
  }
}

struct BodyHost {
  std::vector<double> pos, vel, angvel, quat, force, torque, invm, invI, radius, kn, ks, mu, res, scale, origin, invh;
  std::vector<int> shape;
  std::vector<long long> node_base;
  int n() const { return (int)shape.size(); }
};

struct BodyDev {
  DArr<double3> pos, vel, angvel, force, torque, origin;
  DArr<Quat> quat;
  DArr<float4> rotm;  // precision form, particles: FP32 rotation matrix rows (written each step)
  DArr<double> invm, radius, kn, ks, mu, res, scale, invh;
  DArr<Sym6> invI;
  DArr<int> shape, key;
  DArr<long long> node_base;
};

struct SlotsDev {
  int cap = 0;
  DArr<int> cnt, id, seg_start, seg_cnt;
};

struct ContactsDev {
  long long cap = 0;
  DArr<int> count, node;
  DArr<double3> spring, point, normal;
  DArr<double> overlap, en_n, en_s;
  bool geom = false;
};

struct BondHost {
  std::vector<int> ids, bonded;
  std::vector<double> B, geo, frames, state;
};

}  // namespace

struct lsdem_solver {
  int device = 0;
  cudaStream_t stream = nullptr;
  int flags = 0;
  int precision = PREC_FP64;
  double rmax_p = 0.;        // largest particle bounding radius (set at initialize)
  std::string err;
  // model
  std::vector<ShapeHost> shapes;
  std::unordered_map<uint64_t, std::vector<int>> shape_by_hash;
  std::map<std::pair<int, uint64_t>, double> radius_cache;  // (shape, scale bits) -> radius
  BodyHost P, W;
  BondHost bonds;
  // frame output: wall vertices (local frame), triangle sets of the bodies' nodes
  // (LSParticle::add's boundaryNodeConnectivity, LSParticle.h:165-172), the writer
  std::vector<std::vector<double>> wall_verts;
  std::vector<std::vector<int>> tri_sets;
  std::map<std::vector<int>, int> tri_set_of;
  std::vector<int> P_tris, W_tris;  // per body: triangle set, -1 none
  long long vtu_layout = 0;
  VtuCtx* vtu = nullptr;
  // CUDA graph of one step per history parity, replayed for steps without a host hook,
  // profiling or contact recording; `graph_gen` changes whenever a step's arguments or
  // launch configuration may change (initialize, capacity growth, setters)
  struct StepGraph { cudaGraphExec_t exec = nullptr; uint64_t key = 0; long long launches = 0; };
  StepGraph sgraph[2];
  long long graph_gen = 0;
  bool graphs = true;
  cudaStream_t gstream = nullptr;  // blocking stream for replay when the solver runs on the legacy stream
  int periodic = 0;
  double dmin[3] = {0, 0, 0}, dmax[3] = {0, 0, 0}, grav[3] = {0, 0, 0};
  // device
  bool ready = false;
  BodyDev dP, dW;
  DArr<int3> s_gsize;
  DArr<long long> s_sdf_off;
  DArr<double> s_sdf;
  DArr<int> s_node_off, s_node_cnt, s_cl_off, s_cl_cnt, s_node_orig;
  DArr<double3> s_node_pos;
  DArr<double4> s_cl;
  DArr<float4> s_clf;   // cluster spheres in FP32 (each component rounded to nearest)
  DArr<float4> s_sub;   // sub-cluster spheres, 4 per cluster (FP32, radius rounded up)
  DArr<double> s_nbox;  // per shape: node bounding box (lo xyz, hi xyz), largest node distance, 0
  DArr<uint4> s_cell16;        // precision form: 16-bit corners of every grid cell
  DArr<long long> s_cell_off;  // per shape, into s_cell16
  DArr<float4> s_node_f;
  DArr<float> s_lip;
  // precision form: screened nodes and queued pairs (per-step scratch)
  DArr<int> mb_node, mb_ctr;
  DArr<int> plist[3], pl_ctr;
  DArr<unsigned long long> scr_stats;  // screen counters (allocated while enabled)
  // learned per-shape SDF (precision forms)
  DArr<float> mlp_params, mlp_m1, mlp_m2, mlp_partial, mlp_loss, mlp_band;
  DArr<float4> mlp_samples;
  DArr<MlpInfer> mlp_inf;
  DArr<MlpNorm> mlp_norm;
  DArr<double3> mlp_origin;
  DArr<double> mlp_h;
  DArr<unsigned> mlp_err;
  std::vector<MlpNorm> h_mlp_norm;
  std::vector<float> h_mlp_band;
  MlpTrainOpts mlp_opt;
  bool mlp_trained = false, mlp_on = false;
  DArr<int4> mb_pair;
  long long mb_cap = 0, mb_pcap = 0;
  // learned form: network queues and pending nodes, per narrowphase launch
  struct NetDev {
    DArr<float4> row;
    DArr<int> cnt, pend_n, ctr;
    DArr<unsigned char> pend_v;
    DArr<int4> pair;
    int qcap = 0, pcap = 0, paircap = 0;
  } net[2];
  long long cap_netq = 0, cap_pend = 0;  // rows per shape, pending nodes per launch (0: not sized yet)
  bool net_dirty = true;                 // the buffers must be (re)allocated before the next step
  std::vector<int> h_node_off, h_cl_off;
  GridP pg{}, wg{};
  DArr<int> cell_idx, cell_start, cell_end, sorted_key;
  DArr<float4> cell_pk;
  DArr<int> bk_counts, bk_fill, bk_offs, bk_scan, bk_big, bk_bigc, bk_tmp;
  // periodic images as a parallel branch of the step: wrapped positions, the image
  // sort's own scratch and packed cells, a second stream and the fork / join events
  DArr<double3> pos_w;
  DArr<float4> cell_pk2;
  DArr<int> bk2_counts, bk2_fill, bk2_offs, bk2_scan, bk2_big, bk2_bigc, bk2_tmp;
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // neighbour lists (exact; see k_candidates): flag word, positions at the last
  // rebuild, lists, this step's keys in sorted order
  bool reuse_on = true;
  bool force_reuse = true;   // the next step sorts and rebuilds (set after any re-allocation)
  bool grow_nbr = false;
  DArr<int> reuse;
  DArr<double3> xb;
  DArr<int> nbr, nbr_cnt;
  DArr<int4> pk_meta;
  DArr<float4> pk_q;
  // support tables of the shapes (pair separation test of the candidate search)
  DArr<double3> sup_pts;
  DArr<long long> sup_off;
  DArr<float4> sup_n, sup_s;
  DArr<float> sup_r, sup_vtx;
  int nbr_cap = 24;
  float skin = 0.f;
  double move2 = 0.;
  long long builds = 0;      // steps that sorted and rebuilt the lists (lists on)
  SlotsDev slots[2][3];      // [history parity][kind]
  ContactsDev con[2];
  int hp = 0;                // parity of the last completed step's history
  int cap_pp = 32, cap_w = 4, cap_g = 16;
  long long cap_c = 0;
  int batch = 16;
  int cur_batch = 1;         // adaptive batch length, doubled after each clean batch
  bool record = false;
  // periodic
  int nsets = 0;
  int set_mask[7] = {0};
  DArr<double3> gpos, gvel;
  DArr<Quat> gquat;
  DArr<int> gkey, key2, g2_idx, g2_start, g2_end, glist, gcount;
  // bonds
  DArr<int> b_ids, b_bonded;
  DArr<double> b_B, b_geo, b_state;
  DArr<double3> b_frames;
  // status + backup
  DArr<Status> status;
  Status* h_status = nullptr;
  int* h_count = nullptr;
  DArr<double3> bk_pos, bk_vel, bk_angvel, bk_force, bk_torque, bk_wpos;
  DArr<Quat> bk_quat, bk_wquat;
  DArr<int> bk_bonded, bk_slot[3][4], bk_cnode;
  DArr<double3> bk_cspring;
  int bk_cap[3] = {0, 0, 0};
  long long hist_count = 0;  // contacts in the history buffer hp
  // host copies of the device state: stale after steps until pulled (pull_host); the
  // body and node counts the device arrays were built for
  bool host_stale = false;
  int dev_np = -1, dev_nw = -1;
  long long dev_nodes = -1;
  int dev_nsets = -1;
  size_t dev_nb = 0;
  bool grow_contacts = false;
  long long steps = 0, reruns = 0, launches = 0;
  double time = 0.0;
  // optional per-phase device timing (CUDA events on the solver stream)
  bool profiling = false;
  // step timing (benchmarks): CUDA events around every step (phase 9), and an
  // optional write of a scratch buffer larger than L2 before each step, outside
  // the events
  bool step_timing = false;
  DArr<unsigned char> flush_buf;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_pending;
  std::vector<cudaEvent_t> event_pool;
  double prof_ms[LSDEM_NUM_PHASES] = {};
  long long prof_calls[LSDEM_NUM_PHASES] = {};

  ~lsdem_solver() {
    if (h_status) cudaFreeHost(h_status);
    if (h_count) cudaFreeHost(h_count);
    for (auto& p : prof_pending) { cudaEventDestroy(p.second.first); cudaEventDestroy(p.second.second); }
    for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
  }
};

namespace {

int fail(lsdem_solver* s, int code, const std::string& m) {
  if (s) s->err = m;
  return code;
}

template <class F>
int guard(lsdem_solver* s, F&& f) {
  try {
    return f();
  } catch (const Fail& e) {
    return fail(s, e.code, e.msg);
  } catch (const std::exception& e) {
    return fail(s, LSDEM_ERR_ARG, e.what());
  }
}

int add_shape_impl(lsdem_solver* s, const double* nodes, int nn, const double* sdf, const int* sz, const double* o,
                   double h) {
  if (sz[0] < 2 || sz[1] < 2 || sz[2] < 2) throw Fail{LSDEM_ERR_ARG, "Invalid level-set grid size (must be >= 2 per axis)"};
  if (!(h > 0.0)) throw Fail{LSDEM_ERR_ARG, "Invalid level-set grid spacing (must be > 0)"};
  if (nn < 0 || nn > 256 * 32) throw Fail{LSDEM_ERR_ARG, "Invalid surface node count (0..8192)"};
  const size_t ng = (size_t)sz[0] * sz[1] * sz[2];
  uint64_t hsh = fnv(nodes, sizeof(double) * 3 * (size_t)nn);
  hsh = fnv(sdf, sizeof(double) * ng, hsh);
  hsh = fnv(sz, sizeof(int) * 3, hsh);
  hsh = fnv(o, sizeof(double) * 3, hsh);
  hsh = fnv(&h, sizeof(double), hsh);
  auto it = s->shape_by_hash.find(hsh);
  if (it != s->shape_by_hash.end()) {
    for (int id : it->second) {
      const ShapeHost& e = s->shapes[id];
      if (e.nodes.size() == 3 * (size_t)nn && e.sdf.size() == ng && e.size[0] == sz[0] && e.size[1] == sz[1] &&
          e.size[2] == sz[2] && e.origin[0] == o[0] && e.origin[1] == o[1] && e.origin[2] == o[2] && e.h == h &&
          std::memcmp(e.nodes.data(), nodes, sizeof(double) * 3 * (size_t)nn) == 0 &&
          std::memcmp(e.sdf.data(), sdf, sizeof(double) * ng) == 0)
        return id;
    }
  }
  ShapeHost sh;
  sh.nodes.assign(nodes, nodes + 3 * (size_t)nn);
  sh.sdf.assign(sdf, sdf + ng);
  for (int a = 0; a < 3; ++a) { sh.size[a] = sz[a]; sh.origin[a] = o[a]; }
  sh.h = h;
  sh.hash = hsh;
  build_clusters(sh);
  s->shapes.push_back(std::move(sh));
  const int id = (int)s->shapes.size() - 1;
  s->shape_by_hash[hsh].push_back(id);
  s->ready = false;
  return id;
}

// radius = max |scale * node| over the body's nodes (LSParticle.h:175-181).
double shape_radius(lsdem_solver* s, int shape, double scale) {
  uint64_t bits;
  std::memcpy(&bits, &scale, 8);
  auto key = std::make_pair(shape, bits);
  auto it = s->radius_cache.find(key);
  if (it != s->radius_cache.end()) return it->second;
  const ShapeHost& sh = s->shapes[shape];
  double r = 0.;
  for (size_t i = 0; i < sh.nodes.size() / 3; ++i) {
    V3 p{scale * sh.nodes[3 * i], scale * sh.nodes[3 * i + 1], scale * sh.nodes[3 * i + 2]};
    r = std::max(hlen(p), r);
  }
  s->radius_cache[key] = r;
  return r;
}

void push_body(lsdem_solver* s, BodyHost& B, int shape, double scale, const double* pos, const double* vel,
               const double* angvel, const double* quat, double invm, const double* invI, double kn, double ks,
               double mu, double e, double radius) {
  const ShapeHost& sh = s->shapes[shape];
  for (int a = 0; a < 3; ++a) {
    B.pos.push_back(pos[a]);
    B.vel.push_back(vel ? vel[a] : 0.);
    B.angvel.push_back(angvel ? angvel[a] : 0.);
    B.origin.push_back(scale == 1.0 ? sh.origin[a] : scale * sh.origin[a]);
    B.force.push_back(0.);
    B.torque.push_back(0.);
  }
  double q[4];
  qnormalize(quat, q);
  for (int a = 0; a < 4; ++a) B.quat.push_back(q[a]);
  B.invm.push_back(invm);
  for (int a = 0; a < 6; ++a) B.invI.push_back(invI ? invI[a] : 0.);
  B.radius.push_back(radius);
  B.kn.push_back(kn > 0. ? kn : 0.);
  B.ks.push_back(ks > 0. ? ks : 0.);
  B.mu.push_back(mu > 0. ? mu : 0.);
  double ee = e;
  if (ee <= 0.0 || ee > 1.0) ee = 1.0;
  B.res.push_back(ee);
  B.scale.push_back(scale);
  B.invh.push_back(1. / (scale == 1.0 ? sh.h : scale * sh.h));
  B.shape.push_back(shape);
}

// ---------------------------------------------------------------------------
// Device set-up.
void alloc_slots(lsdem_solver* s, bool keep_unchanged = false) {
  const int n = s->P.n();
  const int caps[3] = {s->cap_pp, s->P.n() ? s->cap_w : 0, s->cap_g};
  for (int h = 0; h < 2; ++h)
    for (int k = 0; k < 3; ++k) {
      SlotsDev& sl = s->slots[h][k];
      const int cap = (k == 1 && s->W.n() == 0) ? 0 : caps[k];
      if (k == 2 && s->nsets == 0) {
        sl.cap = 0;
        sl.cnt.release(); sl.id.release(); sl.seg_start.release(); sl.seg_cnt.release();
        continue;
      }
      const size_t m = (size_t)std::max(n, 1) * std::max(cap, 1);
      // unchanged kind: keep the arrays (restore rewrites their contents)
      if (keep_unchanged && sl.cap == cap && sl.id.n == m && sl.cnt.n == (size_t)std::max(n, 1)) continue;
      sl.cap = cap;
      CK(sl.cnt.alloc((size_t)std::max(n, 1)));
      CK(sl.cnt.zero(s->stream));
      CK(sl.id.alloc(m));
      CK(sl.seg_start.alloc(m));
      CK(sl.seg_cnt.alloc(m));
      CK(sl.seg_cnt.zero(s->stream));
    }
  // precision form: flat pair lists, one entry per slot
  for (int k = 0; k < 3; ++k) {
    const int cap = s->slots[0][k].cap;
    const size_t m = (size_t)std::max(n, 1) * std::max(cap, 1);
    if (s->precision == PREC_FP64 || cap == 0) { s->plist[k].release(); continue; }
    if ((long long)n * cap > 0x7fffffffLL) throw Fail{LSDEM_ERR_NOMEM, "pair list index exceeds 32 bits"};
    if (s->plist[k].n != m) CK(s->plist[k].alloc(m));
  }
  if (s->precision != PREC_FP64 && !s->pl_ctr.p) {
    CK(s->pl_ctr.alloc(4));
    CK(s->pl_ctr.zero(s->stream));
  }
}

void alloc_contacts(lsdem_solver* s, ContactsDev& c, long long cap) {
  c.cap = cap;
  CK(c.count.alloc(1));
  CK(c.count.zero(s->stream));
  CK(c.node.alloc((size_t)std::max(cap, 1LL)));
  CK(c.spring.alloc((size_t)std::max(cap, 1LL)));
  c.point.release(); c.normal.release(); c.overlap.release(); c.en_n.release(); c.en_s.release();
  c.geom = false;
}

// Learned form: the network queues (rows per shape), the pending nodes and the pair
// records of both narrowphase launches. Per-step scratch: contents are not kept.
void alloc_net(lsdem_solver* s) {
  const int n = std::max(s->P.n(), 1);
  const int ns = std::max((int)s->shapes.size(), 1);
  if (s->cap_pend <= 0) s->cap_pend = std::max<long long>(1 << 20, (long long)n * 8);
  if (s->cap_netq <= 0) s->cap_netq = std::max<long long>(1 << 14, s->cap_pend / ns * 2);
  s->cap_pend = std::min<long long>(s->cap_pend, 0x7fffffffLL);
  s->cap_netq = std::min<long long>(s->cap_netq, 0x7fffffffLL / ns);
  for (int l = 0; l < 2; ++l) {
    auto& N = s->net[l];
    const long long pairs = l == 0 ? (long long)n * (s->slots[0][0].cap + s->slots[0][1].cap)
                                   : (long long)n * s->slots[0][2].cap;
    if (l == 1 && s->nsets == 0) {
      N.qcap = N.pcap = N.paircap = 0;
      N.row.release(); N.cnt.release(); N.pend_n.release(); N.ctr.release();
      N.pend_v.release(); N.pair.release();
      continue;
    }
    N.qcap = (int)s->cap_netq;
    N.pcap = (int)s->cap_pend;
    N.paircap = (int)std::min<long long>(std::max<long long>(pairs, 1), 0x7fffffffLL);
    CK(N.row.alloc((size_t)ns * N.qcap * 2));
    CK(N.cnt.alloc(ns)); CK(N.cnt.zero(s->stream));
    CK(N.pend_n.alloc(N.pcap));
    CK(N.pend_v.alloc(N.pcap));
    CK(N.pair.alloc(N.paircap));
    CK(N.ctr.alloc(2)); CK(N.ctr.zero(s->stream));
  }
  s->net_dirty = false;
}

// Scratch of the precision form, sized with the contact capacity.
void alloc_maybe(lsdem_solver* s) {
  if (s->precision == PREC_FP64) return;
  const long long cap = std::min<long long>(s->cap_c, 0x7fffffffLL);
  if (s->mb_cap == cap && s->mb_node.p) return;
  s->mb_cap = cap;
  s->mb_pcap = std::max<long long>(cap / 2, 1024);
  CK(s->mb_node.alloc((size_t)cap));
  CK(s->mb_pair.alloc((size_t)(2 * s->mb_pcap)));
  CK(s->mb_ctr.alloc(4));
  CK(s->mb_ctr.zero(s->stream));
}

void ensure_geom(lsdem_solver* s, ContactsDev& c) {
  if (c.geom) return;
  const size_t m = (size_t)std::max(c.cap, 1LL);
  CK(c.point.alloc(m));
  CK(c.normal.alloc(m));
  CK(c.overlap.alloc(m));
  CK(c.en_n.alloc(m));
  CK(c.en_s.alloc(m));
  c.geom = true;
}

void upload_bodies(lsdem_solver* s, BodyHost& H, BodyDev& D) {
  const size_t n = (size_t)H.n();
  cudaStream_t st = s->stream;
  CK(D.pos.upload((const double3*)H.pos.data(), n, st));
  CK(D.vel.upload((const double3*)H.vel.data(), n, st));
  CK(D.angvel.upload((const double3*)H.angvel.data(), n, st));
  // forces of the last step (zero before the first): the first half kick of a new
  // phase uses them, as the reference's upload of its host copy does (LSParticle.h:700-710)
  CK(D.force.upload((const double3*)H.force.data(), n, st));
  CK(D.torque.upload((const double3*)H.torque.data(), n, st));
  CK(D.origin.upload((const double3*)H.origin.data(), n, st));
  CK(D.quat.upload((const Quat*)H.quat.data(), n, st));
  CK(D.invm.upload(H.invm.data(), n, st));
  CK(D.invI.upload((const Sym6*)H.invI.data(), n, st));
  CK(D.radius.upload(H.radius.data(), n, st));
  CK(D.kn.upload(H.kn.data(), n, st));
  CK(D.ks.upload(H.ks.data(), n, st));
  CK(D.mu.upload(H.mu.data(), n, st));
  CK(D.res.upload(H.res.data(), n, st));
  CK(D.scale.upload(H.scale.data(), n, st));
  CK(D.invh.upload(H.invh.data(), n, st));
  CK(D.shape.upload(H.shape.data(), n, st));
  CK(D.key.alloc(std::max<size_t>(n, 1)));
  if (!H.node_base.empty()) CK(D.node_base.upload(H.node_base.data(), n, st));
  if (&D == &s->dP && s->precision != PREC_FP64) CK(D.rotm.alloc(3 * std::max<size_t>(n, 1)));
  else D.rotm.release();
}

// Brings the host copies of the bodies' state up to date with the device after steps:
// particle position, velocity, angular velocity, orientation, force and torque, wall
// position and orientation, bond flags and state (the reference downloads them at every
// output, LSSolver.h:625-635, so that its host-side edits and the next phase's upload start
// from the last step). Called before every host-side read or edit of that state.
void pull_host(lsdem_solver* s) {
  if (!s->host_stale) return;
  cudaStream_t st = s->stream;
  const size_t n = (size_t)std::min(s->dev_np, s->P.n()), nw = (size_t)std::min(s->dev_nw, s->W.n());
  auto dl = [&](std::vector<double>& h, const void* d, size_t bytes) {
    if (bytes) CK(cudaMemcpyAsync(h.data(), d, bytes, cudaMemcpyDeviceToHost, st));
  };
  dl(s->P.pos, s->dP.pos.p, 24 * n);
  dl(s->P.vel, s->dP.vel.p, 24 * n);
  dl(s->P.angvel, s->dP.angvel.p, 24 * n);
  dl(s->P.quat, s->dP.quat.p, 32 * n);
  dl(s->P.force, s->dP.force.p, 24 * n);
  dl(s->P.torque, s->dP.torque.p, 24 * n);
  dl(s->W.pos, s->dW.pos.p, 24 * nw);
  dl(s->W.quat, s->dW.quat.p, 32 * nw);
  const size_t nb = std::min(s->dev_nb, s->bonds.bonded.size());
  if (nb) {
    CK(cudaMemcpyAsync(s->bonds.bonded.data(), s->b_bonded.p, sizeof(int) * nb, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(s->bonds.state.data(), s->b_state.p, sizeof(double) * 9 * nb, cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  s->host_stale = false;
}

void set_grid(GridP& g, const double* mn, const double* mx_in, double cell) {  // spatialGrid::set
  double mx[3] = {mx_in[0], mx_in[1], mx_in[2]};
  for (int a = 0; a < 3; ++a)
    if (mx[a] <= mn[a]) mx[a] = mn[a] + cell;
  int size[3] = {2, 2, 2};
  double inv[3] = {0, 0, 0};
  if (!(std::fabs(cell) <= 1.0e-20)) {
    for (int a = 0; a < 3; ++a) {
      const double d = mx[a] - mn[a];
      size[a] = d > 2. * cell ? int(d / cell) : 2;
      inv[a] = (d > 0.0) ? (double(size[a]) / d) : 0.0;
    }
  }
  g.mn = make_double3(mn[0], mn[1], mn[2]);
  g.mx = make_double3(mx[0], mx[1], mx[2]);
  g.inv = make_double3(inv[0], inv[1], inv[2]);
  g.size = make_int3(size[0], size[1], size[2]);
  g.ncells = size[0] * size[1] * size[2];
}

void alloc_bucket(lsdem_solver* s, int n, int ncells, bool second = false) {
  const int nb = ncells + 2;
  auto& c = second ? s->bk2_counts : s->bk_counts;
  auto& f = second ? s->bk2_fill : s->bk_fill;
  auto& o = second ? s->bk2_offs : s->bk_offs;
  auto& sc = second ? s->bk2_scan : s->bk_scan;
  auto& b = second ? s->bk2_big : s->bk_big;
  auto& bc = second ? s->bk2_bigc : s->bk_bigc;
  auto& t = second ? s->bk2_tmp : s->bk_tmp;
  CK(c.alloc(nb + 1));
  CK(f.alloc(nb + 1));
  CK(o.alloc(nb + 1));
  CK(sc.alloc(scan_temp_elems(nb + 1)));
  CK(b.alloc((size_t)n / 65 + 1));
  CK(bc.alloc(2));
  CK(t.alloc((size_t)std::max(n, 1)));
}

void backup_history(lsdem_solver* s);
void restore_history(lsdem_solver* s, int hp0);

void initialize(lsdem_solver* s) {
  // A new phase of the same bodies keeps the contact history of the last step, as the
  // reference keeps its contact arrays when their size is unchanged (SolidInteraction.h:24-27,
  // PeriodicBoundary.h:23-39): saved here, put back after the buffers are rebuilt.
  pull_host(s);
  long long nodes_now = 0;
  for (int i = 0; i < s->P.n(); ++i) nodes_now += (long long)(s->shapes[s->P.shape[i]].nodes.size() / 3);
  int nsets_now = 0;
  {
    const int ax = s->periodic & 7;
    for (int m = 1; m < 8; ++m)
      if ((m & ax) == m) ++nsets_now;
    if (s->periodic & 8) nsets_now = 3;
  }
  const bool carry = s->hist_count > 0 && s->dev_np == s->P.n() && s->dev_nw == s->W.n() &&
                     s->dev_nodes == nodes_now && s->dev_nsets == nsets_now;
  const long long carried = carry ? s->hist_count : 0;
  if (carry) backup_history(s);
  CK(cudaSetDevice(s->device));
  cudaStream_t st = s->stream;
  // shapes
  std::vector<int3> gs;
  std::vector<long long> sdf_off;
  std::vector<double> sdf;
  std::vector<int> node_off, node_cnt, cl_off, cl_cnt, node_orig;
  std::vector<double3> node_pos;
  std::vector<double4> cl;
  for (const ShapeHost& sh : s->shapes) {
    gs.push_back(make_int3(sh.size[0], sh.size[1], sh.size[2]));
    sdf_off.push_back((long long)sdf.size());
    sdf.insert(sdf.end(), sh.sdf.begin(), sh.sdf.end());
    node_off.push_back((int)node_pos.size());
    const int M = (int)sh.perm.size();
    node_cnt.push_back(M);
    for (int k = 0; k < M; ++k) {
      const double* p = &sh.nodes[3 * sh.perm[k]];
      node_pos.push_back(make_double3(p[0], p[1], p[2]));
      node_orig.push_back(sh.perm[k]);
    }
    cl_off.push_back((int)cl.size());
    cl_cnt.push_back((int)(sh.cl.size() / 4));
    for (size_t c = 0; c < sh.cl.size() / 4; ++c)
      cl.push_back(make_double4(sh.cl[4 * c], sh.cl[4 * c + 1], sh.cl[4 * c + 2], sh.cl[4 * c + 3]));
  }
  s->h_node_off = node_off;
  s->h_cl_off = cl_off;
  CK(s->s_gsize.upload(gs.data(), gs.size(), st));
  CK(s->s_sdf_off.upload(sdf_off.data(), sdf_off.size(), st));
  CK(s->s_sdf.upload(sdf.data(), sdf.size(), st));
  CK(s->s_node_off.upload(node_off.data(), node_off.size(), st));
  CK(s->s_node_cnt.upload(node_cnt.data(), node_cnt.size(), st));
  CK(s->s_cl_off.upload(cl_off.data(), cl_off.size(), st));
  CK(s->s_cl_cnt.upload(cl_cnt.data(), cl_cnt.size(), st));
  CK(s->s_node_pos.upload(node_pos.data(), node_pos.size(), st));
  CK(s->s_node_orig.upload(node_orig.data(), node_orig.size(), st));
  CK(s->s_cl.upload(cl.data(), cl.size(), st));
  {
    std::vector<float4> clf(cl.size());
    for (size_t c = 0; c < cl.size(); ++c)
      clf[c] = make_float4((float)cl[c].x, (float)cl[c].y, (float)cl[c].z, (float)cl[c].w);
    CK(s->s_clf.upload(clf.data(), clf.size(), st));
  }
  {
    // support tables: per shape, points whose convex hull holds every point where the
    // trilinear phi is <= 0, template units. The grid is refined by two (points at half
    // spacings): phi restricted to one of the eight sub-cells of a cell is trilinear
    // with the sub-cell's corner values, and a multilinear function takes its minimum
    // over a box at a corner, so a point with phi <= 0 lies in a sub-cell with a corner
    // phi <= 0. Those corners are marked (each with a tolerance above the rounding of
    // its interpolation), the marks dilated by one refined point in every direction
    // (the corners of every such sub-cell), and only the points with a 6-neighbour
    // outside the set kept (the largest projection of a lattice set is reached there).
    std::vector<double3> pts;
    std::vector<long long> poff{0};
    for (const ShapeHost& sh : s->shapes) {
      const int gx = sh.size[0], gy = sh.size[1], gz = sh.size[2];
      const int nx = 2 * gx - 1, ny = 2 * gy - 1, nz = 2 * gz - 1;
      const size_t N = (size_t)nx * ny * nz;
      auto id = [&](int x, int y, int z) { return (size_t)x + (size_t)nx * (y + (size_t)ny * z); };
      auto gv = [&](int x, int y, int z) { return sh.sdf[(size_t)x + (size_t)gx * (y + (size_t)gy * z)]; };
      std::vector<uint8_t> m(N, 0), t(N);
      for (int z = 0; z + 1 < gz; ++z)
        for (int y = 0; y + 1 < gy; ++y)
          for (int x = 0; x + 1 < gx; ++x) {
            double c[8], lo = 1e300, hi = -1e300, mag = 0.;
            for (int k = 0; k < 8; ++k) {
              c[k] = gv(x + (k & 1), y + ((k >> 1) & 1), z + (k >> 2));
              lo = std::min(lo, c[k]);
              hi = std::max(hi, c[k]);
              mag = std::max(mag, std::fabs(c[k]));
            }
            const double tol = 1e-12 * mag;
            if (lo > tol) continue;  // phi > 0 on the whole cell
            for (int k = 0; k < 27; ++k) {
              const int i = k % 3, j = (k / 3) % 3, l = k / 9;
              double v;
              if (hi <= tol) {
                v = lo;  // phi <= 0 on the whole cell
              } else {
                const double fx = 0.5 * i, fy = 0.5 * j, fz = 0.5 * l;
                const double c00 = c[0] * (1 - fx) + c[1] * fx, c10 = c[2] * (1 - fx) + c[3] * fx;
                const double c01 = c[4] * (1 - fx) + c[5] * fx, c11 = c[6] * (1 - fx) + c[7] * fx;
                v = (c00 * (1 - fy) + c10 * fy) * (1 - fz) + (c01 * (1 - fy) + c11 * fy) * fz;
              }
              if (v <= tol) m[id(2 * x + i, 2 * y + j, 2 * z + l)] = 1;
            }
          }
      // separable dilation by one point along x, y, z (the 27-neighbourhood)
      for (int ax = 0; ax < 3; ++ax) {
        for (int z = 0; z < nz; ++z)
          for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
              const int c[3] = {x, y, z}, lim[3] = {nx, ny, nz};
              uint8_t v = m[id(x, y, z)];
              if (c[ax] > 0) v |= m[id(x - (ax == 0), y - (ax == 1), z - (ax == 2))];
              if (c[ax] + 1 < lim[ax]) v |= m[id(x + (ax == 0), y + (ax == 1), z + (ax == 2))];
              t[id(x, y, z)] = v;
            }
        m.swap(t);
      }
      for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
          for (int x = 0; x < nx; ++x) {
            if (!m[id(x, y, z)]) continue;
            const bool edge = x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1;
            if (!edge && m[id(x - 1, y, z)] && m[id(x + 1, y, z)] && m[id(x, y - 1, z)] && m[id(x, y + 1, z)] &&
                m[id(x, y, z - 1)] && m[id(x, y, z + 1)])
              continue;
            pts.push_back(make_double3(sh.origin[0] + 0.5 * sh.h * x, sh.origin[1] + 0.5 * sh.h * y,
                                       sh.origin[2] + 0.5 * sh.h * z));
          }
      poff.push_back((long long)pts.size());
    }
    const int ns = (int)s->shapes.size();
    CK(s->sup_pts.upload(pts.data(), pts.size(), st));
    CK(s->sup_off.upload(poff.data(), poff.size(), st));
    CK(s->sup_n.alloc((size_t)ns * SUP_CELLS));
    CK(s->sup_s.alloc((size_t)ns * SUP_CELLS));
    CK(s->sup_r.alloc((size_t)std::max(ns, 1)));
    CK(s->sup_vtx.alloc((size_t)2 * ns * SUP_VERTS));
    launch_support_tables(ns, s->s_node_pos.p, s->s_node_off.p, s->s_node_cnt.p, s->sup_pts.p, s->sup_off.p,
                          s->sup_vtx.p, s->sup_n.p, s->sup_s.p, s->sup_r.p, st);
    CK(cudaGetLastError());
  }
  {
    std::vector<float4> sub;
    for (const ShapeHost& sh : s->shapes)
      for (size_t q = 0; q < sh.sub.size() / 4; ++q) {
        const double r = sh.sub[4 * q + 3];
        sub.push_back(make_float4((float)sh.sub[4 * q], (float)sh.sub[4 * q + 1], (float)sh.sub[4 * q + 2],
                                  r < 0 ? -1.f : (float)(r * (1.0 + 1e-6)) + 1e-30f));
      }
    CK(s->s_sub.upload(sub.data(), sub.size(), st));
  }
  {
    std::vector<double> nbox;
    for (const ShapeHost& sh : s->shapes) {
      double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300}, r2 = 0.;
      for (size_t i = 0; i + 2 < sh.nodes.size(); i += 3) {
        for (int k = 0; k < 3; ++k) {
          lo[k] = std::min(lo[k], sh.nodes[i + k]);
          hi[k] = std::max(hi[k], sh.nodes[i + k]);
        }
        r2 = std::max(r2, sh.nodes[i] * sh.nodes[i] + sh.nodes[i + 1] * sh.nodes[i + 1] + sh.nodes[i + 2] * sh.nodes[i + 2]);
      }
      if (sh.nodes.empty()) for (int k = 0; k < 3; ++k) lo[k] = hi[k] = 0.;
      nbox.insert(nbox.end(), {lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], std::sqrt(r2) * (1.0 + 1e-12), 0.});
    }
    CK(s->s_nbox.upload(nbox.data(), nbox.size(), st));
  }
  {
    // per template, in spacings: the largest difference of neighbouring SDF values
    // (bound of each partial derivative of the trilinear interpolant per grid
    // unit) and the largest gradient-norm bound of a cell, sqrt of the sum over
    // axes of the cell's largest edge difference squared
    std::vector<float> lip;
    for (const ShapeHost& sh : s->shapes) {
      const int nx = sh.size[0], ny = sh.size[1], nz = sh.size[2];
      const size_t sy = (size_t)nx, sz = (size_t)nx * ny;
      auto at = [&](int x, int y, int z) { return sh.sdf[(size_t)x + sy * y + sz * z]; };
      double m = 0., g = 0.;
      for (int z = 0; z + 1 < nz; ++z)
        for (int y = 0; y + 1 < ny; ++y)
          for (int x = 0; x + 1 < nx; ++x) {
            double e[3] = {0., 0., 0.};
            for (int b = 0; b < 4; ++b) {
              const int u = b & 1, v = b >> 1;
              e[0] = std::max(e[0], std::fabs(at(x + 1, y + u, z + v) - at(x, y + u, z + v)));
              e[1] = std::max(e[1], std::fabs(at(x + u, y + 1, z + v) - at(x + u, y, z + v)));
              e[2] = std::max(e[2], std::fabs(at(x + u, y + v, z + 1) - at(x + u, y + v, z)));
            }
            m = std::max(m, std::max(e[0], std::max(e[1], e[2])));
            g = std::max(g, std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]));
          }
      lip.push_back((float)(m / sh.h * (1.0 + 1e-6)));
      lip.push_back((float)(g / sh.h * (1.0 + 1e-6)));
    }
    CK(s->s_lip.upload(lip.data(), lip.size(), st));
  }
  if (s->precision != PREC_FP64) {
    // precision form: phi / h of each template in 16 bits, FP32 node copy
    // cell-major 16-bit store: the 8 corners of cell (i, j, k) in 16 bytes, corner
    // c = dx + 2 dy + 4 dz at 16-bit lane c, cells x-fastest
    std::vector<uint4> cells;
    std::vector<long long> cell_off;
    for (const ShapeHost& sh : s->shapes) {
      const int nx = sh.size[0], ny = sh.size[1], nz = sh.size[2];
      cell_off.push_back((long long)cells.size());
      auto enc = [&](double v) -> unsigned {
        const float u = (float)(v / sh.h);
        unsigned short r;
        if (s->precision == PREC_FP32_BF16) {
          const __nv_bfloat16 b = __float2bfloat16_rn(u);
          std::memcpy(&r, &b, 2);
        } else {
          const __half hh = __float2half_rn(u);
          std::memcpy(&r, &hh, 2);
        }
        return r;
      };
      auto at = [&](int x, int y, int z) { return sh.sdf[(size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z)]; };
      for (int z = 0; z + 1 < nz; ++z)
        for (int y = 0; y + 1 < ny; ++y)
          for (int x = 0; x + 1 < nx; ++x) {
            unsigned c[8];
            for (int q = 0; q < 8; ++q) c[q] = enc(at(x + (q & 1), y + ((q >> 1) & 1), z + (q >> 2)));
            cells.push_back(make_uint4(c[0] | c[1] << 16, c[2] | c[3] << 16, c[4] | c[5] << 16, c[6] | c[7] << 16));
          }
    }
    std::vector<float4> nf(node_pos.size());
    for (size_t i = 0; i < node_pos.size(); ++i)
      nf[i] = make_float4((float)node_pos[i].x, (float)node_pos[i].y, (float)node_pos[i].z, 0.f);
    CK(s->s_cell16.upload(cells.data(), cells.size(), st));
    CK(s->s_cell_off.upload(cell_off.data(), cell_off.size(), st));
    CK(s->s_node_f.upload(nf.data(), nf.size(), st));
  }
  // node ids (LSBoundaryNode order: particle by particle, caller node order)
  s->P.node_base.resize(s->P.n());
  long long nb = 0;
  for (int i = 0; i < s->P.n(); ++i) {
    s->P.node_base[i] = nb;
    nb += (long long)(s->shapes[s->P.shape[i]].nodes.size() / 3);
  }
  upload_bodies(s, s->P, s->dP);
  upload_bodies(s, s->W, s->dW);
  // grids: cell = 2 x max bounding radius (LSParticle.h:241-256)
  double rp = 0., rw = 0.;
  for (double r : s->P.radius) rp = std::max(rp, r);
  s->rmax_p = rp;
  for (double r : s->W.radius) rw = std::max(rw, r);
  set_grid(s->pg, s->dmin, s->dmax, s->P.n() ? 2.0 * rp : 0.0);
  set_grid(s->wg, s->dmin, s->dmax, s->W.n() ? 2.0 * rw : 0.0);
  const int n = s->P.n();
  CK(s->cell_idx.alloc(std::max(n, 1)));
  CK(s->cell_pk.alloc(std::max(n, 1)));
  {
    // neighbour-list margin: a tenth of the largest bounding radius; rebuilt when a
    // particle moved 0.4 of it (pairs approach by at most twice that)
    const double sr = 0.1 * s->rmax_p;
    s->skin = (float)sr;
    s->move2 = (0.4 * sr) * (0.4 * sr);
    CK(s->reuse.alloc(1));
    CK(s->xb.alloc(std::max(n, 1)));
    CK(s->nbr_cnt.alloc(std::max(n, 1)));
    CK(s->pk_meta.alloc(std::max(n, 1)));
    CK(s->pk_q.alloc(std::max(n, 1)));
    CK(s->nbr.alloc((size_t)std::max(n, 1) * s->nbr_cap));
    s->force_reuse = true;
  }
  CK(s->sorted_key.alloc(std::max(n, 1)));
  CK(s->cell_start.alloc(s->pg.ncells));
  CK(s->cell_end.alloc(s->pg.ncells));
  alloc_bucket(s, n, s->pg.ncells);
  // periodic image sets: single axes in x, y, z order, then pairs, then xyz
  s->nsets = 0;
  const int ax = s->periodic & 7;
  const int order[7] = {1, 2, 4, 3, 5, 6, 7};
  for (int k = 0; k < 7; ++k)
    if ((order[k] & ax) == order[k]) s->set_mask[s->nsets++] = order[k];
  if (s->periodic & 8) {  // sector: images turned by 90, 180 and 270 degrees
    s->nsets = 3;
    s->set_mask[0] = 8; s->set_mask[1] = 16; s->set_mask[2] = 32;
    CK(s->gquat.alloc((size_t)3 * std::max(n, 1)));
    CK(s->gvel.alloc((size_t)3 * std::max(n, 1)));
  }
  if (s->nsets > 0) {
    CK(s->gpos.alloc((size_t)s->nsets * std::max(n, 1)));
    CK(s->gkey.alloc((size_t)s->nsets * std::max(n, 1)));
    CK(s->glist.alloc((size_t)s->nsets * std::max(n, 1)));
    CK(s->gcount.alloc(1));
    CK(s->key2.alloc(std::max(n, 1)));
    CK(s->g2_idx.alloc(std::max(n, 1)));
    CK(s->g2_start.alloc(s->pg.ncells));
    CK(s->g2_end.alloc(s->pg.ncells));
    // the image sort's own scratch: the particle sort's offsets stay valid between sorts
    alloc_bucket(s, n, s->pg.ncells, true);
    if (!(s->periodic & 8)) {  // translated images: the parallel branch's own buffers
      CK(s->pos_w.alloc(std::max(n, 1)));
      CK(s->cell_pk2.alloc(std::max(n, 1)));
      if (!s->st2) CK(cudaStreamCreate(&s->st2));
      if (!s->ev_fork) CK(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming));
      if (!s->ev_join) CK(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming));
    }
  }
  // history buffers
  if (s->cap_c <= 0) s->cap_c = std::max<long long>(1 << 16, (long long)n * 128);
  alloc_slots(s);
  alloc_contacts(s, s->con[0], s->cap_c);
  alloc_contacts(s, s->con[1], s->cap_c);
  alloc_maybe(s);
  s->hp = 0;
  s->hist_count = 0;
  if (carry) {
    if (carried > s->con[0].cap) {
      s->cap_c = std::max<long long>(s->cap_c, carried + carried / 2);
      alloc_contacts(s, s->con[0], s->cap_c);
      alloc_contacts(s, s->con[1], s->cap_c);
      alloc_maybe(s);
    }
    s->hist_count = carried;
    restore_history(s, 0);
    const int c32 = (int)carried;
    CK(cudaMemcpyAsync(s->con[0].count.p, &c32, sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    s->force_reuse = true;
  }
  s->net_dirty = true;
  s->dev_np = s->P.n();
  s->dev_nw = s->W.n();
  s->dev_nodes = nodes_now;
  s->dev_nsets = s->nsets;
  s->dev_nb = s->bonds.bonded.size();
  // bonds
  const size_t nbnd = s->bonds.bonded.size();
  if (nbnd) {
    CK(s->b_ids.upload(s->bonds.ids.data(), s->bonds.ids.size(), st));
    CK(s->b_bonded.upload(s->bonds.bonded.data(), nbnd, st));
    CK(s->b_B.upload(s->bonds.B.data(), s->bonds.B.size(), st));
    CK(s->b_geo.upload(s->bonds.geo.data(), s->bonds.geo.size(), st));
    CK(s->b_frames.upload((const double3*)s->bonds.frames.data(), s->bonds.frames.size() / 3, st));
    CK(s->b_state.upload(s->bonds.state.data(), s->bonds.state.size(), st));
  }
  CK(s->status.alloc(1));
  CK(s->status.zero(st));
  if (!s->h_status) CK(cudaMallocHost((void**)&s->h_status, sizeof(Status)));
  if (!s->h_count) CK(cudaMallocHost((void**)&s->h_count, sizeof(int)));
  CK(cudaStreamSynchronize(st));
  s->ready = true;
}

StepArgs make_args(lsdem_solver* s, double dt) {
  StepArgs a{};
  auto bv = [&](BodyDev& D, int n) {
    BodyView v;
    v.n = n;
    v.pos = D.pos.p; v.vel = D.vel.p; v.angvel = D.angvel.p; v.force = D.force.p; v.torque = D.torque.p;
    v.quat = D.quat.p; v.invmass = D.invm.p; v.invI = D.invI.p; v.radius = D.radius.p; v.kn = D.kn.p;
    v.ks = D.ks.p; v.mu = D.mu.p; v.res = D.res.p; v.shape = D.shape.p; v.scale = D.scale.p;
    v.origin = D.origin.p; v.invh = D.invh.p; v.node_base = D.node_base.p; v.key = D.key.p;
    v.rotm = D.rotm.p;
    return v;
  };
  a.P = bv(s->dP, s->P.n());
  a.W = bv(s->dW, s->W.n());
  a.S.gsize = s->s_gsize.p; a.S.sdf_off = s->s_sdf_off.p; a.S.sdf = s->s_sdf.p;
  a.S.node_off = s->s_node_off.p; a.S.node_cnt = s->s_node_cnt.p; a.S.cl_off = s->s_cl_off.p;
  a.S.cl_cnt = s->s_cl_cnt.p; a.S.node_pos = s->s_node_pos.p; a.S.node_orig = s->s_node_orig.p;
  a.S.cl_sphere = s->s_cl.p;
  a.S.cl_sphere_f = s->s_clf.p;
  a.S.node_box = s->s_nbox.p;
  a.S.sub_sphere = s->s_sub.p;
  a.S.cell16 = s->s_cell16.p;
  a.S.cell_off = s->s_cell_off.p;
  a.S.node_pos_f = s->s_node_f.p;
  a.S.lip = s->s_lip.p;
  a.S.sup_n = s->sup_n.p;
  a.S.sup_s = s->sup_s.p;
  a.S.sup_r = s->sup_r.p;
  a.pg = s->pg;
  a.wg = s->wg;
  a.cell_idx = s->cell_idx.p; a.cell_start = s->cell_start.p; a.cell_end = s->cell_end.p;
  a.cell_pk = s->cell_pk.p;
  a.cell_off = s->bk_offs.p;
  auto sv = [](SlotsDev& d) {
    SlotView v;
    v.cap = d.cap; v.cnt = d.cnt.p; v.id = d.id.p; v.seg_start = d.seg_start.p; v.seg_cnt = d.seg_cnt.p;
    return v;
  };
  const int cur = 1 - s->hp, old = s->hp;
  a.pp = sv(s->slots[cur][0]); a.pw = sv(s->slots[cur][1]); a.pgh = sv(s->slots[cur][2]);
  a.pp_old = sv(s->slots[old][0]); a.pw_old = sv(s->slots[old][1]); a.pgh_old = sv(s->slots[old][2]);
  auto cv = [](ContactsDev& c, bool geom) {
    ContactView v;
    v.cap = (int)std::min<long long>(c.cap, 0x7fffffff);
    v.count = c.count.p; v.node = c.node.p; v.spring = c.spring.p;
    v.point = geom ? c.point.p : nullptr; v.normal = geom ? c.normal.p : nullptr;
    v.overlap = geom ? c.overlap.p : nullptr; v.en_n = geom ? c.en_n.p : nullptr; v.en_s = geom ? c.en_s.p : nullptr;
    return v;
  };
  a.C = cv(s->con[cur], false);
  a.C_old = cv(s->con[old], false);
  a.G.nsets = s->nsets;
  for (int k = 0; k < 7; ++k) a.G.mask[k] = s->set_mask[k];
  a.G.sector = (s->periodic & 8) ? 1 : 0;
  a.G.gquat = s->gquat.p;
  a.G.gvel = s->gvel.p;
  a.G.gpos = s->gpos.p;
  a.G.gkey = s->gkey.p;
  a.G.list = s->glist.p;
  a.G.count = s->gcount.p;
  a.status = s->status.p;
  a.dt = dt;
  a.gravity = make_double3(s->grav[0], s->grav[1], s->grav[2]);
  a.flags = s->flags;
  a.precision = s->precision;
  a.rmax = s->rmax_p;
  const bool reuse = s->reuse_on && s->reuse.p;
  a.reuse = reuse ? s->reuse.p : nullptr;
  a.move2 = s->move2;
  a.skin = s->skin;
  a.xb = s->xb.p;
  a.nbr = reuse ? s->nbr.p : nullptr;
  a.nbr_cnt = s->nbr_cnt.p;
  a.nbr_cap = s->nbr_cap;
  a.pk_meta = s->pk_meta.p;
  a.pk_q = s->pk_q.p;
  a.mb.node = s->mb_node.p; a.mb.cap = (int)s->mb_cap;
  a.mb.pair = s->mb_pair.p; a.mb.pcap = (int)s->mb_pcap;
  a.mb.ctr = s->precision == PREC_FP64 ? nullptr : s->mb_ctr.p;
  for (int k = 0; k < 3; ++k) a.pl.list[k] = s->plist[k].p;
  a.pl.ctr = s->precision == PREC_FP64 ? nullptr : s->pl_ctr.p;
  a.screen_stats = s->scr_stats.p;
  const bool learned = s->mlp_on && s->mlp_trained && s->precision != PREC_FP64;
  a.mlp_inf = learned ? s->mlp_inf.p : nullptr;
  a.mlp_norm = s->mlp_norm.p;
  a.mlp_band = s->mlp_band.p;
  a.nshapes = (int)s->shapes.size();
  for (int l = 0; l < 2; ++l) {
    auto& N = s->net[l];
    NetView& v = a.net[l];
    v = NetView{};
    if (!learned || !N.ctr.p) continue;
    v.row = N.row.p; v.cnt = N.cnt.p; v.qcap = N.qcap;
    v.pend_n = N.pend_n.p; v.pend_v = N.pend_v.p; v.pcap = N.pcap;
    v.pair = N.pair.p; v.paircap = N.paircap; v.ctr = N.ctr.p;
  }
  return a;
}

// Phase timing: events recorded on the solver stream around each phase;
// resolved after the batch synchronisation.
cudaEvent_t pool_event(lsdem_solver* s) {
  if (!s->event_pool.empty()) {
    cudaEvent_t e = s->event_pool.back();
    s->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  CK(cudaEventCreate(&e));
  return e;
}
struct PhaseTimer {
  lsdem_solver* s;
  int id;
  cudaEvent_t a = nullptr, b = nullptr;
  PhaseTimer(lsdem_solver* s_, int id_) : s(s_), id(id_) {
    if (!s->profiling) return;
    a = pool_event(s);
    b = pool_event(s);
    CK(cudaEventRecord(a, s->stream));
  }
  ~PhaseTimer() {
    if (!a) return;
    cudaEventRecord(b, s->stream);
    s->prof_pending.push_back({id, {a, b}});
  }
};
void resolve_profile(lsdem_solver* s, bool keep) {
  for (auto& p : s->prof_pending) {
    if (keep) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, p.second.first, p.second.second);
      s->prof_ms[p.first] += ms;
      s->prof_calls[p.first] += 1;
    }
    s->event_pool.push_back(p.second.first);
    s->event_pool.push_back(p.second.second);
  }
  s->prof_pending.clear();
}

// One time step in the reference order (LSSolver.h:1000-1011, 1104-1128).
// The launches of one step up to the external-force hook: integration, cell sort,
// candidates, narrowphase and contact forces, periodic images, bonds.
void step_pre(lsdem_solver* s, double dt, bool record) {
  cudaStream_t st = s->stream;
  StepArgs a = make_args(s, dt);
  if (record) {
    ContactsDev& c = s->con[1 - s->hp];
    ensure_geom(s, c);
    a.C.point = c.point.p; a.C.normal = c.normal.p; a.C.overlap = c.overlap.p; a.C.en_n = c.en_n.p;
    a.C.en_s = c.en_s.p;
  }
  { PhaseTimer pt(s, 0); launch_integrate_first(a, st); }
  BucketScratch w{s->bk_counts.p, s->bk_fill.p, s->bk_offs.p, s->bk_scan.p, s->bk_big.p, s->bk_bigc.p, s->bk_tmp.p};
  {
    PhaseTimer pt(s, 1);
    bucket_sort(a.P.key, a.P.n, s->pg.ncells, w, s->cell_idx.p, s->sorted_key.p, s->cell_start.p, s->cell_end.p, st,
                a.reuse);
  }
  BucketScratch w2{s->bk2_counts.p, s->bk2_fill.p, s->bk2_offs.p, s->bk2_scan.p, s->bk2_big.p, s->bk2_bigc.p,
                   s->bk2_tmp.p};
  const bool branch = s->nsets > 0 && !(s->periodic & 8) && !s->profiling;
  if (branch) {
    // The periodic images run beside the particle candidates, screen and contact
    // pass, which read the pre-wrap positions: the image branch writes the wrapped
    // positions into pos_w and screens the images against them (its own sort scratch,
    // packed cells, pair list, slots and contact-pass queue; forces and contacts are
    // added with atomics). Joined, the wrapped positions are copied over.
    StepArgs a2 = a;
    a2.P.pos = s->pos_w.p;
    a2.cell_pk = s->cell_pk2.p;
    a2.pk_meta = nullptr;
    cudaStream_t s2 = s->st2;
    CK(cudaEventRecord(s->ev_fork, st));
    CK(cudaStreamWaitEvent(s2, s->ev_fork, 0));
    launch_periodic(a, s->periodic, s->pos_w.p, s2);
    launch_clamped_keys(a2, s->key2.p, s2);
    bucket_sort(s->key2.p, a.P.n, s->pg.ncells, w2, s->g2_idx.p, nullptr, s->g2_start.p, s->g2_end.p, s2);
    launch_ghost_candidates(a2, s->g2_idx.p, w2.offs, s2);
    launch_narrowphase(a2, 4, s2);
    launch_net_screen(a2, 1, s2);
    launch_net_compact(a2, 1, s2);
    if (s->precision != PREC_FP64) launch_contact_pass(a2, 1, s2);
    CK(cudaEventRecord(s->ev_join, s2));
    launch_candidates(a, st);
    launch_narrowphase(a, s->W.n() > 0 ? 3 : 1, st);
    launch_net_screen(a, 0, st);
    launch_net_compact(a, 0, st);
    if (s->precision != PREC_FP64) launch_contact_pass(a, 0, st);
    CK(cudaStreamWaitEvent(st, s->ev_join, 0));
    if (a.P.n > 0) CK(cudaMemcpyAsync(a.P.pos, s->pos_w.p, sizeof(double3) * a.P.n, cudaMemcpyDeviceToDevice, st));
  } else {
    { PhaseTimer pt(s, 2); launch_candidates(a, st); }
    { PhaseTimer pt(s, 3); launch_narrowphase(a, s->W.n() > 0 ? 3 : 1, st); }
    if (a.mlp_inf) { PhaseTimer pt(s, 10); launch_net_screen(a, 0, st); }
    if (s->precision != PREC_FP64) {
      PhaseTimer pt(s, 8);
      launch_net_compact(a, 0, st);
      launch_contact_pass(a, 0, st);
    }
    if (s->nsets > 0) {
      {
        PhaseTimer pt(s, 4);
        launch_periodic(a, s->periodic, a.P.pos, st);
        launch_clamped_keys(a, s->key2.p, st);
        bucket_sort(s->key2.p, a.P.n, s->pg.ncells, w2, s->g2_idx.p, nullptr, s->g2_start.p, s->g2_end.p, st);
        launch_ghost_candidates(a, s->g2_idx.p, w2.offs, st);
      }
      { PhaseTimer pt(s, 5); launch_narrowphase(a, 4, st); }
      if (a.mlp_inf) { PhaseTimer pt(s, 10); launch_net_screen(a, 1, st); }
      if (s->precision != PREC_FP64) {
        PhaseTimer pt(s, 8);
        launch_net_compact(a, 1, st);
        launch_contact_pass(a, 1, st);
      }
    }
  }
  if (!s->bonds.bonded.empty()) {
    PhaseTimer pt(s, 6);
    BondView b{(int)s->bonds.bonded.size(), s->b_ids.p, s->b_B.p, s->b_geo.p, s->b_frames.p, s->b_bonded.p,
               s->b_state.p};
    launch_bonds(a, b, st);
  }
  // kernels launched up to here: kick/drift/keys, cell sort (10; with neighbour lists
  // they return at once between rebuilds), packing + candidates, narrowphase; periodic:
  // wrap/images, clamped keys, cell sort (9), image compaction + packing + candidates,
  // ghost narrowphase; bonds. The precision forms add one contact pass per narrowphase
  // and a separate wall screen; the learned form the network pass and the compaction
  // after each screen.
  const bool fp32 = s->precision != PREC_FP64;
  const int lrn = a.mlp_inf ? 2 : 0;
  const int nf = fp32 ? 1 + (s->W.n() > 0 ? 1 : 0) + lrn : 0;
  const int ng = fp32 ? 1 + lrn : 0;
  if (a.P.n > 0) s->launches += 14 + nf + (s->nsets > 0 ? 15 + ng : 0) + (s->bonds.bonded.empty() ? 0 : 1);
  CK(cudaGetLastError());
}

// The rest of a step after the hook: the second half kick.
void step_post(lsdem_solver* s, double dt) {
  StepArgs a = make_args(s, dt);
  { PhaseTimer pt(s, 7); launch_kick(a, s->stream); }
  if (a.P.n > 0) s->launches += 1;
  CK(cudaGetLastError());
  s->hp = 1 - s->hp;
}

void step_once(lsdem_solver* s, double dt, bool record, lsdem_hook hook, void* user, double t) {
  step_pre(s, dt, record);
  if (hook) hook(user, t);
  step_post(s, dt);
}

// Snapshot of everything a batch may change, taken at the batch start.
void backup_state(lsdem_solver* s);
void backup(lsdem_solver* s) {
  backup_state(s);
  backup_history(s);
}

// Body state and bond flags (what one step changes besides the new contact list).
void backup_state(lsdem_solver* s) {
  cudaStream_t st = s->stream;
  const size_t n = (size_t)s->P.n(), nw = (size_t)s->W.n();
  // backup buffers grow geometrically (never per batch: a free synchronises the device)
  auto cp = [&](auto& dst, auto& src, size_t m) {
    if (dst.n < m) CK(dst.alloc(std::max(m + m / 2, (size_t)1024)));
    if (m) CK(cudaMemcpyAsync(dst.p, src.p, m * sizeof(*src.p), cudaMemcpyDeviceToDevice, st));
  };
  cp(s->bk_pos, s->dP.pos, n); cp(s->bk_vel, s->dP.vel, n); cp(s->bk_angvel, s->dP.angvel, n);
  cp(s->bk_quat, s->dP.quat, n); cp(s->bk_force, s->dP.force, n); cp(s->bk_torque, s->dP.torque, n);
  cp(s->bk_wpos, s->dW.pos, nw); cp(s->bk_wquat, s->dW.quat, nw);
  cp(s->bk_bonded, s->b_bonded, s->bonds.bonded.size());
}

// The contact history of the last step (candidate slots with their contact segments,
// contact nodes and springs) into the backup buffers.
void backup_history(lsdem_solver* s) {
  cudaStream_t st = s->stream;
  const size_t n = (size_t)s->P.n();
  auto cp = [&](auto& dst, auto& src, size_t m) {
    if (dst.n < m) CK(dst.alloc(std::max(m + m / 2, (size_t)1024)));
    if (m) CK(cudaMemcpyAsync(dst.p, src.p, m * sizeof(*src.p), cudaMemcpyDeviceToDevice, st));
  };
  for (int k = 0; k < 3; ++k) {
    SlotsDev& sl = s->slots[s->hp][k];
    s->bk_cap[k] = sl.cap;
    if (!sl.cnt.p) continue;
    cp(s->bk_slot[k][0], sl.cnt, n);
    cp(s->bk_slot[k][1], sl.id, n * sl.cap);
    cp(s->bk_slot[k][2], sl.seg_start, n * sl.cap);
    cp(s->bk_slot[k][3], sl.seg_cnt, n * sl.cap);
  }
  const size_t nc = (size_t)s->hist_count;
  cp(s->bk_cnode, s->con[s->hp].node, nc);
  cp(s->bk_cspring, s->con[s->hp].spring, nc);
}

void restore_state(lsdem_solver* s, int hp0);
void restore(lsdem_solver* s, int hp0) {
  restore_state(s, hp0);
  restore_history(s, hp0);
}

void restore_state(lsdem_solver* s, int hp0) {
  s->force_reuse = true;
  cudaStream_t st = s->stream;
  s->hp = hp0;
  const size_t n = (size_t)s->P.n(), nw = (size_t)s->W.n();
  auto cp = [&](auto& dst, auto& src, size_t m) {
    if (m) CK(cudaMemcpyAsync(dst.p, src.p, m * sizeof(*src.p), cudaMemcpyDeviceToDevice, st));
  };
  cp(s->dP.pos, s->bk_pos, n); cp(s->dP.vel, s->bk_vel, n); cp(s->dP.angvel, s->bk_angvel, n);
  cp(s->dP.quat, s->bk_quat, n); cp(s->dP.force, s->bk_force, n); cp(s->dP.torque, s->bk_torque, n);
  cp(s->dW.pos, s->bk_wpos, nw); cp(s->dW.quat, s->bk_wquat, nw);
  cp(s->b_bonded, s->bk_bonded, s->bonds.bonded.size());
}

// The backed-up contact history into the buffers of parity hp0 (capacities may have
// grown since the backup: slots are copied row by row).
void restore_history(lsdem_solver* s, int hp0) {
  cudaStream_t st = s->stream;
  const size_t n = (size_t)s->P.n();
  auto cp = [&](auto& dst, auto& src, size_t m) {
    if (m) CK(cudaMemcpyAsync(dst.p, src.p, m * sizeof(*src.p), cudaMemcpyDeviceToDevice, st));
  };
  for (int k = 0; k < 3; ++k) {
    SlotsDev& sl = s->slots[hp0][k];
    if (!sl.cnt.p) continue;
    const int oc = s->bk_cap[k];
    cp(sl.cnt, s->bk_slot[k][0], n);
    if (oc > 0 && n > 0) {
      for (int a = 1; a < 4; ++a) {
        DArr<int>& dst = a == 1 ? sl.id : (a == 2 ? sl.seg_start : sl.seg_cnt);
        CK(cudaMemcpy2DAsync(dst.p, sizeof(int) * sl.cap, s->bk_slot[k][a].p, sizeof(int) * oc,
                             sizeof(int) * std::min(oc, sl.cap), n, cudaMemcpyDeviceToDevice, st));
      }
    }
  }
  const size_t nc = (size_t)s->hist_count;
  cp(s->con[hp0].node, s->bk_cnode, nc);
  cp(s->con[hp0].spring, s->bk_cspring, nc);
}

// New capacities from the largest demands of the last batch: a capacity
// grows when it overflowed or when the demand passed 80 % of it (so that the
// next batch is unlikely to overflow). Returns true when any capacity changes.
bool plan_growth(lsdem_solver* s, const Status& st, long long last_contacts) {
  bool changed = false;
  auto up = [&](int& cap, int need, bool ovf) {
    if (ovf || need * 5 > cap * 4) {
      const int nc = std::max(cap * 2, need + need / 2 + 4);
      if (nc != cap) { cap = nc; changed = true; }
    }
  };
  up(s->cap_pp, st.need_pp, st.flags & OVF_PP);
  if (s->W.n() > 0) up(s->cap_w, st.need_wall, st.flags & OVF_WALL);
  if (s->nsets > 0) up(s->cap_g, st.need_ghost, st.flags & OVF_GHOST);
  if (s->reuse_on) {
    const int old = s->nbr_cap;
    up(s->nbr_cap, st.need_nbr, st.flags & OVF_NBR);
    if (s->nbr_cap != old) s->grow_nbr = true;
  }
  const long long needc = std::max<long long>(st.need_contact, last_contacts);
  if ((st.flags & OVF_CONTACT) || needc * 5 > s->cap_c * 4) {
    s->cap_c = std::max<long long>(s->cap_c * 2, needc + needc / 2 + 1024);
    changed = true;
    s->grow_contacts = true;
  }
  if (changed) s->net_dirty = true;  // pair records are sized with the candidate slots
  // learned form: network rows per shape and pending nodes
  auto up64 = [&](long long& cap, long long need) {
    if (need * 5 > cap * 4) {
      cap = std::max<long long>(cap * 2, need + need / 2 + 1024);
      changed = true;
      s->net_dirty = true;
    }
  };
  if (s->net[0].ctr.p) {
    up64(s->cap_netq, st.need_netq);
    up64(s->cap_pend, st.need_pend);
    if ((st.flags & OVF_NET) && !s->net_dirty) {  // overflowed without a recorded demand: double both
      s->cap_netq *= 2;
      s->cap_pend *= 2;
      s->net_dirty = changed = true;
    }
  }
  return changed;
}

// Reallocates slot arrays of both parities (and both contact lists when they
// grow); their contents come back from the backup by restore().
void grow(lsdem_solver* s) {
  ++s->graph_gen;
  s->force_reuse = true;
  if (s->net_dirty && s->net[0].ctr.p) alloc_net(s);
  if (s->grow_nbr) {
    CK(s->nbr.alloc((size_t)std::max(s->P.n(), 1) * s->nbr_cap));
    s->grow_nbr = false;
  }
  alloc_slots(s, true);
  if (s->grow_contacts) {
    const bool g0 = s->con[0].geom, g1 = s->con[1].geom;
    alloc_contacts(s, s->con[0], s->cap_c);
    alloc_contacts(s, s->con[1], s->cap_c);
    if (g0) ensure_geom(s, s->con[0]);
    if (g1) ensure_geom(s, s->con[1]);
    alloc_maybe(s);
    s->grow_contacts = false;
  }
}

// Step timing: L2 flush (when a buffer is set) and the step's start event.
cudaEvent_t step_start(lsdem_solver* s) {
  if (s->flush_buf.n) CK(cudaMemsetAsync(s->flush_buf.p, (int)(s->steps & 0xff), s->flush_buf.n, s->stream));
  cudaEvent_t e = pool_event(s);
  CK(cudaEventRecord(e, s->stream));
  return e;
}

// One step replayed from a CUDA graph: the launches of step_once captured once per
// history parity and key (the generation of the step's arguments, dt, capacities),
// then launched as one unit, which removes the per-launch host cost and most of the
// gaps between the step's ~30 short kernels. On the legacy default stream (which
// cannot be captured) the graph runs on a private blocking stream: the legacy stream
// and blocking streams are ordered with each other both ways, so the copies, events
// and app kernels on the legacy stream keep their order around the step.
static void step_graph_pre(lsdem_solver* s, double dt) {
  const int hp = s->hp;
  uint64_t key = 1469598103934665603ull;
  auto mix = [&](uint64_t v) { key = (key ^ v) * 1099511628211ull; };
  uint64_t dtb;
  std::memcpy(&dtb, &dt, 8);
  mix((uint64_t)s->graph_gen); mix(dtb); mix((uint64_t)s->P.n()); mix((uint64_t)s->W.n());
  mix((uint64_t)s->nsets); mix((uint64_t)s->bonds.bonded.size()); mix((uint64_t)s->precision);
  mix((uint64_t)s->flags); mix((uint64_t)s->mb_cap); mix((uint64_t)s->mb_pcap);
  mix((uint64_t)s->cap_pp); mix((uint64_t)s->cap_w); mix((uint64_t)s->cap_g); mix((uint64_t)s->cap_c);
  mix((uint64_t)s->mlp_on); mix((uint64_t)(s->scr_stats.p != nullptr)); mix((uint64_t)s->periodic);
  mix((uint64_t)s->cap_netq); mix((uint64_t)s->cap_pend); mix((uint64_t)(uintptr_t)s->net[0].row.p);
  if (!s->stream && !s->gstream) CK(cudaStreamCreate(&s->gstream));
  cudaStream_t gs = s->stream ? s->stream : s->gstream;
  lsdem_solver::StepGraph& G = s->sgraph[hp];
  if (!G.exec || G.key != key) {
    if (G.exec) { cudaGraphExecDestroy(G.exec); G.exec = nullptr; }
    const long long l0 = s->launches;
    cudaStream_t saved = s->stream;
    s->stream = gs;
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(gs, cudaStreamCaptureModeRelaxed));
    try {
      step_pre(s, dt, false);
    } catch (...) {
      cudaStreamEndCapture(gs, &graph);
      if (graph) cudaGraphDestroy(graph);
      s->stream = saved;
      s->hp = hp;
      throw;
    }
    s->stream = saved;
    CK(cudaStreamEndCapture(gs, &graph));
    const cudaError_t e = cudaGraphInstantiate(&G.exec, graph, 0);
    cudaGraphDestroy(graph);
    CK(e);
    G.key = key;
    G.launches = s->launches - l0;
    s->launches = l0;
    s->hp = hp;  // the capture did not run the step
  }
  CK(cudaGraphLaunch(G.exec, gs));
  s->launches += G.launches;
}

static void step_graph(lsdem_solver* s, double dt, lsdem_hook hook, void* user, double t) {
  step_graph_pre(s, dt);
  if (hook) hook(user, t);
  step_post(s, dt);
}

// Steps with an external-force hook: each step's capacity status is read before its hook
// runs (one host synchronisation per step, as the reference's per-step count reads), and a
// step that overflowed is re-run with grown capacities first, so the hook runs exactly once
// per step, after the step's complete contact and bond forces (LSSolver.h:1000-1011).
static int run_steps_hooked(lsdem_solver* s, double dt, long long nsteps, lsdem_hook hook, void* user) {
  cudaStream_t st = s->stream;
  for (long long k = 0; k < nsteps; ++k) {
    const bool rec = s->record && (k == nsteps - 1);
    const int hp0 = s->hp;
    cudaEvent_t ea = s->step_timing ? step_start(s) : nullptr;
    // the step leaves the history of parity hp0 untouched until step_post: only the body
    // state is saved per step, the history only before a re-allocation
    backup_state(s);
    Status stat{};
    for (int attempt = 0;; ++attempt) {
      CK(cudaMemsetAsync(s->status.p, 0, sizeof(Status), st));
      if (s->force_reuse && s->reuse.p) {  // sort and rebuild in this step
        CK(cudaMemsetAsync(s->reuse.p, 0xff, sizeof(int), st));
        s->force_reuse = false;
      }
      if (s->graphs && !rec && !s->profiling && s->P.n() > 0) step_graph_pre(s, dt);
      else step_pre(s, dt, rec);
      // this step's contacts are in the buffer of the other parity until step_post
      CK(cudaMemcpyAsync(s->h_status, s->status.p, sizeof(Status), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(s->h_count, s->con[1 - s->hp].count.p, sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      stat = *s->h_status;
      if (stat.errors) throw Fail{LSDEM_ERR_CUDA, "a tensor-core wait in the network pass gave up"};
      resolve_profile(s, stat.flags == 0);  // every pending event has completed
      if (stat.flags == 0) break;
      if (attempt > 8) throw Fail{LSDEM_ERR_NOMEM, "capacity growth did not converge"};
      plan_growth(s, stat, *s->h_count);
      backup_history(s);
      grow(s);
      restore(s, hp0);
      s->reruns++;
    }
    const long long count = *s->h_count;
    hook(user, s->time);
    step_post(s, dt);
    if (ea) {
      cudaEvent_t eb = pool_event(s);
      CK(cudaEventRecord(eb, st));
      s->prof_pending.push_back({9, {ea, eb}});  // resolved after the next synchronisation
    }
    s->hist_count = count;
    s->steps += 1;
    s->time += dt;
    s->builds += stat.builds;
    if (plan_growth(s, stat, s->hist_count)) {
      const int hp1 = s->hp;
      backup(s);
      grow(s);
      restore(s, hp1);
    }
  }
  CK(cudaStreamSynchronize(st));
  resolve_profile(s, true);
  s->host_stale = true;
  return LSDEM_OK;
}

int run_steps(lsdem_solver* s, double dt, long long nsteps, lsdem_hook hook, void* user) {
  if (!s->ready) throw Fail{LSDEM_ERR_STATE, "lsdem_step before lsdem_initialize"};
  if (!(dt > 0.)) throw Fail{LSDEM_ERR_ARG, "Invalid timeStep"};
  const bool learned = s->mlp_on && s->mlp_trained && s->precision != PREC_FP64;
  if (learned && (s->net_dirty || !s->net[0].ctr.p)) {
    alloc_net(s);
    ++s->graph_gen;
  }
  if (hook) return run_steps_hooked(s, dt, nsteps, hook, user);
  cudaStream_t st = s->stream;
  long long done = 0;
  while (done < nsteps) {
    const long long B = std::min<long long>(std::max(1, std::min(s->cur_batch, s->batch)), nsteps - done);
    const int hp0 = s->hp;
    // the batch's state backup is timed with its first step
    cudaEvent_t first = s->step_timing ? step_start(s) : nullptr;
    backup(s);
    Status stat{};
    for (int attempt = 0;; ++attempt) {
      CK(cudaMemsetAsync(s->status.p, 0, sizeof(Status), st));
      double t = s->time;
      for (long long k = 0; k < B; ++k) {
        const bool rec = s->record && (done + k == nsteps - 1);
        cudaEvent_t ea = nullptr;
        if (s->step_timing) ea = (k == 0 && attempt == 0) ? first : step_start(s);
        if (s->force_reuse && s->reuse.p) {  // sort and rebuild in this step
          CK(cudaMemsetAsync(s->reuse.p, 0xff, sizeof(int), st));
          s->force_reuse = false;
        }
        if (s->graphs && !rec && !s->profiling && s->P.n() > 0)
          step_graph(s, dt, hook, user, t);
        else
          step_once(s, dt, rec, hook, user, t);
        if (ea) {
          cudaEvent_t eb = pool_event(s);
          CK(cudaEventRecord(eb, st));
          s->prof_pending.push_back({9, {ea, eb}});
        }
        t += dt;
      }
      CK(cudaMemcpyAsync(s->h_status, s->status.p, sizeof(Status), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(s->h_count, s->con[s->hp].count.p, sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      stat = *s->h_status;
      if (stat.errors) throw Fail{LSDEM_ERR_CUDA, "a tensor-core wait in the network pass gave up"};
      resolve_profile(s, stat.flags == 0);
      if (stat.flags == 0) {
        s->hist_count = *s->h_count;
        break;
      }
      if (attempt > 8) throw Fail{LSDEM_ERR_NOMEM, "capacity growth did not converge"};
      plan_growth(s, stat, *s->h_count);
      grow(s);
      restore(s, hp0);
      s->reruns++;
      s->cur_batch = 1;
    }
    done += B;
    s->steps += B;
    s->time += dt * (double)B;
    s->builds += stat.builds;
    // grow ahead of an overflow: keep the history just written
    if (plan_growth(s, stat, s->hist_count)) {
      const int hp1 = s->hp;
      backup(s);
      grow(s);
      restore(s, hp1);
    } else {
      s->cur_batch = std::min(s->batch, s->cur_batch * 2);
    }
  }
  s->host_stale = true;
  return LSDEM_OK;
}

template <class T>
std::vector<T> dl(const DArr<T>& d, size_t n, cudaStream_t st) {
  std::vector<T> h(n);
  if (n) CK(cudaMemcpyAsync(h.data(), d.p, n * sizeof(T), cudaMemcpyDeviceToHost, st));
  return h;
}

}  // namespace

namespace {
// Walks the history buffer of the last step: owner A, slot j, segment.
template <class F>
void walk_contacts(lsdem_solver* s, int kind, F&& f) {
  cudaStream_t st = s->stream;
  const int n = s->P.n();
  SlotsDev& sl = s->slots[s->hp][kind];
  if (!sl.cnt.p || sl.cap == 0) return;
  auto cnt = dl(sl.cnt, (size_t)n, st);
  auto id = dl(sl.id, (size_t)n * sl.cap, st);
  auto ss = dl(sl.seg_start, (size_t)n * sl.cap, st);
  auto sc = dl(sl.seg_cnt, (size_t)n * sl.cap, st);
  CK(cudaStreamSynchronize(st));
  for (int A = 0; A < n; ++A) {
    const int m = std::min(cnt[A], sl.cap);
    for (int j = 0; j < m; ++j) {
      const size_t k = (size_t)A * sl.cap + j;
      f(A, id[k], ss[k], sc[k]);
    }
  }
}

}  // namespace

// ===========================================================================
extern "C" {

int lsdem_create(int device, void* stream, lsdem_solver** out) {
  if (!out) return LSDEM_ERR_ARG;
  lsdem_solver* s = new lsdem_solver();
  s->device = device;
  s->stream = (cudaStream_t)stream;
  *out = s;
  return LSDEM_OK;
}

void lsdem_destroy(lsdem_solver* s) {
  if (!s) return;
  if (s->ready) cudaStreamSynchronize(s->stream);
  if (s->vtu) vtu_free(s->vtu);
  for (auto& g : s->sgraph)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (s->gstream) cudaStreamDestroy(s->gstream);
  if (s->st2) cudaStreamDestroy(s->st2);
  if (s->ev_fork) cudaEventDestroy(s->ev_fork);
  if (s->ev_join) cudaEventDestroy(s->ev_join);
  delete s;
}

const char* lsdem_last_error(const lsdem_solver* s) { return s ? s->err.c_str() : "null solver"; }

int lsdem_set_flags(lsdem_solver* s, int flags) {
  if (s) ++s->graph_gen;
  if (!s) return LSDEM_ERR_ARG;
  s->flags = flags & (FIX_GRADIENT | FIX_SQRTF);
  return LSDEM_OK;
}

int lsdem_mass_properties(const double* sdf, const int* size3, const double* origin3, double spacing, double density,
                          double* out16) {
  if (!sdf || !size3 || !origin3 || !out16) return LSDEM_ERR_ARG;
  if (size3[0] < 2 || size3[1] < 2 || size3[2] < 2 || !(spacing > 0.)) return LSDEM_ERR_ARG;
  mass_props(sdf, size3, origin3, spacing, density, out16);
  return LSDEM_OK;
}

int lsdem_add_shape(lsdem_solver* s, const double* nodes, int n_nodes, const double* sdf, const int* size3,
                    const double* origin3, double spacing, int* shape_id) {
  if (!s || !sdf || !size3 || !origin3 || (n_nodes > 0 && !nodes)) return fail(s, LSDEM_ERR_ARG, "null argument");
  return guard(s, [&] {
    int id = add_shape_impl(s, nodes, n_nodes, sdf, size3, origin3, spacing);
    if (shape_id) *shape_id = id;
    return LSDEM_OK;
  });
}

int lsdem_add_particles(lsdem_solver* s, int n, const int* shape, const double* scale, const double* pos,
                        const double* vel, const double* angvel, const double* quat, const double* inv_mass,
                        const double* inv_inertia6, const double* kn, const double* ks, const double* mu,
                        const double* e, int* first_index) {
  if (!s || n < 0 || !shape || !pos || !quat || !inv_mass || !kn || !ks || !mu || !e)
    return fail(s, LSDEM_ERR_ARG, "null argument");
  return guard(s, [&] {
    pull_host(s);
    for (int i = 0; i < n; ++i)
      if (shape[i] < 0 || shape[i] >= (int)s->shapes.size()) throw Fail{LSDEM_ERR_ARG, "unknown shape id"};
    if (first_index) *first_index = s->P.n();
    for (int i = 0; i < n; ++i) {
      const double sc = scale ? scale[i] : 1.0;
      if (!(sc > 0.)) throw Fail{LSDEM_ERR_ARG, "scale must be > 0"};
      push_body(s, s->P, shape[i], sc, pos + 3 * i, vel ? vel + 3 * i : nullptr, angvel ? angvel + 3 * i : nullptr,
                quat + 4 * i, inv_mass[i], inv_inertia6 ? inv_inertia6 + 6 * i : nullptr, kn[i], ks[i], mu[i], e[i],
                shape_radius(s, shape[i], sc));
    }
    s->ready = false;
    return LSDEM_OK;
  });
}

int lsdem_add_ls_particle(lsdem_solver* s, const double* nodes, int n_nodes, const double* sdf, const int* size3,
                          const double* origin3, double spacing, const double* pos, const double* vel,
                          const double* angvel, const double* quat, double kn, double ks, double mu, double e,
                          double density, int* index) {
  if (!s || !sdf || !size3 || !origin3 || !pos || !quat) return fail(s, LSDEM_ERR_ARG, "null argument");
  return guard(s, [&] {
    pull_host(s);
    if (size3[0] < 2 || size3[1] < 2 || size3[2] < 2) throw Fail{LSDEM_ERR_ARG, "Invalid level-set grid size"};
    if (!(spacing > 0.)) throw Fail{LSDEM_ERR_ARG, "Invalid level-set grid spacing"};
    double mp[16];
    mass_props(sdf, size3, origin3, spacing, density, mp);
    const double mass = mp[0];
    const double c[3] = {mp[1], mp[2], mp[3]};
    double qn[4];
    qnormalize(quat, qn);
    V3 off = hrotate(qn, V3{c[0], c[1], c[2]});
    const double pnew[3] = {pos[0] + off.x, pos[1] + off.y, pos[2] + off.z};
    std::vector<double> nn(3 * (size_t)n_nodes);
    for (int i = 0; i < n_nodes; ++i)
      for (int a = 0; a < 3; ++a) nn[3 * i + a] = nodes[3 * i + a] - c[a];
    const double onew[3] = {origin3[0] - c[0], origin3[1] - c[1], origin3[2] - c[2]};
    const int sh = add_shape_impl(s, nn.data(), n_nodes, sdf, size3, onew, spacing);
    if (index) *index = s->P.n();
    const double invm = mass > 0. ? 1. / mass : 0.;
    push_body(s, s->P, sh, 1.0, pnew, vel, angvel, qn, invm, mp + 10, kn, ks, mu, e, shape_radius(s, sh, 1.0));
    s->ready = false;
    return LSDEM_OK;
  });
}

int lsdem_add_wall(lsdem_solver* s, const double* verts, int n_verts, const double* sdf, const int* size3,
                   const double* origin3, double spacing, const double* pos, const double* quat, double mu, double e,
                   int* index) {
  if (!s || !sdf || !size3 || !origin3 || !pos || !quat || (n_verts > 0 && !verts))
    return fail(s, LSDEM_ERR_ARG, "null argument");
  return guard(s, [&] {
    pull_host(s);
    // walls keep their vertices as nodes (LSSolver.h:255-271); only the radius uses them
    const int sh = add_shape_impl(s, verts, 0, sdf, size3, origin3, spacing);
    double r = 0.;
    for (int i = 0; i < n_verts; ++i) r = std::max(r, hlen(v3(verts + 3 * i)));
    if (index) *index = s->W.n();
    push_body(s, s->W, sh, 1.0, pos, nullptr, nullptr, quat, 0., nullptr, 0., 0., mu, e, r);
    s->wall_verts.emplace_back(verts, verts + 3 * (size_t)std::max(n_verts, 0));
    s->ready = false;
    return LSDEM_OK;
  });
}

static int set_vec(lsdem_solver* s, std::vector<double>& v, int n, int index, const double* x, bool add) {
  if (!s || !x) return LSDEM_ERR_ARG;
  if (index < 0 || index >= n) return LSDEM_OK;  // reference: silently ignored
  if (const int rc = guard(s, [&] { pull_host(s); return LSDEM_OK; })) return rc;
  for (int a = 0; a < 3; ++a) v[3 * (size_t)index + a] = add ? v[3 * (size_t)index + a] + x[a] : x[a];
  s->ready = false;
  return LSDEM_OK;
}
int lsdem_move_particle(lsdem_solver* s, int index, const double* o) { return s ? set_vec(s, s->P.pos, s->P.n(), index, o, true) : LSDEM_ERR_ARG; }
int lsdem_move_wall(lsdem_solver* s, int index, const double* o) { return s ? set_vec(s, s->W.pos, s->W.n(), index, o, true) : LSDEM_ERR_ARG; }
int lsdem_set_wall_velocity(lsdem_solver* s, int index, const double* v) { return s ? set_vec(s, s->W.vel, s->W.n(), index, v, false) : LSDEM_ERR_ARG; }
int lsdem_set_wall_angular_velocity(lsdem_solver* s, int index, const double* w) { return s ? set_vec(s, s->W.angvel, s->W.n(), index, w, false) : LSDEM_ERR_ARG; }

// VBondedInteraction::add (VBondedInteraction.h:74-195) with the initial frame
// vectors of getInitialOrthogonalUnitVectorsN2/N3 (:10-22).
static int add_bond_impl(lsdem_solver* s, int i, int j, const double* pi, const double* qi, const double* pj,
                         const double* qj, const double* point, const double* normal, double Rb, double Lb, double Eb,
                         double nu, double ten, double coh, double fmu) {
  V3 gn = v3(normal);
  if (std::fabs(gn.x * gn.x + gn.y * gn.y + gn.z * gn.z) <= 1.0e-20) return fail(s, LSDEM_ERR_ARG, "Invalid bond normal");
  if (Rb <= 0.) return fail(s, LSDEM_ERR_ARG, "Invalid bond radius");
  if (Lb <= 0.) return fail(s, LSDEM_ERR_ARG, "Invalid bond length");
  if (Eb <= 0.) return fail(s, LSDEM_ERR_ARG, "Invalid Young's modulus");
  if (nu <= -1.0 || nu >= 0.5) return fail(s, LSDEM_ERR_ARG, "Invalid Poisson ratio");
  const double Gb = Eb / (2. * (1. + nu));
  const double Ab = M_PI * Rb * Rb;
  const double Ib = Ab * Rb * Rb / 4.;
  const double Jb = 2. * Ib;
  const double Kn = Eb * Ab / Lb, Kt = Gb * Jb / Lb, Ks = 12. * Eb * Ib / (Lb * Lb * Lb), Kb = Eb * Ib / Lb;
  const double B1 = Kn, B2 = Lb * Lb * Ks, B4 = Kt, B3 = Kb - B2 / 4. - B4 / 2.;
  const double inv_len = 1.0 / hlen(gn);
  const V3 n{gn.x * inv_len, gn.y * inv_len, gn.z * inv_len};
  const V3 c = v3(point);
  const V3 gpi{c.x + 0.5 * Lb * n.x, c.y + 0.5 * Lb * n.y, c.z + 0.5 * Lb * n.z};
  const V3 gpj{c.x - 0.5 * Lb * n.x, c.y - 0.5 * Lb * n.y, c.z - 0.5 * Lb * n.z};
  const V3 lpi = hrotate_inv(V3{gpi.x - pi[0], gpi.y - pi[1], gpi.z - pi[2]}, qi);
  const V3 lpj = hrotate_inv(V3{gpj.x - pj[0], gpj.y - pj[1], gpj.z - pj[2]}, qj);
  const V3 n1i{-n.x, -n.y, -n.z};
  const V3 ref = (std::fabs(n1i.x) < 0.9) ? V3{1., 0., 0.} : V3{0., 1., 0.};
  const V3 n2i = hnormalize(hcross(ref, n1i));
  const V3 n3i = hnormalize(hcross(n1i, n2i));
  const V3 n1j{-n1i.x, -n1i.y, -n1i.z};
  const V3 loc[8] = {hnormalize(hrotate_inv(n1i, qi)), hnormalize(hrotate_inv(n2i, qi)), hnormalize(hrotate_inv(n3i, qi)), lpi,
                     hnormalize(hrotate_inv(n1j, qj)), hnormalize(hrotate_inv(n2i, qj)), hnormalize(hrotate_inv(n3i, qj)), lpj};
  BondHost& b = s->bonds;
  b.ids.push_back(i); b.ids.push_back(j);
  b.bonded.push_back(1);
  b.B.insert(b.B.end(), {B1, B2, B3, B4});
  b.geo.insert(b.geo.end(), {Rb, Lb, ten, coh, fmu});
  for (const V3& v : loc) b.frames.insert(b.frames.end(), {v.x, v.y, v.z});
  b.state.insert(b.state.end(), {0., 0., 0., 0., 0., 0., c.x, c.y, c.z});
  s->ready = false;
  return LSDEM_OK;
}

int lsdem_add_bond(lsdem_solver* s, int master, int slave, const double* point3, const double* normal3, double radius,
                   double initial_length, double youngs, double poisson, double tensile, double cohesion, double mu) {
  if (!s || !point3 || !normal3) return LSDEM_ERR_ARG;
  if (master >= s->P.n() || slave >= s->P.n() || master < 0 || slave < 0) return LSDEM_OK;  // reference: ignored
  if (const int rc = guard(s, [&] { pull_host(s); return LSDEM_OK; })) return rc;
  return add_bond_impl(s, master, slave, &s->P.pos[3 * (size_t)master], &s->P.quat[4 * (size_t)master],
                       &s->P.pos[3 * (size_t)slave], &s->P.quat[4 * (size_t)slave], point3, normal3, radius,
                       initial_length, youngs, poisson, tensile, cohesion, mu);
}

// ---------------------------------------------------------------------------
// Learned per-shape SDF

MlpShapeData mlp_shape_data(lsdem_solver* s) {
  MlpShapeData D;
  D.norm = s->mlp_norm.p; D.gsize = s->s_gsize.p; D.origin = s->mlp_origin.p; D.h = s->mlp_h.p;
  D.sdf = s->s_sdf.p; D.sdf_off = s->s_sdf_off.p; D.node_off = s->s_node_off.p; D.node_cnt = s->s_node_cnt.p;
  D.node_pos = s->s_node_pos.p;
  return D;
}

int lsdem_train_learned_sdf(lsdem_solver* s, int iterations, int batch, int samples, double lr,
                            unsigned long long seed, double* loss_out, double* err_out) {
  if (s) ++s->graph_gen;
  if (!s || iterations < 1 || batch < 128 || batch % 128 != 0 || samples < batch || !(lr > 0.)) return LSDEM_ERR_ARG;
  if (!s->ready) return fail(s, LSDEM_ERR_STATE, "lsdem_train_learned_sdf before lsdem_initialize");
  return guard(s, [&] {
    cudaStream_t st = s->stream;
    const int ns = (int)s->shapes.size();
    if (ns == 0) return LSDEM_OK;
    // normalisation: centre and half the largest extent of each template's grid box
    s->h_mlp_norm.assign(ns, MlpNorm{});
    std::vector<double3> org(ns);
    std::vector<double> hh(ns);
    for (int k = 0; k < ns; ++k) {
      const ShapeHost& sh = s->shapes[k];
      double ext = 0.;
      for (int a = 0; a < 3; ++a) ext = std::max(ext, (sh.size[a] - 1) * sh.h);
      MlpNorm& nm = s->h_mlp_norm[k];
      nm.cx = (float)(sh.origin[0] + 0.5 * (sh.size[0] - 1) * sh.h);
      nm.cy = (float)(sh.origin[1] + 0.5 * (sh.size[1] - 1) * sh.h);
      nm.cz = (float)(sh.origin[2] + 0.5 * (sh.size[2] - 1) * sh.h);
      nm.R = (float)(0.5 * ext);
      nm.r_over_h = (float)(0.5 * ext / sh.h);
      org[k] = make_double3(sh.origin[0], sh.origin[1], sh.origin[2]);
      hh[k] = sh.h;
    }
    CK(s->mlp_norm.upload(s->h_mlp_norm.data(), ns, st));
    CK(s->mlp_origin.upload(org.data(), ns, st));
    CK(s->mlp_h.upload(hh.data(), ns, st));
    // initial weights: Glorot-uniform, zero biases
    std::vector<float> p0((size_t)ns * MLP_NP, 0.f);
    uint64_t r = seed * 0x9e3779b97f4a7c15ull + 1;
    auto uni = [&](double a) {
      r ^= r << 13; r ^= r >> 7; r ^= r << 17;
      return (float)(a * (2.0 * (double)(r >> 11) / 9007199254740992.0 - 1.0));
    };
    for (int k = 0; k < ns; ++k) {
      float* P = &p0[(size_t)k * MLP_NP];
      for (int i = 0; i < 192; ++i) P[MLP_W1 + i] = uni(std::sqrt(6.0 / (3 + 64)));
      for (int i = 0; i < 4096; ++i) P[MLP_W2 + i] = uni(std::sqrt(6.0 / (64 + 64)));
      for (int i = 0; i < 64; ++i) P[MLP_W3 + i] = uni(std::sqrt(6.0 / (64 + 1)));
    }
    CK(s->mlp_params.upload(p0.data(), p0.size(), st));
    CK(s->mlp_m1.alloc(p0.size())); CK(s->mlp_m1.zero(st));
    CK(s->mlp_m2.alloc(p0.size())); CK(s->mlp_m2.zero(st));
    const int nblk = batch / 128;
    CK(s->mlp_partial.alloc((size_t)ns * nblk * MLP_NP));
    CK(s->mlp_loss.alloc((size_t)ns * nblk));
    CK(s->mlp_samples.alloc((size_t)ns * samples));
    const MlpShapeData D = mlp_shape_data(s);
    mlp_samples(D, ns, samples, seed, s->mlp_opt, s->mlp_samples.p, st);
    CK(cudaGetLastError());
    // Adam with a cosine learning-rate schedule down to 1 % of lr
    for (int it = 0; it < iterations; ++it) {
      const double c = 0.5 * (1.0 + std::cos(M_PI * it / (double)iterations));
      const float lr_t = (float)(lr * (0.01 + 0.99 * c));
      CK(mlp_train_step(s->mlp_params.p, s->mlp_samples.p, ns, samples, batch, it, s->mlp_partial.p, s->mlp_loss.p,
                        s->mlp_m1.p, s->mlp_m2.p, lr_t, it + 1, st));
    }
    // loss of the last batch (mean squared error of phi / R, FP32 master weights)
    std::vector<float> lb = dl(s->mlp_loss, (size_t)ns * nblk, st);
    CK(s->mlp_inf.alloc(ns));
    mlp_pack(s->mlp_params.p, ns, s->mlp_inf.p, st);
    // trust band of each shape: 2 % of its size (twice its largest node distance)
    std::vector<float> delta(ns);
    for (int k = 0; k < ns; ++k) {
      const ShapeHost& sh = s->shapes[k];
      double rmax = 0.;
      for (size_t i = 0; i + 2 < sh.nodes.size(); i += 3)
        rmax = std::max(rmax, std::sqrt(sh.nodes[i] * sh.nodes[i] + sh.nodes[i + 1] * sh.nodes[i + 1] +
                                        sh.nodes[i + 2] * sh.nodes[i + 2]));
      delta[k] = (float)(0.02 * 2.0 * rmax);
    }
    DArr<float> ddelta;
    CK(ddelta.upload(delta.data(), ns, st));
    CK(s->mlp_err.alloc(2 * (size_t)ns)); CK(s->mlp_err.zero(st));
    DArr<int> dfail;
    CK(dfail.alloc(1)); CK(dfail.zero(st));
    mlp_validate(D, ns, s->mlp_inf.p, samples, seed ^ 0x5eedf00dull, s->mlp_opt, ddelta.p, s->mlp_err.p, dfail.p, st);
    CK(cudaGetLastError());
    std::vector<unsigned> eb = dl(s->mlp_err, 2 * (size_t)ns, st);
    std::vector<int> hf = dl(dfail, 1, st);
    CK(cudaStreamSynchronize(st));
    if (hf[0]) throw Fail{LSDEM_ERR_CUDA, "tensor-core wait gave up in the network validation"};
    s->h_mlp_band.assign(ns, 0.f);
    for (int k = 0; k < ns; ++k) {
      float e, ein;
      std::memcpy(&e, &eb[2 * k], 4);
      std::memcpy(&ein, &eb[2 * k + 1], 4);
      s->h_mlp_norm[k].err = e;
      s->h_mlp_norm[k].err_in = ein;
      s->h_mlp_norm[k].delta = delta[k];
      // network threshold in template spacings: the trust band plus 1.25 x the
      // one-sided error there, so that phi_net above it means phi_grid > delta
      const ShapeHost& sh = s->shapes[k];
      s->h_mlp_band[k] = (float)((1.25 * ein + delta[k]) / sh.h);
      double l = 0.;
      for (int b = 0; b < nblk; ++b) l += lb[(size_t)k * nblk + b];
      if (loss_out) loss_out[k] = l / batch;
      if (err_out) err_out[k] = e;
    }
    CK(s->mlp_norm.upload(s->h_mlp_norm.data(), ns, st));
    CK(s->mlp_band.upload(s->h_mlp_band.data(), ns, st));
    CK(cudaStreamSynchronize(st));
    s->mlp_trained = true;
    return LSDEM_OK;
  });
}

int lsdem_set_learned_training(lsdem_solver* s, double clip_lo, double clip_hi, double near_fraction) {
  if (!s) return LSDEM_ERR_ARG;
  // the trust band (at most 4 % of R) must lie inside the clip range
  if (!(clip_lo >= -1.0 && clip_lo <= -0.05 && clip_hi >= 0.1 && clip_hi <= 2.0 && near_fraction >= 0.0 &&
        near_fraction <= 1.0))
    return fail(s, LSDEM_ERR_ARG,
                "lsdem_set_learned_training: clip_lo in [-1, -0.05], clip_hi in [0.1, 2], near_fraction in [0, 1]");
  s->mlp_opt.clip_lo = (float)clip_lo;
  s->mlp_opt.clip_hi = (float)clip_hi;
  s->mlp_opt.near = (float)near_fraction;
  return LSDEM_OK;
}

int lsdem_set_learned_sdf(lsdem_solver* s, int on) {
  if (s) ++s->graph_gen;
  if (!s) return LSDEM_ERR_ARG;
  if (on && !s->mlp_trained) return fail(s, LSDEM_ERR_STATE, "lsdem_set_learned_sdf before lsdem_train_learned_sdf");
  s->mlp_on = on != 0;
  return LSDEM_OK;
}

int lsdem_get_learned_sdf(lsdem_solver* s, int shape, float* params, float* norm) {
  if (!s || shape < 0) return LSDEM_ERR_ARG;
  if (!s->mlp_trained || shape >= (int)s->h_mlp_norm.size()) return fail(s, LSDEM_ERR_STATE, "no trained network");
  return guard(s, [&] {
    if (params)
      CK(cudaMemcpy(params, s->mlp_params.p + (size_t)shape * MLP_NP, sizeof(float) * MLP_NP, cudaMemcpyDeviceToHost));
    if (norm) {
      const MlpNorm& n = s->h_mlp_norm[shape];
      const float v[8] = {n.cx, n.cy, n.cz, n.R, n.err, s->h_mlp_band[shape], n.err_in, n.delta};
      std::memcpy(norm, v, sizeof(v));
    }
    return LSDEM_OK;
  });
}

int lsdem_mlp_eval(lsdem_solver* s, int shape, int n, const double* pts, float* phi) {
  if (!s || shape < 0 || n < 0 || (n && (!pts || !phi))) return LSDEM_ERR_ARG;
  if (!s->mlp_trained || shape >= (int)s->h_mlp_norm.size()) return fail(s, LSDEM_ERR_STATE, "no trained network");
  return guard(s, [&] {
    DArr<double3> dp;
    DArr<float> dphi;
    CK(dp.upload((const double3*)pts, (size_t)n, s->stream));
    CK(dphi.alloc((size_t)std::max(n, 1)));
    DArr<int> dfail;
    CK(dfail.alloc(1)); CK(dfail.zero(s->stream));
    mlp_infer(s->mlp_inf.p + shape, s->h_mlp_norm[shape], dp.p, n, dphi.p, dfail.p, s->stream);
    CK(cudaGetLastError());
    if (n) CK(cudaMemcpyAsync(phi, dphi.p, sizeof(float) * n, cudaMemcpyDeviceToHost, s->stream));
    std::vector<int> hf = dl(dfail, 1, s->stream);
    CK(cudaStreamSynchronize(s->stream));
    if (hf[0]) throw Fail{LSDEM_ERR_CUDA, "tensor-core wait gave up in the network evaluation"};
    return LSDEM_OK;
  });
}

int lsdem_mlp_gradient(int device, int n, const float* params, const float* pts, float* loss, float* grad,
                       float* y) {
  if (n <= 0 || n % 128 != 0 || !params || !pts) return LSDEM_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return LSDEM_ERR_NODEVICE;
  try {
    DArr<float> dpar, dpart, dloss, dy;
    DArr<float4> dpts;
    CK(dpar.upload(params, MLP_NP, nullptr));
    CK(dpts.upload((const float4*)pts, (size_t)n, nullptr));
    const int nblk = n / 128;
    CK(dpart.alloc((size_t)nblk * MLP_NP));
    CK(dloss.alloc((size_t)nblk));
    CK(mlp_grad_once(dpar.p, dpts.p, n, dpart.p, dloss.p, nullptr));
    std::vector<float> part = dl(dpart, (size_t)nblk * MLP_NP, nullptr);
    std::vector<float> lb = dl(dloss, (size_t)nblk, nullptr);
    if (y) {
      CK(dy.alloc((size_t)n));
      mlp_forward(dpar.p, dpts.p, n, dy.p, nullptr);
      CK(cudaMemcpy(y, dy.p, sizeof(float) * n, cudaMemcpyDeviceToHost));
    }
    CK(cudaDeviceSynchronize());
    if (grad)
      for (int k = 0; k < MLP_NP; ++k) {
        double g = 0.;
        for (int b = 0; b < nblk; ++b) g += part[(size_t)b * MLP_NP + k];
        grad[k] = k <= MLP_B3 ? (float)g : 0.f;
      }
    if (loss) {
      double l = 0.;
      for (float v : lb) l += v;
      *loss = (float)(l / n);
    }
    return LSDEM_OK;
  } catch (const Fail& e) {
    return e.code;
  }
}

int lsdem_set_precision(lsdem_solver* s, int mode) {
  if (!s || mode < PREC_FP64 || mode > PREC_FP32_BF16) return LSDEM_ERR_ARG;
  s->precision = mode;
  s->ready = false;
  return LSDEM_OK;
}

int lsdem_set_periodic(lsdem_solver* s, int axes) {
  if (!s) return LSDEM_ERR_ARG;
  if ((axes & 8) && (axes & 7))
    return fail(s, LSDEM_ERR_ARG, "sector periodicity cannot be combined with x, y or z periodicity");
  s->periodic = axes & 15;
  s->ready = false;
  return LSDEM_OK;
}

int lsdem_set_record_contacts(lsdem_solver* s, int on) {
  if (!s) return LSDEM_ERR_ARG;
  s->record = on != 0;
  return LSDEM_OK;
}

int lsdem_set_capacity(lsdem_solver* s, int pp, int w, int g, long long c, int batch) {
  if (s) ++s->graph_gen;
  if (!s) return LSDEM_ERR_ARG;
  if (pp > 0) s->cap_pp = pp;
  if (w > 0) s->cap_w = w;
  if (g > 0) s->cap_g = g;
  if (c > 0) s->cap_c = c;
  if (batch > 0) s->batch = batch;
  s->ready = false;
  return LSDEM_OK;
}

int lsdem_initialize(lsdem_solver* s, const double* min3, const double* max3, const double* gravity3) {
  if (!s || !min3 || !max3) return fail(s, LSDEM_ERR_ARG, "null argument");
  for (int a = 0; a < 3; ++a)
    if (!(max3[a] - min3[a] > 0.0)) return fail(s, LSDEM_ERR_ARG, "Invalid simulation domain size");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= s->device)
    return fail(s, LSDEM_ERR_NODEVICE, "no usable CUDA device");
  for (int a = 0; a < 3; ++a) {
    s->dmin[a] = min3[a];
    s->dmax[a] = max3[a];
    s->grav[a] = gravity3 ? gravity3[a] : 0.;
  }
  ++s->vtu_layout;
  ++s->graph_gen;
  s->time = 0.0;  // each phase starts at time 0, as the reference's compute loop (LSSolver.h:994-996)
  return guard(s, [&] {
    initialize(s);
    return LSDEM_OK;
  });
}

int lsdem_step(lsdem_solver* s, double dt, long long nsteps, lsdem_hook hook, void* user) {
  if (!s) return LSDEM_ERR_ARG;
  if (nsteps <= 0) return LSDEM_OK;
  return guard(s, [&] { return run_steps(s, dt, nsteps, hook, user); });
}

long long lsdem_num(const lsdem_solver* s, int what) {
  if (!s) return -1;
  switch (what) {
    case 0: return s->P.n();
    case 1: return s->W.n();
    case 2: return (long long)s->bonds.bonded.size();
    case 3: {
      long long nb = 0;
      for (int i = 0; i < s->P.n(); ++i) nb += (long long)(s->shapes[s->P.shape[i]].nodes.size() / 3);
      return nb;
    }
    case 4: return (long long)s->shapes.size();
    case 5: return s->ready ? s->pg.ncells : 0;
    case 6: return s->steps;
    case 7: return s->reruns;
    case 8: return s->launches;
    case 9: return s->builds;
    default: return -1;
  }
}

double lsdem_time(const lsdem_solver* s) { return s ? s->time : 0.0; }

int lsdem_get_state(lsdem_solver* s, double* pos, double* vel, double* angvel, double* quat, double* force,
                    double* torque) {
  if (!s) return LSDEM_ERR_ARG;
  if (!s->ready) {
    if (const int rc = guard(s, [&] { pull_host(s); return LSDEM_OK; })) return rc;
    const size_t n = (size_t)s->P.n();
    if (pos) std::memcpy(pos, s->P.pos.data(), 24 * n);
    if (vel) std::memcpy(vel, s->P.vel.data(), 24 * n);
    if (angvel) std::memcpy(angvel, s->P.angvel.data(), 24 * n);
    if (quat) std::memcpy(quat, s->P.quat.data(), 32 * n);
    if (force) std::memcpy(force, s->P.force.data(), 24 * n);
    if (torque) std::memcpy(torque, s->P.torque.data(), 24 * n);
    return LSDEM_OK;
  }
  return guard(s, [&] {
    const size_t n = (size_t)s->P.n();
    cudaStream_t st = s->stream;
    if (pos && n) CK(cudaMemcpyAsync(pos, s->dP.pos.p, 24 * n, cudaMemcpyDeviceToHost, st));
    if (vel && n) CK(cudaMemcpyAsync(vel, s->dP.vel.p, 24 * n, cudaMemcpyDeviceToHost, st));
    if (angvel && n) CK(cudaMemcpyAsync(angvel, s->dP.angvel.p, 24 * n, cudaMemcpyDeviceToHost, st));
    if (quat && n) CK(cudaMemcpyAsync(quat, s->dP.quat.p, 32 * n, cudaMemcpyDeviceToHost, st));
    if (force && n) CK(cudaMemcpyAsync(force, s->dP.force.p, 24 * n, cudaMemcpyDeviceToHost, st));
    if (torque && n) CK(cudaMemcpyAsync(torque, s->dP.torque.p, 24 * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return LSDEM_OK;
  });
}

int lsdem_get_wall_state(lsdem_solver* s, double* pos, double* vel, double* angvel, double* quat) {
  if (!s) return LSDEM_ERR_ARG;
  const size_t n = (size_t)s->W.n();
  if (!s->ready) {
    if (const int rc = guard(s, [&] { pull_host(s); return LSDEM_OK; })) return rc;
    if (pos) std::memcpy(pos, s->W.pos.data(), 24 * n);
    if (vel) std::memcpy(vel, s->W.vel.data(), 24 * n);
    if (angvel) std::memcpy(angvel, s->W.angvel.data(), 24 * n);
    if (quat) std::memcpy(quat, s->W.quat.data(), 32 * n);
    return LSDEM_OK;
  }
  return guard(s, [&] {
    cudaStream_t st = s->stream;
    if (pos && n) CK(cudaMemcpyAsync(pos, s->dW.pos.p, 24 * n, cudaMemcpyDeviceToHost, st));
    if (vel && n) CK(cudaMemcpyAsync(vel, s->dW.vel.p, 24 * n, cudaMemcpyDeviceToHost, st));
    if (angvel && n) CK(cudaMemcpyAsync(angvel, s->dW.angvel.p, 24 * n, cudaMemcpyDeviceToHost, st));
    if (quat && n) CK(cudaMemcpyAsync(quat, s->dW.quat.p, 32 * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return LSDEM_OK;
  });
}

int lsdem_set_state(lsdem_solver* s, const double* pos, const double* vel, const double* angvel, const double* quat) {
  if (!s) return LSDEM_ERR_ARG;
  const size_t n = (size_t)s->P.n();
  if (!s->ready) {
    if (const int rc = guard(s, [&] { pull_host(s); return LSDEM_OK; })) return rc;
    if (pos) std::memcpy(s->P.pos.data(), pos, 24 * n);
    if (vel) std::memcpy(s->P.vel.data(), vel, 24 * n);
    if (angvel) std::memcpy(s->P.angvel.data(), angvel, 24 * n);
    if (quat) std::memcpy(s->P.quat.data(), quat, 32 * n);
    return LSDEM_OK;
  }
  return guard(s, [&] {
    cudaStream_t st = s->stream;
    if (pos && n) CK(cudaMemcpyAsync(s->dP.pos.p, pos, 24 * n, cudaMemcpyHostToDevice, st));
    if (vel && n) CK(cudaMemcpyAsync(s->dP.vel.p, vel, 24 * n, cudaMemcpyHostToDevice, st));
    if (angvel && n) CK(cudaMemcpyAsync(s->dP.angvel.p, angvel, 24 * n, cudaMemcpyHostToDevice, st));
    if (quat && n) CK(cudaMemcpyAsync(s->dP.quat.p, quat, 32 * n, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    s->host_stale = true;
    return LSDEM_OK;
  });
}

int lsdem_get_particle_params(const lsdem_solver* s, double* inv_mass, double* inv_inertia6, double* radius,
                              double* kn, double* ks, double* mu, double* e, int* shape, double* scale,
                              double* origin3, double* invh, long long* node_base) {
  if (!s) return LSDEM_ERR_ARG;
  const BodyHost& P = s->P;
  const size_t n = (size_t)P.n();
  if (inv_mass) std::memcpy(inv_mass, P.invm.data(), 8 * n);
  if (inv_inertia6) std::memcpy(inv_inertia6, P.invI.data(), 48 * n);
  if (radius) std::memcpy(radius, P.radius.data(), 8 * n);
  if (kn) std::memcpy(kn, P.kn.data(), 8 * n);
  if (ks) std::memcpy(ks, P.ks.data(), 8 * n);
  if (mu) std::memcpy(mu, P.mu.data(), 8 * n);
  if (e) std::memcpy(e, P.res.data(), 8 * n);
  if (shape) std::memcpy(shape, P.shape.data(), 4 * n);
  if (scale) std::memcpy(scale, P.scale.data(), 8 * n);
  if (origin3) std::memcpy(origin3, P.origin.data(), 24 * n);
  if (invh) std::memcpy(invh, P.invh.data(), 8 * n);
  if (node_base) {
    long long nb = 0;
    for (size_t i = 0; i < n; ++i) {
      node_base[i] = nb;
      nb += (long long)(s->shapes[P.shape[i]].nodes.size() / 3);
    }
  }
  return LSDEM_OK;
}

int lsdem_get_wall_params(const lsdem_solver* s, double* radius, double* mu, double* e, int* shape, double* origin3,
                          double* invh) {
  if (!s) return LSDEM_ERR_ARG;
  const BodyHost& W = s->W;
  const size_t n = (size_t)W.n();
  if (radius) std::memcpy(radius, W.radius.data(), 8 * n);
  if (mu) std::memcpy(mu, W.mu.data(), 8 * n);
  if (e) std::memcpy(e, W.res.data(), 8 * n);
  if (shape) std::memcpy(shape, W.shape.data(), 4 * n);
  if (origin3) std::memcpy(origin3, W.origin.data(), 24 * n);
  if (invh) std::memcpy(invh, W.invh.data(), 8 * n);
  return LSDEM_OK;
}

int lsdem_get_shape(const lsdem_solver* s, int shape, double* nodes, double* sdf, int* size3, double* origin3,
                    double* spacing, int* n_nodes) {
  if (!s || shape < 0 || shape >= (int)s->shapes.size()) return LSDEM_ERR_ARG;
  const ShapeHost& sh = s->shapes[shape];
  if (nodes) std::memcpy(nodes, sh.nodes.data(), 8 * sh.nodes.size());
  if (sdf) std::memcpy(sdf, sh.sdf.data(), 8 * sh.sdf.size());
  if (size3) for (int a = 0; a < 3; ++a) size3[a] = sh.size[a];
  if (origin3) for (int a = 0; a < 3; ++a) origin3[a] = sh.origin[a];
  if (spacing) *spacing = sh.h;
  if (n_nodes) *n_nodes = (int)(sh.nodes.size() / 3);
  return LSDEM_OK;
}

static void grid_out(const GridP& g, double* mn, double* mx, double* inv, int* size) {
  if (mn) { mn[0] = g.mn.x; mn[1] = g.mn.y; mn[2] = g.mn.z; }
  if (mx) { mx[0] = g.mx.x; mx[1] = g.mx.y; mx[2] = g.mx.z; }
  if (inv) { inv[0] = g.inv.x; inv[1] = g.inv.y; inv[2] = g.inv.z; }
  if (size) { size[0] = g.size.x; size[1] = g.size.y; size[2] = g.size.z; }
}
int lsdem_get_grid(const lsdem_solver* s, double* mn, double* mx, double* inv, int* size) {
  if (!s || !s->ready) return LSDEM_ERR_STATE;
  grid_out(s->pg, mn, mx, inv, size);
  return LSDEM_OK;
}
int lsdem_get_wall_grid(const lsdem_solver* s, double* mn, double* mx, double* inv, int* size) {
  if (!s || !s->ready) return LSDEM_ERR_STATE;
  grid_out(s->wg, mn, mx, inv, size);
  return LSDEM_OK;
}

int lsdem_get_hash(lsdem_solver* s, int* key, int* sorted_idx, int* sorted_key, int* cell_start, int* cell_end) {
  if (!s || !s->ready) return LSDEM_ERR_STATE;
  return guard(s, [&] {
    const size_t n = (size_t)s->P.n(), nc = (size_t)s->pg.ncells;
    cudaStream_t st = s->stream;
    if (s->reuse_on && n) {
      // with neighbour lists the last sort may predate the current keys: sort them now
      // (the lists refer to the old order, so the next step rebuilds them)
      BucketScratch w{s->bk_counts.p, s->bk_fill.p, s->bk_offs.p, s->bk_scan.p, s->bk_big.p, s->bk_bigc.p,
                      s->bk_tmp.p};
      bucket_sort(s->dP.key.p, (int)n, s->pg.ncells, w, s->cell_idx.p, s->sorted_key.p, s->cell_start.p,
                  s->cell_end.p, st);
      CK(cudaGetLastError());
      s->force_reuse = true;
    }
    if (key && n) CK(cudaMemcpyAsync(key, s->dP.key.p, 4 * n, cudaMemcpyDeviceToHost, st));
    if (sorted_idx && n) CK(cudaMemcpyAsync(sorted_idx, s->cell_idx.p, 4 * n, cudaMemcpyDeviceToHost, st));
    if (sorted_key && n) CK(cudaMemcpyAsync(sorted_key, s->sorted_key.p, 4 * n, cudaMemcpyDeviceToHost, st));
    if (cell_start) CK(cudaMemcpyAsync(cell_start, s->cell_start.p, 4 * nc, cudaMemcpyDeviceToHost, st));
    if (cell_end) CK(cudaMemcpyAsync(cell_end, s->cell_end.p, 4 * nc, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return LSDEM_OK;
  });
}

int lsdem_count_contacts(lsdem_solver* s, int kind, long long* n) {
  if (!s || !n || kind < 0 || kind > 2) return LSDEM_ERR_ARG;
  if (!s->ready) { *n = 0; return LSDEM_OK; }
  return guard(s, [&] {
    long long t = 0;
    walk_contacts(s, kind, [&](int, int, int, int c) { t += c; });
    *n = t;
    return LSDEM_OK;
  });
}

int lsdem_get_contacts(lsdem_solver* s, int kind, long long cap, long long* node, int* partner, int* image,
                       double* spring, double* point, double* normal, double* overlap, double* en_n, double* en_s) {
  if (!s || kind < 0 || kind > 2) return LSDEM_ERR_ARG;
  if (!s->ready) return LSDEM_OK;
  return guard(s, [&] {
    cudaStream_t st = s->stream;
    ContactsDev& c = s->con[s->hp];
    const size_t nc = (size_t)s->hist_count;
    auto cn = dl(c.node, nc, st);
    auto cs = dl(c.spring, nc, st);
    const bool g = c.geom && (point || normal || overlap || en_n || en_s);
    std::vector<double3> cp, cnm;
    std::vector<double> co, ce, cf;
    if (g) { cp = dl(c.point, nc, st); cnm = dl(c.normal, nc, st); co = dl(c.overlap, nc, st); ce = dl(c.en_n, nc, st); cf = dl(c.en_s, nc, st); }
    CK(cudaStreamSynchronize(st));
    std::vector<long long> nbase(s->P.n());
    long long nb = 0;
    for (int i = 0; i < s->P.n(); ++i) { nbase[i] = nb; nb += (long long)(s->shapes[s->P.shape[i]].nodes.size() / 3); }
    long long out = 0;
    walk_contacts(s, kind, [&](int A, int pid, int start, int cntk) {
      const ShapeHost& sh = s->shapes[s->P.shape[A]];
      for (int t = 0; t < cntk; ++t) {
        if (out >= cap) return;
        const size_t k = (size_t)start + t;
        if (node) node[out] = nbase[A] + sh.perm[cn[k]];
        if (partner) partner[out] = kind == 2 ? (pid >> 3) : pid;
        if (image) image[out] = kind == 2 ? s->set_mask[pid & 7] : 0;
        if (spring) { spring[3 * out] = cs[k].x; spring[3 * out + 1] = cs[k].y; spring[3 * out + 2] = cs[k].z; }
        if (g) {
          if (point) { point[3 * out] = cp[k].x; point[3 * out + 1] = cp[k].y; point[3 * out + 2] = cp[k].z; }
          if (normal) { normal[3 * out] = cnm[k].x; normal[3 * out + 1] = cnm[k].y; normal[3 * out + 2] = cnm[k].z; }
          if (overlap) overlap[out] = co[k];
          if (en_n) en_n[out] = ce[k];
          if (en_s) en_s[out] = cf[k];
        }
        ++out;
      }
    });
    return LSDEM_OK;
  });
}

int lsdem_create_bonds_from_contacts(lsdem_solver* s, double radius, double L0, double E, double nu, double ten,
                                     double coh, double mu) {
  if (!s) return LSDEM_ERR_ARG;
  if (!s->ready) return LSDEM_OK;  // no contact list yet
  return guard(s, [&] {
    long long n = 0;
    lsdem_count_contacts(s, LSDEM_CONTACT_PARTICLE, &n);
    if (n == 0) return LSDEM_OK;
    if (!s->con[s->hp].geom) throw Fail{LSDEM_ERR_STATE, "contact geometry not recorded (lsdem_set_record_contacts)"};
    // the bond constants are the same for every bond: checked once, as add_bond_impl does
    if (radius <= 0.) throw Fail{LSDEM_ERR_ARG, "Invalid bond radius"};
    if (L0 <= 0.) throw Fail{LSDEM_ERR_ARG, "Invalid bond length"};
    if (E <= 0.) throw Fail{LSDEM_ERR_ARG, "Invalid Young's modulus"};
    if (nu <= -1.0 || nu >= 0.5) throw Fail{LSDEM_ERR_ARG, "Invalid Poisson ratio"};
    pull_host(s);
    cudaStream_t st = s->stream;
    const int np = s->P.n();
    SlotsDev& sl = s->slots[s->hp][LSDEM_CONTACT_PARTICLE];
    const SlotView v{sl.cap, sl.cnt.p, sl.id.p, sl.seg_start.p, sl.seg_cnt.p};
    // contacts per owner, their offsets, then one bond per contact in list order, on the device
    DArr<int> cnt, offs, tmp;
    CK(cnt.alloc(np)); CK(offs.alloc(np)); CK(tmp.alloc(scan_temp_elems(np)));
    bonds_from_contacts_count(v, np, cnt.p, st);
    scan_i32(cnt.p, offs.p, np, tmp.p, false, st);
    int last[2] = {0, 0};
    CK(cudaMemcpyAsync(&last[0], offs.p + np - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&last[1], cnt.p + np - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const size_t nb = (size_t)last[0] + last[1];
    if (nb == 0) return LSDEM_OK;
    DArr<int> ids, bad;
    DArr<double3> frames, bpt;
    CK(ids.alloc(2 * nb)); CK(bad.alloc(1)); CK(bad.zero(st));
    CK(frames.alloc(8 * nb)); CK(bpt.alloc(nb));
    ContactsDev& c = s->con[s->hp];
    bonds_from_contacts_make(v, np, offs.p, c.point.p, c.normal.p, s->dP.pos.p, s->dP.quat.p, L0, ids.p, frames.p,
                             bpt.p, bad.p, st);
    CK(cudaGetLastError());
    std::vector<int> hid = dl(ids, 2 * nb, st), hbad = dl(bad, 1, st);
    std::vector<double3> hfr = dl(frames, 8 * nb, st), hpt = dl(bpt, nb, st);
    CK(cudaStreamSynchronize(st));
    if (hbad[0]) throw Fail{LSDEM_ERR_ARG, "Invalid bond normal"};
    // constants of add_bond_impl (VBondedInteraction.h:74-195)
    const double Gb = E / (2. * (1. + nu));
    const double Ab = M_PI * radius * radius;
    const double Ib = Ab * radius * radius / 4.;
    const double Jb = 2. * Ib;
    const double Kn = E * Ab / L0, Kt = Gb * Jb / L0, Ks = 12. * E * Ib / (L0 * L0 * L0), Kb = E * Ib / L0;
    const double B1 = Kn, B2 = L0 * L0 * Ks, B4 = Kt, B3 = Kb - B2 / 4. - B4 / 2.;
    BondHost& b = s->bonds;
    for (size_t k = 0; k < nb; ++k) {
      b.ids.push_back(hid[2 * k]); b.ids.push_back(hid[2 * k + 1]);
      b.bonded.push_back(1);
      b.B.insert(b.B.end(), {B1, B2, B3, B4});
      b.geo.insert(b.geo.end(), {radius, L0, ten, coh, mu});
      for (int f = 0; f < 8; ++f) b.frames.insert(b.frames.end(), {hfr[8 * k + f].x, hfr[8 * k + f].y, hfr[8 * k + f].z});
      b.state.insert(b.state.end(), {0., 0., 0., 0., 0., 0., hpt[k].x, hpt[k].y, hpt[k].z});
    }
    s->ready = false;
    return LSDEM_OK;
  });
}

int lsdem_get_bonds(lsdem_solver* s, int* ids2, int* bonded, double* state9) {
  if (!s) return LSDEM_ERR_ARG;
  const size_t nb = s->bonds.bonded.size();
  if (ids2) std::memcpy(ids2, s->bonds.ids.data(), 8 * nb);
  if (!s->ready || nb == 0) {
    if (const int rc = guard(s, [&] { pull_host(s); return LSDEM_OK; })) return rc;
    if (bonded) std::memcpy(bonded, s->bonds.bonded.data(), 4 * nb);
    if (state9) std::memcpy(state9, s->bonds.state.data(), 72 * nb);
    return LSDEM_OK;
  }
  return guard(s, [&] {
    cudaStream_t st = s->stream;
    if (bonded) CK(cudaMemcpyAsync(bonded, s->b_bonded.p, 4 * nb, cudaMemcpyDeviceToHost, st));
    if (state9) CK(cudaMemcpyAsync(state9, s->b_state.p, 72 * nb, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return LSDEM_OK;
  });
}

int lsdem_get_bond_params(lsdem_solver* s, double* B4, double* geo5, double* frames24) {
  if (!s) return LSDEM_ERR_ARG;
  const size_t nb = s->bonds.bonded.size();
  if (B4 && nb) std::memcpy(B4, s->bonds.B.data(), sizeof(double) * 4 * nb);
  if (geo5 && nb) std::memcpy(geo5, s->bonds.geo.data(), sizeof(double) * 5 * nb);
  if (frames24 && nb) std::memcpy(frames24, s->bonds.frames.data(), sizeof(double) * 24 * nb);
  return LSDEM_OK;
}

int lsdem_device_pointers(lsdem_solver* s, void** force, void** torque, void** vel, void** angvel, void** pos,
                          void** quat) {
  if (!s || !s->ready) return LSDEM_ERR_STATE;
  if (force) *force = s->dP.force.p;
  if (torque) *torque = s->dP.torque.p;
  if (vel) *vel = s->dP.vel.p;
  if (angvel) *angvel = s->dP.angvel.p;
  if (pos) *pos = s->dP.pos.p;
  if (quat) *quat = s->dP.quat.p;
  return LSDEM_OK;
}

void* lsdem_stream(const lsdem_solver* s) { return s ? (void*)s->stream : nullptr; }


int lsdem_set_graphs(lsdem_solver* s, int on) {
  if (!s) return LSDEM_ERR_ARG;
  s->graphs = on != 0;
  return LSDEM_OK;
}

int lsdem_set_neighbour_lists(lsdem_solver* s, int on) {
  if (!s) return LSDEM_ERR_ARG;
  if (s->reuse_on != (on != 0)) {
    s->reuse_on = on != 0;
    ++s->graph_gen;
    s->force_reuse = true;
  }
  return LSDEM_OK;
}

int lsdem_set_profiling(lsdem_solver* s, int on) {
  if (!s) return LSDEM_ERR_ARG;
  s->profiling = on != 0;
  for (int k = 0; k < LSDEM_NUM_PHASES; ++k)
    if (k != 9) { s->prof_ms[k] = 0.; s->prof_calls[k] = 0; }
  return LSDEM_OK;
}

int lsdem_set_step_timing(lsdem_solver* s, int on, long long l2_flush_bytes) {
  if (!s || l2_flush_bytes < 0) return LSDEM_ERR_ARG;
  return guard(s, [&] {
    CK(cudaStreamSynchronize(s->stream));
    s->step_timing = on != 0;
    s->prof_ms[9] = 0.;
    s->prof_calls[9] = 0;
    if (on && l2_flush_bytes > 0) {
      if (s->flush_buf.n != (size_t)l2_flush_bytes) CK(s->flush_buf.alloc((size_t)l2_flush_bytes));
    } else {
      s->flush_buf.release();
    }
    return LSDEM_OK;
  });
}

int lsdem_get_profile(const lsdem_solver* s, double* ms, long long* calls) {
  if (!s) return LSDEM_ERR_ARG;
  for (int k = 0; k < LSDEM_NUM_PHASES; ++k) {
    if (ms) ms[k] = s->prof_ms[k];
    if (calls) calls[k] = s->prof_calls[k];
  }
  return LSDEM_OK;
}

int lsdem_step_stats(lsdem_solver* s, long long* out4) {
  if (!s || !out4) return LSDEM_ERR_ARG;
  if (!s->ready) { for (int k = 0; k < 4; ++k) out4[k] = 0; return LSDEM_OK; }
  return guard(s, [&] {
    long long pairs[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k) {
      SlotsDev& sl = s->slots[s->hp][k];
      if (!sl.cnt.p || sl.cap == 0) continue;
      auto c = dl(sl.cnt, (size_t)s->P.n(), s->stream);
      CK(cudaStreamSynchronize(s->stream));
      for (int v : c) pairs[k] += std::min(v, sl.cap);
    }
    out4[0] = pairs[0]; out4[1] = pairs[1]; out4[2] = pairs[2]; out4[3] = s->hist_count;
    return LSDEM_OK;
  });
}

int lsdem_set_screen_stats(lsdem_solver* s, int on) {
  if (s) ++s->graph_gen;
  if (!s) return LSDEM_ERR_ARG;
  return guard(s, [&] {
    if (on) {
      CK(s->scr_stats.alloc(11));
      CK(s->scr_stats.zero(s->stream));
    } else {
      CK(cudaStreamSynchronize(s->stream));
      s->scr_stats.release();
    }
    return LSDEM_OK;
  });
}

int lsdem_get_screen_stats(lsdem_solver* s, long long* out8) {
  if (!s || !out8) return LSDEM_ERR_ARG;
  return guard(s, [&] {
    for (int k = 0; k < 8; ++k) out8[k] = 0;
    if (!s->scr_stats.p) return LSDEM_OK;
    auto c = dl(s->scr_stats, 8, s->stream);
    CK(cudaStreamSynchronize(s->stream));
    for (int k = 0; k < 8; ++k) out8[k] = (long long)c[k];
    return LSDEM_OK;
  });
}

int lsdem_get_screen_queue(lsdem_solver* s, long long* out3) {
  if (!s || !out3) return LSDEM_ERR_ARG;
  return guard(s, [&] {
    for (int k = 0; k < 3; ++k) out3[k] = 0;
    if (!s->scr_stats.p) return LSDEM_OK;
    auto c = dl(s->scr_stats, 11, s->stream);
    CK(cudaStreamSynchronize(s->stream));
    for (int k = 0; k < 3; ++k) out3[k] = (long long)c[8 + k];
    return LSDEM_OK;
  });
}

// Random sequential addition of spheres (largest first, in the given order)
// in the box [lo, hi), optionally periodic, using a uniform cell list.
// Returns LSDEM_ERR_ARG when a sphere cannot be placed in max_tries.
// ---------------------------------------------------------------------------
// Frame output

int lsdem_set_triangles(lsdem_solver* s, int kind, int index, const int* tris, int n_tris) {
  if (!s || (kind != 0 && kind != 1) || n_tris < 0 || (n_tris > 0 && !tris)) return LSDEM_ERR_ARG;
  const int nb = kind == 0 ? s->P.n() : s->W.n();
  if (index < 0 || index >= nb) return fail(s, LSDEM_ERR_ARG, "body index out of range");
  const int nn = kind == 0 ? (int)(s->shapes[s->P.shape[index]].nodes.size() / 3)
                           : (int)(s->wall_verts[index].size() / 3);
  for (int k = 0; k < 3 * n_tris; ++k)
    if (tris[k] < 0 || tris[k] >= nn) return fail(s, LSDEM_ERR_ARG, "triangle vertex index out of range");
  std::vector<int>& ids = kind == 0 ? s->P_tris : s->W_tris;
  if ((int)ids.size() < nb) ids.resize(nb, -1);
  if (n_tris == 0) {
    ids[index] = -1;
  } else {
    std::vector<int> t(tris, tris + 3 * (size_t)n_tris);
    auto it = s->tri_set_of.find(t);
    if (it == s->tri_set_of.end()) {
      it = s->tri_set_of.emplace(t, (int)s->tri_sets.size()).first;
      s->tri_sets.push_back(std::move(t));
    }
    ids[index] = it->second;
  }
  ++s->vtu_layout;
  return LSDEM_OK;
}

int lsdem_write_vtu(lsdem_solver* s, const char* dir, unsigned long long frame, unsigned long long step, double time) {
  if (!s || !dir) return LSDEM_ERR_ARG;
  if (!s->ready) return fail(s, LSDEM_ERR_STATE, "write_vtu before initialize");
  return guard(s, [&] {
    VtuInput in;
    in.dir = dir;
    in.frame = frame; in.step = step; in.time = time;
    in.solver_stream = s->stream;
    in.layout = s->vtu_layout;
    const int n = s->P.n();
    in.n = n;
    in.pos = s->dP.pos.p; in.vel = s->dP.vel.p; in.angvel = s->dP.angvel.p;
    in.quat = reinterpret_cast<const Quat*>(s->dP.quat.p);
    in.radius = s->dP.radius.p;
    std::vector<long long> nbase(n + 1, 0);
    for (int i = 0; i < n; ++i) nbase[i + 1] = nbase[i] + (long long)(s->shapes[s->P.shape[i]].nodes.size() / 3);
    in.node_base = nbase.data();
    in.shape = s->P.shape.data();
    in.scale = s->P.scale.data();
    for (const ShapeHost& sh : s->shapes) in.tnodes.push_back(&sh.nodes);
    std::vector<int> ptris(s->P_tris);
    ptris.resize(n, -1);
    in.tri_set = ptris.data();
    for (const auto& t : s->tri_sets) in.tri_sets.push_back(&t);
    // walls: current state (few), vertices and triangles
    const int nw = s->W.n();
    in.nw = nw;
    std::vector<double> wp(3 * nw), wv(3 * nw), ww(3 * nw), wq(4 * nw);
    if (nw) {
      int rc = lsdem_get_wall_state(s, wp.data(), wv.data(), ww.data(), wq.data());
      if (rc) throw Fail{rc, "wall state"};
    }
    in.wpos = wp.data(); in.wvel = wv.data(); in.wangvel = ww.data(); in.wquat = wq.data();
    for (int w = 0; w < nw; ++w) {
      in.wall_verts.push_back(&s->wall_verts[w]);
      const int k = w < (int)s->W_tris.size() ? s->W_tris[w] : -1;
      in.wall_tris.push_back(k < 0 ? nullptr : &s->tri_sets[k]);
    }
    // contacts of the particle and wall lists, as recorded at the last step
    for (int kind : {LSDEM_CONTACT_PARTICLE, LSDEM_CONTACT_WALL}) {
      long long m = 0;
      lsdem_count_contacts(s, kind, &m);
      if (m > 0 && !s->con[s->hp].geom) throw Fail{LSDEM_ERR_STATE, "contact geometry not recorded (lsdem_set_record_contacts)"};
      VtuContacts& c = kind == LSDEM_CONTACT_PARTICLE ? in.pp : in.pw;
      c.point.resize(3 * m); c.normal.resize(3 * m); c.spring.resize(3 * m); c.en_n.resize(m); c.en_s.resize(m);
      std::vector<double> ov(m);
      if (m > 0) {
        int rc = lsdem_get_contacts(s, kind, m, nullptr, nullptr, nullptr, c.spring.data(), c.point.data(),
                                    c.normal.data(), ov.data(), c.en_n.data(), c.en_s.data());
        if (rc) throw Fail{rc, "contacts"};
      }
    }
    const size_t nbd = s->bonds.bonded.size();
    in.bond_ids.resize(2 * nbd); in.bond_bonded.resize(nbd); in.bond_state.resize(9 * nbd);
    if (nbd) lsdem_get_bonds(s, in.bond_ids.data(), in.bond_bonded.data(), in.bond_state.data());
    try {
      vtu_write(s->vtu, in);
    } catch (const VtuError& e) {
      throw Fail{LSDEM_ERR_CUDA, "write_vtu: " + e.msg};
    }
    return LSDEM_OK;
  });
}

int lsdem_pack_rsa(int n, const double* radius, const double* lo, const double* hi, int periodic, unsigned long long seed,
                   int max_tries, const int* keep, double* pos_out) {
  if (n < 0 || !radius || !lo || !hi || !pos_out) return LSDEM_ERR_ARG;
  if (n == 0) return LSDEM_OK;
  double rmax = 0.;
  for (int i = 0; i < n; ++i) rmax = std::max(rmax, radius[i]);
  double L[3];
  int dims[3];
  for (int a = 0; a < 3; ++a) {
    L[a] = hi[a] - lo[a];
    dims[a] = std::max(1, (int)(L[a] / (2.0 * rmax)));
  }
  const size_t ncell = (size_t)dims[0] * dims[1] * dims[2];
  std::vector<std::vector<int>> cells(ncell);
  uint64_t st = seed * 0x9E3779B97F4A7C15ull + 1;
  auto rnd = [&]() {  // splitmix64 -> [0, 1)
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  auto cell_index = [&](const double* p) {
    int c[3];
    for (int a = 0; a < 3; ++a) {
      double u = (p[a] - lo[a]) / L[a];
      if (periodic) u -= std::floor(u);
      c[a] = std::min(dims[a] - 1, std::max(0, (int)(u * dims[a])));
    }
    return ((size_t)c[2] * dims[1] + c[1]) * dims[0] + c[0];
  };
  if (keep)
    for (int i = 0; i < n; ++i)
      if (keep[i]) cells[cell_index(pos_out + 3 * (size_t)i)].push_back(i);
  for (int i = 0; i < n; ++i) {
    if (keep && keep[i]) continue;
    const double r = radius[i];
    bool placed = false;
    for (int t = 0; t < max_tries && !placed; ++t) {
      double p[3];
      int c[3];
      for (int a = 0; a < 3; ++a) {
        p[a] = periodic ? lo[a] + rnd() * L[a] : lo[a] + r + rnd() * (L[a] - 2 * r);
        c[a] = std::min(dims[a] - 1, std::max(0, (int)((p[a] - lo[a]) / L[a] * dims[a])));
      }
      bool ok = true;
      for (int dz = -1; dz <= 1 && ok; ++dz)
        for (int dy = -1; dy <= 1 && ok; ++dy)
          for (int dx = -1; dx <= 1 && ok; ++dx) {
            int cc[3] = {c[0] + dx, c[1] + dy, c[2] + dz};
            bool skip = false;
            for (int a = 0; a < 3; ++a) {
              if (cc[a] < 0 || cc[a] >= dims[a]) {
                if (!periodic) skip = true;
                cc[a] = (cc[a] + dims[a]) % dims[a];
              }
            }
            if (skip) continue;
            for (int j : cells[((size_t)cc[2] * dims[1] + cc[1]) * dims[0] + cc[0]]) {
              double d2 = 0.;
              for (int a = 0; a < 3; ++a) {
                double dd = pos_out[3 * (size_t)j + a] - p[a];
                if (periodic) dd -= L[a] * std::round(dd / L[a]);
                d2 += dd * dd;
              }
              const double R = r + radius[j];
              if (d2 < R * R) { ok = false; break; }
            }
          }
      if (ok) {
        for (int a = 0; a < 3; ++a) pos_out[3 * (size_t)i + a] = p[a];
        cells[((size_t)c[2] * dims[1] + c[1]) * dims[0] + c[0]].push_back(i);
        placed = true;
      }
    }
    if (!placed) return LSDEM_ERR_ARG;
  }
  return LSDEM_OK;
}


// ---------------------------------------------------------------------------
// Snapshots: the dynamic state of a running solver in one binary file (no counterpart
// in the reference, whose host mirrors are written only as VTU frames). Layout, little
// endian: "LSDEMSNP", u32 version 1; i32 particles, walls, image sets, 0; i64 surface
// nodes, bonds, steps; f64 time; particles: position, velocity, angular velocity (3 f64
// each), orientation (4), force, torque (3); walls: position, velocity, angular velocity
// (3), orientation (4); bonds: flag (i32), state (9 f64); contact history: i64 contacts,
// per partner kind (particles, walls, images) i32 slot capacity and, when > 0, i32 per
// particle slot count, then per particle and slot partner id, segment start and segment
// length (i32); per contact i32 node and 3 f64 spring.

}  // extern "C"

namespace {
struct SnapIO {
  FILE* f;
  bool ok = true;
  void w(const void* p, size_t b) { if (b && std::fwrite(p, 1, b, f) != b) ok = false; }
  void r(void* p, size_t b) { if (b && std::fread(p, 1, b, f) != b) ok = false; }
};
constexpr char kSnapMagic[8] = {'L', 'S', 'D', 'E', 'M', 'S', 'N', 'P'};

template <class T>
void snap_dl(SnapIO& io, const DArr<T>& d, size_t n, cudaStream_t st) {
  std::vector<T> h(n);
  if (n) CK(cudaMemcpyAsync(h.data(), d.p, n * sizeof(T), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  io.w(h.data(), n * sizeof(T));
}
template <class T>
void snap_ul(SnapIO& io, DArr<T>& d, size_t n, cudaStream_t st) {
  std::vector<T> h(n);
  io.r(h.data(), n * sizeof(T));
  if (!io.ok) throw Fail{LSDEM_ERR_ARG, "snapshot file truncated"};
  if (n) CK(cudaMemcpyAsync(d.p, h.data(), n * sizeof(T), cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
}
}  // namespace

extern "C" {

int lsdem_snapshot_save(lsdem_solver* s, const char* path) {
  if (!s || !path) return LSDEM_ERR_ARG;
  if (!s->ready) return fail(s, LSDEM_ERR_STATE, "lsdem_snapshot_save before lsdem_initialize");
  return guard(s, [&] {
    FILE* f = std::fopen(path, "wb");
    if (!f) throw Fail{LSDEM_ERR_ARG, std::string("cannot open ") + path};
    SnapIO io{f};
    cudaStream_t st = s->stream;
    CK(cudaStreamSynchronize(st));
    const int np = s->P.n(), nw = s->W.n();
    const uint32_t ver = 1;
    const int32_t hdr[4] = {np, nw, s->nsets, 0};
    const long long nb = (long long)s->bonds.bonded.size();
    const long long h64[3] = {s->dev_nodes, nb, s->steps};
    io.w(kSnapMagic, 8); io.w(&ver, 4); io.w(hdr, 16); io.w(h64, 24); io.w(&s->time, 8);
    snap_dl(io, s->dP.pos, np, st); snap_dl(io, s->dP.vel, np, st); snap_dl(io, s->dP.angvel, np, st);
    snap_dl(io, s->dP.quat, np, st); snap_dl(io, s->dP.force, np, st); snap_dl(io, s->dP.torque, np, st);
    snap_dl(io, s->dW.pos, nw, st); snap_dl(io, s->dW.vel, nw, st); snap_dl(io, s->dW.angvel, nw, st);
    snap_dl(io, s->dW.quat, nw, st);
    snap_dl(io, s->b_bonded, (size_t)nb, st); snap_dl(io, s->b_state, (size_t)nb * 9, st);
    io.w(&s->hist_count, 8);
    for (int k = 0; k < 3; ++k) {
      SlotsDev& sl = s->slots[s->hp][k];
      const int32_t cap = sl.cnt.p ? sl.cap : 0;
      io.w(&cap, 4);
      if (cap <= 0) continue;
      const size_t m = (size_t)np * cap;
      snap_dl(io, sl.cnt, np, st); snap_dl(io, sl.id, m, st); snap_dl(io, sl.seg_start, m, st);
      snap_dl(io, sl.seg_cnt, m, st);
    }
    snap_dl(io, s->con[s->hp].node, (size_t)s->hist_count, st);
    snap_dl(io, s->con[s->hp].spring, (size_t)s->hist_count, st);
    const bool ok = io.ok;
    if (std::fclose(f) != 0 || !ok) throw Fail{LSDEM_ERR_ARG, std::string("cannot write ") + path};
    return LSDEM_OK;
  });
}

int lsdem_snapshot_load(lsdem_solver* s, const char* path) {
  if (!s || !path) return LSDEM_ERR_ARG;
  if (!s->ready) return fail(s, LSDEM_ERR_STATE, "lsdem_snapshot_load before lsdem_initialize");
  return guard(s, [&] {
    FILE* f = std::fopen(path, "rb");
    if (!f) throw Fail{LSDEM_ERR_ARG, std::string("cannot open ") + path};
    struct Closer { FILE* f; ~Closer() { std::fclose(f); } } closer{f};
    SnapIO io{f};
    cudaStream_t st = s->stream;
    char magic[8];
    uint32_t ver = 0;
    int32_t hdr[4];
    long long h64[3];
    double t = 0.;
    io.r(magic, 8); io.r(&ver, 4); io.r(hdr, 16); io.r(h64, 24); io.r(&t, 8);
    if (!io.ok || std::memcmp(magic, kSnapMagic, 8) != 0 || ver != 1) throw Fail{LSDEM_ERR_ARG, "not a snapshot file"};
    const int np = s->P.n(), nw = s->W.n();
    const long long nb = (long long)s->bonds.bonded.size();
    if (hdr[0] != np || hdr[1] != nw || hdr[2] != s->nsets || h64[0] != s->dev_nodes || h64[1] != nb)
      throw Fail{LSDEM_ERR_ARG, "snapshot does not match the solver's bodies, nodes, bonds or image sets"};
    CK(cudaStreamSynchronize(st));
    snap_ul(io, s->dP.pos, np, st); snap_ul(io, s->dP.vel, np, st); snap_ul(io, s->dP.angvel, np, st);
    snap_ul(io, s->dP.quat, np, st); snap_ul(io, s->dP.force, np, st); snap_ul(io, s->dP.torque, np, st);
    snap_ul(io, s->dW.pos, nw, st); snap_ul(io, s->dW.vel, nw, st); snap_ul(io, s->dW.angvel, nw, st);
    snap_ul(io, s->dW.quat, nw, st);
    snap_ul(io, s->b_bonded, (size_t)nb, st); snap_ul(io, s->b_state, (size_t)nb * 9, st);
    // walls' prescribed velocities are host settings too
    if (nw) {
      CK(cudaMemcpy(s->W.vel.data(), s->dW.vel.p, 24 * (size_t)nw, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(s->W.angvel.data(), s->dW.angvel.p, 24 * (size_t)nw, cudaMemcpyDeviceToHost));
    }
    long long hc = 0;
    io.r(&hc, 8);
    int32_t caps[3] = {0, 0, 0};
    std::vector<std::vector<int>> slot_data[3];
    for (int k = 0; k < 3; ++k) {
      io.r(&caps[k], 4);
      if (!io.ok || caps[k] < 0) throw Fail{LSDEM_ERR_ARG, "snapshot file truncated"};
      if (caps[k] == 0) continue;
      const size_t m = (size_t)np * caps[k];
      slot_data[k].resize(4);
      slot_data[k][0].resize(np);
      for (int a = 1; a < 4; ++a) slot_data[k][a].resize(m);
      io.r(slot_data[k][0].data(), 4 * (size_t)np);
      for (int a = 1; a < 4; ++a) io.r(slot_data[k][a].data(), 4 * m);
    }
    std::vector<int> node((size_t)hc);
    std::vector<double3> spring((size_t)hc);
    io.r(node.data(), 4 * (size_t)hc);
    io.r(spring.data(), 24 * (size_t)hc);
    if (!io.ok) throw Fail{LSDEM_ERR_ARG, "snapshot file truncated"};
    // capacities at least those of the file
    bool realloc = false;
    int* capv[3] = {&s->cap_pp, &s->cap_w, &s->cap_g};
    for (int k = 0; k < 3; ++k)
      if (caps[k] > *capv[k]) { *capv[k] = caps[k]; realloc = true; }
    if (realloc) alloc_slots(s);
    if (hc > s->con[0].cap) {
      s->cap_c = std::max<long long>(s->cap_c, hc + hc / 2);
      alloc_contacts(s, s->con[0], s->cap_c);
      alloc_contacts(s, s->con[1], s->cap_c);
      alloc_maybe(s);
    }
    for (int k = 0; k < 3; ++k) {
      SlotsDev& sl = s->slots[s->hp][k];
      if (!sl.cnt.p) continue;
      CK(cudaMemset(sl.cnt.p, 0, 4 * (size_t)std::max(np, 1)));
      if (caps[k] == 0 || np == 0) continue;
      CK(cudaMemcpy(sl.cnt.p, slot_data[k][0].data(), 4 * (size_t)np, cudaMemcpyHostToDevice));
      for (int a = 1; a < 4; ++a) {
        DArr<int>& dst = a == 1 ? sl.id : (a == 2 ? sl.seg_start : sl.seg_cnt);
        CK(cudaMemcpy2D(dst.p, sizeof(int) * sl.cap, slot_data[k][a].data(), sizeof(int) * caps[k],
                        sizeof(int) * caps[k], np, cudaMemcpyHostToDevice));
      }
    }
    if (hc) {
      CK(cudaMemcpy(s->con[s->hp].node.p, node.data(), 4 * (size_t)hc, cudaMemcpyHostToDevice));
      CK(cudaMemcpy(s->con[s->hp].spring.p, spring.data(), 24 * (size_t)hc, cudaMemcpyHostToDevice));
    }
    const int c32 = (int)hc;
    CK(cudaMemcpy(s->con[s->hp].count.p, &c32, sizeof(int), cudaMemcpyHostToDevice));
    s->con[s->hp].geom = false;
    s->hist_count = hc;
    s->time = t;
    s->steps = h64[2];
    s->host_stale = true;
    s->force_reuse = true;
    ++s->graph_gen;
    return LSDEM_OK;
  });
}

}  // extern "C"
