// Internal interface between the host runtime and the CUDA kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>
#include "common.cuh"
#include "mlp.cuh"

namespace lsdem {

// Compatibility switches for two arithmetic quirks of the reference
// (both on by default, so results follow the reference):
//   LSDEM_FIX_GRADIENT: use the true x weight in the SDF gradient instead of the
//     int-truncated one (LSParticleContactDetectionKernel.cuh:34-52);
//   LSDEM_FIX_SQRTF: double-precision square roots in the damping terms instead
//     of sqrtf (contactKernel.cuh:51,53,58).
enum { FIX_GRADIENT = 1, FIX_SQRTF = 2 };

// Overflow bits of the device status word.
enum { OVF_PP = 1, OVF_WALL = 2, OVF_GHOST = 4, OVF_CONTACT = 8, OVF_NBR = 16, OVF_NET = 32 };

// Largest demands seen during a batch (whether or not they overflowed), used
// to grow capacities ahead of an overflow.
struct Status {
  int flags;
  int need_pp;       // largest per-particle particle-candidate count
  int need_wall;     // largest per-particle wall-candidate count
  int need_ghost;    // largest per-particle ghost-candidate count
  int need_contact;  // largest contact total
  int need_nbr;      // largest per-particle neighbour-list length
  int builds;        // steps that sorted and rebuilt the neighbour lists
  int need_netq;     // learned form: largest rows of one shape's network queue
  int need_pend;     // learned form: largest count of nodes awaiting the network
  int errors;        // a bounded wait in a kernel gave up (results of the batch not valid)
  int pad;
};

// Shape templates: SDF grid + surface nodes in cluster order.
struct ShapeView {
  const int3* gsize;          // per shape
  const long long* sdf_off;   // per shape, into sdf
  const double* sdf;          // FP64 SDF store
  const int* node_off;        // per shape, into node_pos
  const int* node_cnt;        // per shape
  const int* cl_off;          // per shape, into cl_sphere
  const int* cl_cnt;          // per shape
  const double3* node_pos;    // node store, cluster order, unscaled
  const int* node_orig;       // original node index within the shape
  const double4* cl_sphere;   // cluster bounding sphere (xyz centre, w radius), unscaled
  const float4* cl_sphere_f;  // the same rounded to FP32 (the precision forms' screen)
  const float4* sub_sphere;   // 4 per cluster (same shape offsets x 4): spheres of 8 nodes,
                              //   unscaled; radius < 0 for a sub-cluster past the last node
  const double* node_box;     // 8 per shape (unscaled): node bounding box lo xyz, hi xyz,
                              //   largest node distance from the body origin, 0
  // precision form: SDF values / template spacing in 16-bit floats (FP16 or BF16
  // bits), cell-major: the 8 corners of cell (i, j, k) in one uint4, corner
  // dx + 2 dy + 4 dz in 16-bit lane order, cells x-fastest; FP32 nodes
  const uint4* cell16;
  const long long* cell_off;    // per shape, into cell16
  const float4* node_pos_f;     // FP32 copy of node_pos
  const float* lip;             // 2 per shape, in spacings: largest |phi| difference of grid
                                //   neighbours; largest gradient-norm bound of a grid cell
  // support tables (cube map of SUP_M x SUP_M cells per face, per shape, template units,
  // rounded up): per cell the values at its four corner directions (p, q), (p + 1, q),
  // (p, q + 1), (p + 1, q + 1) of the largest projection of the nodes (sup_n) and of the
  // points bounding the solid (sup_s, where the trilinear phi can be <= 0)
  const float4* sup_n;
  const float4* sup_s;
  const float* sup_r;           // per shape: largest |p| over the sup_s points, rounded up
};

// Arithmetic form of the narrowphase and contact forces.
enum { PREC_FP64 = 0, PREC_FP32_FP16 = 1, PREC_FP32_BF16 = 2 };

// Support tables: cells per cube-map face side; corner directions of the cells.
constexpr int SUP_M = 24;
constexpr int SUP_CELLS = 6 * SUP_M * SUP_M;
constexpr int SUP_VERTS = 6 * (SUP_M + 1) * (SUP_M + 1);
void launch_support_tables(int nshapes, const double3* node_pos, const int* node_off, const int* node_cnt,
                           const double3* pts, const long long* pts_off, float* vtx, float4* sup_n, float4* sup_s,
                           float* sup_r, cudaStream_t s);

// A set of rigid bodies (particles or walls).
struct BodyView {
  int n;
  double3* pos;
  double3* vel;
  double3* angvel;
  double3* force;
  double3* torque;
  Quat* quat;
  const double* invmass;
  const Sym6* invI;
  const double* radius;
  const double* kn;
  const double* ks;
  const double* mu;
  const double* res;
  const int* shape;
  const double* scale;       // uniform template scale
  const double3* origin;     // grid node (0,0,0) in body frame (scaled)
  const double* invh;        // inverse grid spacing (scaled)
  const long long* node_base;  // global id of the first surface node (particles)
  int* key;                  // cell key of this step, -1 outside the domain
  float4* rotm;              // precision form, particles: rows of the FP32 rotation matrix
                             //   of quat (3 per body, written by k_integrate_first)
};

// Per-particle candidate slots of one partner kind, with the contact segment
// each slot produced.
struct SlotView {
  int cap;
  int* cnt;        // per particle
  int* id;         // n * cap partner ids
  int* seg_start;  // n * cap
  int* seg_cnt;    // n * cap
};

struct ContactView {
  int cap;
  int* count;          // device counter
  int* node;           // node index within the owner's shape (cluster order)
  double3* spring;     // tangential spring (FP64 history)
  double3* point;      // optional geometry (nullptr when not recorded)
  double3* normal;
  double* overlap;
  double* en_n;
  double* en_s;
};

// Ghost images of the periodic boundary: up to 7 image sets (translations along x,
// y, z and their combinations), or the 3 rotated sets of sector periodicity.
struct GhostView {
  int nsets;
  int mask[7];         // axes of each set (bit 0 x, 1 y, 2 z); sector sets 8, 16, 32 (90, 180, 270 degrees)
  int sector;          // sector periodicity: images rotated about the z axis through the domain minimum
  Quat* gquat;         // sector: nsets * n image orientations
  double3* gvel;       // sector: nsets * n image velocities
  double3* gpos;       // nsets * n
  int* gkey;           // nsets * n, clamped cell or -1
  int* list;           // nsets * n: visible images (set * n + particle), compacted
  int* count;          // number of entries in list
};

// Scratch of the bucket sort: counts, fill and offsets of cells + 3 buckets each,
// scan partial sums (scan_temp_elems), the list of buckets over 64 members (n / 65 + 1),
// two counters (buckets over 64, buckets of 9 to 64 members), and n entries that hold
// the list of 9-to-64-member buckets and then the large buckets' copies.
struct BucketScratch {
  int* counts;
  int* fill;
  int* offs;
  int* scan_tmp;
  int* big_list;
  int* big_count;  // 2 entries
  int* tmp;
};

size_t scan_temp_elems(long long n);
// gate (optional): the launches return at once when *gate is zero
void scan_i32(const int* in, int* out, long long n, int* tmp, bool inclusive, cudaStream_t s,
              const int* gate = nullptr);
void scan_i64(const long long* in, long long* out, long long n, long long* tmp, bool inclusive, cudaStream_t s);
void bucket_sort(const int* key, int n, int ncells, BucketScratch& w, int* sorted_idx, int* sorted_key, int* start,
                 int* end, cudaStream_t s, const int* gate = nullptr);

// Precision form: nodes the FP32 screen could not reject, by pair, for the FP64
// contact pass. One node cursor per step; one pair list per narrowphase launch
// (0: particles and walls, 1: periodic images).
struct MaybeView {
  int* node;    // cap node ids
  int cap;
  int4* pair;   // 2 * pcap entries {A, kind << 24 | slot, node start, node count}
  int pcap;
  int* ctr;     // [0] node cursor, [1 + launch] pairs queued
};

// Precision form: flat lists of candidate pairs (A * cap + slot) per partner
// kind, appended by the candidate searches, so that the screen gives one warp
// to each pair rather than to each owner particle.
struct PairLists {
  int* list[3];  // particles, walls, images: n * cap entries each
  int* ctr;      // [kind] entries appended this step (nullptr: lists not built)
};

// Learned form, per narrowphase launch (0: particles and walls, 1: periodic images):
// the screen passes every node it cannot reject by the partner's bounds to the
// network of the partner's shape (rows grouped by shape, for 128-row tensor-core
// tiles) and keeps, per pair in node order, the nodes awaiting the verdict; the
// network pass writes each verdict (after the grid test of the nodes it keeps) and
// the compaction pass queues the surviving nodes of each pair for the FP64 pass.
struct NetView {
  float4* row;            // nshapes * qcap rows of two float4: (u.x, u.y, u.z, pending index bits;
                          //   bit 31 set: within the error of the grid boundary) and (grid point
                          //   in the partner's grid x, y, z, the pair's threshold T)
  int* cnt;               // nshapes: rows appended this step
  int qcap;               // rows per shape
  int* pend_n;            // pcap: node index
  unsigned char* pend_v;  // pcap: 1 when the node goes on to the FP64 test
  int pcap;
  int4* pair;             // paircap: {A, kind << 24 | slot, pending start, pending count}
  int paircap;
  int* ctr;               // [0] pending cursor, [1] pair records
};

struct StepArgs {
  BodyView P;       // particles
  BodyView W;       // walls
  ShapeView S;
  GridP pg;         // particle grid
  GridP wg;         // wall grid
  const int* cell_idx;    // particle grid: sorted particle index
  float4* cell_pk;        // particle grid, sorted order: FP32 centre and bounding radius
  const int* cell_off;    // particle grid: sorted position of the first body of cell k at [k + 1]
                          //   (bucket offsets of the cell sort, ncells + 3 entries)
  const int* cell_start;
  const int* cell_end;
  SlotView pp, pw, pgh;          // this step
  SlotView pp_old, pw_old, pgh_old;  // previous step
  ContactView C, C_old;
  GhostView G;
  Status* status;
  double dt;
  double3 gravity;
  int flags;        // FIX_* bits
  int precision;    // PREC_*
  double rmax;      // largest particle bounding radius
  MaybeView mb;
  PairLists pl;
  // precision form, optional: screen counters (pairs, clusters tested, clusters
  // kept, 16-bit grid lookups of nodes, node tests, nodes queued for FP64,
  // network evaluations of nodes, sub-clusters kept)
  unsigned long long* screen_stats;
  // precision forms, optional: learned per-shape SDF in front of the grid screen
  const MlpInfer* mlp_inf;   // per shape (nullptr: off)
  const MlpNorm* mlp_norm;   // per shape
  const float* mlp_band;     // per shape: trust band + error bound, in template spacings
  NetView net[2];            // learned form, per narrowphase launch
  int nshapes;
  // Neighbour lists (exact, optional): *reuse is set non-zero when a particle moved
  // more than sqrt(move2) from its position at the last list build; the cell sort and
  // the list rebuild run only then. The step's kick clears it.
  int* reuse;
  double move2;
  float skin;             // neighbour-list margin beyond the candidate reach (length)
  double3* xb;            // particle order: position at the last list build
  int* nbr;               // sorted order of the last sort: entry j of position t at j * n + t
  int* nbr_cnt;           // sorted order: entries, -1 when the list overflowed
  int nbr_cap;
  int4* pk_meta;          // sorted order, written with cell_pk: cell key, body index, shape, FP32 scale bits
  float4* pk_q;           // sorted order, written with cell_pk: FP32 orientation
};

// Template data for the learned-SDF kernels (mlp.cu).
struct MlpShapeData {
  const MlpNorm* norm;
  const int3* gsize;
  const double3* origin;   // template grid origin
  const double* h;         // template grid spacing
  const double* sdf;
  const long long* sdf_off;
  const int* node_off;
  const int* node_cnt;
  const double3* node_pos;
};
void mlp_samples(const MlpShapeData& D, int nshapes, int S, unsigned long long seed, const MlpTrainOpts& opt,
                 float4* samples, cudaStream_t st);
cudaError_t mlp_train_step(float* params, const float4* samples, int nshapes, int S, int B, long long it,
                           float* partial, float* loss, float* m1, float* m2, float lr, int step, cudaStream_t st);
void mlp_pack(const float* params, int nshapes, MlpInfer* out, cudaStream_t st);
// fail (device int): set to 1 when a tensor-core wait gave up (results not valid)
void mlp_validate(const MlpShapeData& D, int nshapes, const MlpInfer* inf, int S2, unsigned long long seed,
                  const MlpTrainOpts& opt, const float* delta, unsigned* err_bits, int* fail, cudaStream_t st);
cudaError_t mlp_grad_once(const float* params, const float4* pts, int n, float* partial, float* loss, cudaStream_t st);
void mlp_forward(const float* params, const float4* pts, int n, float* y, cudaStream_t st);
void mlp_infer(const MlpInfer* inf, const MlpNorm& nm, const double3* pts, int n, float* phi, int* fail,
               cudaStream_t st);

void launch_integrate_first(const StepArgs& a, cudaStream_t s);
void launch_candidates(const StepArgs& a, cudaStream_t s);
void launch_narrowphase(const StepArgs& a, int kinds, cudaStream_t s);
// precision form: FP64 contact pass over the pairs queued by the screen of
// launch li (0: particles and walls, 1: periodic images)
void launch_contact_pass(const StepArgs& a, int li, cudaStream_t s);
// learned form, after the screen of launch li: the network pass (tensor cores) and the
// compaction of the surviving nodes for the contact pass (no-ops without the network)
void launch_net_screen(const StepArgs& a, int li, cudaStream_t s);
void launch_net_compact(const StepArgs& a, int li, cudaStream_t s);
void launch_kick(const StepArgs& a, cudaStream_t s);
void launch_periodic(const StepArgs& a, int axes, double3* out, cudaStream_t s);
// g2_off: bucket offsets of the image search's cell sort (cell k at [k + 1])
void launch_ghost_candidates(const StepArgs& a, const int* g2_idx, const int* g2_off, cudaStream_t s);
void launch_clamped_keys(const StepArgs& a, int* key2, cudaStream_t s);

// V-bonds.
struct BondView {
  int n;
  const int* ids;        // 2 per bond: master, slave
  const double* B;       // 4 per bond
  const double* geo;     // 5 per bond: radius, L0, tensile, cohesion, mu
  const double3* frames; // 8 per bond: master n1,n2,n3,pos, slave n1,n2,n3,pos
  int* bonded;
  double* state;         // 9 per bond: Un, Us, Ub, Ut, sigma_max, tau_max, point xyz
};
void launch_bonds(const StepArgs& a, const BondView& b, cudaStream_t s);
// Bonds from the recorded particle-particle contacts (bonds.cu): contacts per owner, then
// one bond per contact at offs[owner] + k: ids (2), frames (8 vectors), point.
void bonds_from_contacts_count(const SlotView& pp, int n, int* cnt, cudaStream_t s);
void bonds_from_contacts_make(const SlotView& pp, int n, const int* offs, const double3* point, const double3* normal,
                              const double3* pos, const Quat* quat, double Lb, int* ids, double3* frames,
                              double3* bpoint, int* bad, cudaStream_t s);


// ---------------------------------------------------------------------------
// Frame output (csrc/vtu.cu): what the writer needs of one solver's frame.
struct VtuError { std::string msg; };
struct VtuContacts { std::vector<double> point, normal, spring, en_n, en_s; };
struct VtuInput {
  std::string dir;                 // phase directory; the files go to its four subdirectories
  unsigned long long frame = 0, step = 0;
  double time = 0.;
  cudaStream_t solver_stream = nullptr;
  long long layout = 0;            // changes whenever bodies, templates or triangles change
  int n = 0;                       // particles; device state in particle order
  const double3* pos = nullptr;
  const double3* vel = nullptr;
  const double3* angvel = nullptr;
  const Quat* quat = nullptr;
  const double* radius = nullptr;  // device
  const long long* node_base = nullptr;  // host, n + 1, caller node order
  const int* shape = nullptr;      // host
  const double* scale = nullptr;   // host
  std::vector<const std::vector<double>*> tnodes;    // per shape, caller order
  const int* tri_set = nullptr;    // host, per particle (-1: no triangles)
  std::vector<const std::vector<int>*> tri_sets;
  int nw = 0;                      // walls; host state
  const double* wpos = nullptr;
  const double* wquat = nullptr;
  const double* wvel = nullptr;
  const double* wangvel = nullptr;
  std::vector<const std::vector<double>*> wall_verts;
  std::vector<const std::vector<int>*> wall_tris;    // null: no triangles
  VtuContacts pp, pw;
  std::vector<int> bond_ids, bond_bonded;
  std::vector<double> bond_state;
};
struct VtuCtx;
void vtu_write(VtuCtx*& ctx, const VtuInput& in);
void vtu_free(VtuCtx* ctx);
}  // namespace lsdem
