// FP64 CPU oracle for the level-set DEM step — TEST INFRASTRUCTURE ONLY.
//
// This file restates, on the CPU and in plain C++, the algorithm of the
// reference solver's GPU hot path so that the CUDA implementation can be
// checked against it. It is used only by tests/, by __graft_entry__.smoke()
// as the checker, and by bench.py's CPU-baseline leg. It is never part of
// the product path.
//
// Every function cites the reference code it follows (paths relative to the
// reference project root):
//   FunDEM/kernel/CUDAKernelFunction/myUtility/mySpatialGrid.cu   (hash, wrap, ghosts)
//   FunDEM/kernel/CUDAKernelFunction/myUtility/mySpatialGrid.h    (grid set-up, cell coords)
//   FunDEM/kernel/CUDAKernelFunction/myUtility/buildHashStartEnd.cu (sort + ranges)
//   FunDEM/kernel/CUDAKernelFunction/LSParticleContactDetectionKernel.cu/.cuh (narrowphase)
//   FunDEM/kernel/CUDAKernelFunction/contactKernel.cu/.cuh        (contact and bond forces)
//   FunDEM/kernel/CUDAKernelFunction/particleIntegrationKernel.cu (integration)
//   FunDEM/kernel/LSSolver.h                                      (mass properties, step order)
//
// Reference quirks kept by default (switch off with the ORA_FIX_* flags):
//   Q1  the SDF gradient takes the x fraction as an int (x weight 1/0),
//       LSParticleContactDetectionKernel.cuh:34-52;
//   Q2  damping uses single-precision sqrtf, contactKernel.cuh:51,53,58.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "ora_math.h"

using namespace ora;

extern "C" {

enum { ORA_FIX_GRADIENT = 1, ORA_FIX_SQRTF = 2 };

// Bodies that can be the SDF side of a test: particles, walls or ghost images.
typedef struct {
  int n;
  const double* pos;        // 3n
  const double* quat;       // 4n (q0 scalar first)
  const double* radius;     // n  (bounding radius, particle-particle test only)
  const double* invh;       // n  inverse grid spacing
  const double* origin;     // 3n grid node (0,0,0) in body frame
  const int* gsize;         // 3n grid node counts
  const long long* sdf_off; // n  first SDF value of this body in `sdf`
  const double* sdf;        // SDF store, index ix + nx*(iy + ny*iz)
  const double* sdf_scale;  // n or NULL: uniform scale s of a scaled template (value = s * stored)
} OraBodies;

// Surface nodes of the node-owning particles.
typedef struct {
  int np;
  const long long* node_base; // np+1: global node ids of particle p are [base[p], base[p+1])
  const long long* node_src;  // np: first node of particle p in node_local
  const double* node_local;   // 3 doubles per node, particle frame
  const double* node_scale;   // np or NULL: node position = s * stored
} OraNodes;

// Uniform hash grid and its sorted occupancy (reference spatialGrid + hash arrays).
typedef struct {
  double min[3], max[3], inv[3];
  int size[3];
  const int* idx;    // sorted body index
  const int* start;  // per cell, -1 if empty
  const int* end;
} OraGrid;

// Dynamic state and contact parameters of a body set.
typedef struct {
  int n;
  const double* pos;
  const double* vel;
  const double* angvel;
  const double* invmass;
  const double* kn;
  const double* ks;
  const double* mu;
  const double* res;
} OraDyn;

}  // extern "C" (types)

#define ORA_API extern "C"

static inline d3 ld3(const double* p, long long i) { return mk(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
static inline void st3(double* p, long long i, d3 v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }
static inline qt ldq(const double* p, long long i) { return qt{p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]}; }

// ---------------------------------------------------------------------------
// Grid set-up: spatialGrid::set (mySpatialGrid.h:212-240).
ORA_API void ora_grid_set(const double* mn, const double* mx_in, double cell, double* inv_out, int* size_out, double* max_out) {
  double mx[3] = {mx_in[0], mx_in[1], mx_in[2]};
  for (int a = 0; a < 3; ++a)
    if (mx[a] <= mn[a]) mx[a] = mn[a] + cell;
  for (int a = 0; a < 3; ++a) max_out[a] = mx[a];
  if (is_zero(cell)) {
    for (int a = 0; a < 3; ++a) { size_out[a] = 2; inv_out[a] = 0.0; }
    return;
  }
  for (int a = 0; a < 3; ++a) {
    double d = mx[a] - mn[a];
    size_out[a] = d > 2. * cell ? int(d / cell) : 2;
    inv_out[a] = (d > 0.0) ? (double(size_out[a]) / d) : 0.0;
  }
}

// Cell coordinate with int() truncation: calculateGridPosition (mySpatialGrid.h:24-31).
static inline void cell_of(d3 p, const double* mn, const double* inv, int* c) {
  c[0] = int((p.x - mn[0]) * inv[0]);
  c[1] = int((p.y - mn[1]) * inv[1]);
  c[2] = int((p.z - mn[2]) * inv[2]);
}

// calculateHashKernel (mySpatialGrid.cu:4-26).
ORA_API void ora_hash(int n, const double* pos, const double* mn, const double* mx, const double* inv, const int* size,
              int* key) {
  for (int i = 0; i < n; ++i) {
    d3 p = ld3(pos, i);
    if (p.x < mn[0] || p.x >= mx[0] || p.y < mn[1] || p.y >= mx[1] || p.z < mn[2] || p.z >= mx[2]) {
      key[i] = -1;
      continue;
    }
    int c[3];
    cell_of(p, mn, inv, c);
    key[i] = lin3(c[0], c[1], c[2], size[0], size[1]);
  }
}

// calculateGhostHashKernel (mySpatialGrid.cu:214-240), including the z-upper
// test against maxBound.y (mySpatialGrid.cu:236).
ORA_API void ora_ghost_hash(int n, const double* gpos, const double* mn, const double* mx, const double* inv,
                    const int* size, int* key) {
  for (int i = 0; i < n; ++i) {
    d3 p = ld3(gpos, i);
    int c[3];
    cell_of(p, mn, inv, c);
    bool out = false;
    if (p.x < mn[0]) { c[0] = 0; out = true; } else if (p.x >= mx[0]) { c[0] = size[0] - 1; out = true; }
    if (p.y < mn[1]) { c[1] = 0; out = true; } else if (p.y >= mx[1]) { c[1] = size[1] - 1; out = true; }
    if (p.z < mn[2]) { c[2] = 0; out = true; } else if (p.z >= mx[1]) { c[2] = size[2] - 1; out = true; }
    key[i] = out ? lin3(c[0], c[1], c[2], size[0], size[1]) : -1;
  }
}

// buildHashStartEnd (buildHashStartEnd.cu:69-137): identity index, stable sort
// of (key, index) by key (thrust::sort_by_key on int keys is a stable radix
// sort), then per-cell half-open ranges, -1 where empty.
ORA_API void ora_sort_ranges(int n, int* key, int* idx, int ncells, int* start, int* end) {
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
  std::vector<int> k2(n);
  for (int i = 0; i < n; ++i) { k2[i] = key[order[i]]; idx[i] = order[i]; }
  std::memcpy(key, k2.data(), sizeof(int) * (size_t)n);
  for (int c = 0; c < ncells; ++c) { start[c] = -1; end[c] = -1; }
  for (int i = 0; i < n; ++i) {
    int h = key[i];
    if (h < 0 || h >= ncells) continue;
    if (i == 0 || key[i - 1] != h) start[h] = i;
    if (i == n - 1 || key[i + 1] != h) end[h] = i + 1;
  }
}

// Periodic wrap along one axis: updatePositionOutOfBoundary{XD,YD}Kernel (mySpatialGrid.cu:28-56),
// extended to z with the same rule.
ORA_API void ora_wrap(int n, double* pos, const double* mn, const double* mx, int axis) {
  double L = mx[axis] - mn[axis];
  for (int i = 0; i < n; ++i) {
    double& c = pos[3 * i + axis];
    if (c < mn[axis]) c += L;
    else if (c >= mx[axis]) c -= L;
  }
}

// Ghost images for one image set: calculateGhostPosition{XD,YD,XYD}Kernel
// (mySpatialGrid.cu:87-152). `mask` bit a set => the set shifts along axis a;
// a particle is imaged when its cell coordinate is 0 along every axis of the set.
ORA_API void ora_ghost_positions(int n, const double* pos, const double* mn, const double* mx, const double* inv, int mask,
                         double* gpos) {
  for (int i = 0; i < n; ++i) {
    d3 p = ld3(pos, i);
    d3 g = p;
    int c[3];
    cell_of(p, mn, inv, c);
    bool hit = true;
    for (int a = 0; a < 3; ++a)
      if ((mask >> a) & 1) hit = hit && (c[a] == 0);
    if (hit) {
      d3 off = mk(0., 0., 0.);
      if (mask & 1) off = off + mk(mx[0] - mn[0], 0., 0.);
      if (mask & 2) off = off + mk(0., mx[1] - mn[1], 0.);
      if (mask & 4) off = off + mk(0., 0., mx[2] - mn[2]);
      g += off;
    }
    st3(gpos, i, g);
  }
}

// Sector periodicity (host arithmetic of the reference's helpers: rotateVector,
// myVec.h:143-182, and rotateQuaternion, myQua.h:131-179).
static d3 rotate_vector(d3 v, d3 om) {
  const double theta2 = dot(om, om);
  if (is_zero(theta2)) {
    const d3 oxv = cross(om, v), oxoxv = cross(om, oxv);
    return v + oxv + 0.5 * oxoxv;
  }
  const double inv = 1.0 / std::sqrt(theta2);
  const double theta = theta2 * inv;
  const double s = std::sin(theta), c = std::cos(theta);
  const double A = s * inv, B = (1.0 - c) * (inv * inv);
  const d3 oxv = cross(om, v), oxoxv = cross(om, oxv);
  return v + A * oxv + B * oxoxv;
}
static qt rotate_quaternion(qt q, d3 om) {
  const double theta2 = om.x * om.x + om.y * om.y + om.z * om.z;
  if (is_zero(theta2)) return q;
  const double theta = std::sqrt(theta2), inv = 1.0 / theta;
  const double ux = om.x * inv, uy = om.y * inv, uz = om.z * inv;
  const double half = 0.5 * theta, c = std::cos(half), s = std::sin(half);
  const double r0 = c, r1 = s * ux, r2 = s * uy, r3 = s * uz;
  qt r{r0 * q.q0 - r1 * q.q1 - r2 * q.q2 - r3 * q.q3, r0 * q.q1 + r1 * q.q0 + r2 * q.q3 - r3 * q.q2,
       r0 * q.q2 - r1 * q.q3 + r2 * q.q0 + r3 * q.q1, r0 * q.q3 + r1 * q.q2 - r2 * q.q1 + r3 * q.q0};
  return normalize(r);
}

// updateVelocityPositionOrientationOutOfSectorKernel (mySpatialGrid.cu:58-85): a particle
// left of x = m.x (y >= m.y) turns by -90 degrees about the z axis through m, one below
// y = m.y (x >= m.x) by +90 degrees (position about m, velocity, orientation; the angular
// velocity is not turned). force / torque (nullable) turn with the particle: the step
// evaluates the particle and wall forces before the wrap.
ORA_API void ora_sector_wrap(int n, double* pos, double* vel, double* quat, double* force, double* torque,
                             const double* mn) {
  const double hp = 0.5 * 3.14159265358979323846;
  const d3 m = mk(mn[0], mn[1], mn[2]);
  for (int i = 0; i < n; ++i) {
    d3 p = ld3(pos, i), v = ld3(vel, i);
    qt q = ldq(quat, i);
    for (int pass = 0; pass < 2; ++pass) {
      const bool hit = pass == 0 ? (p.x < m.x && p.y >= m.y) : (p.y < m.y && p.x >= m.x);
      if (!hit) continue;
      const d3 om = mk(0., 0., pass == 0 ? -hp : hp);
      v = rotate_vector(v, om);
      p = m + rotate_vector(p - m, om);
      q = rotate_quaternion(q, om);
      if (force) st3(force, i, rotate_vector(ld3(force, i), om));
      if (torque) st3(torque, i, rotate_vector(ld3(torque, i), om));
    }
    st3(pos, i, p);
    st3(vel, i, v);
    quat[4 * i] = q.q0; quat[4 * i + 1] = q.q1; quat[4 * i + 2] = q.q2; quat[4 * i + 3] = q.q3;
  }
}

// calculateSectorGhostVelocityPositionOrientationKernel (mySpatialGrid.cu:154-212): sets
// R90, R180, R270 (3 x n each); a particle is turned by 90 degrees when its cell row along
// y is 0, by 270 when its cell column along x is 0, by 180 when both, else copied.
ORA_API void ora_sector_ghosts(int n, const double* pos, const double* vel, const double* quat, const double* mn,
                               const double* inv, double* gpos, double* gvel, double* gquat) {
  const double hp = 0.5 * 3.14159265358979323846;
  const d3 m = mk(mn[0], mn[1], mn[2]);
  const double ang[3] = {hp, 2.0 * hp, -hp};
  for (int i = 0; i < n; ++i) {
    const d3 p = ld3(pos, i), v = ld3(vel, i);
    const qt q = ldq(quat, i);
    int c[3];
    cell_of(p, mn, inv, c);
    for (int s = 0; s < 3; ++s) {
      const bool on = s == 0 ? c[1] == 0 : (s == 1 ? (c[1] == 0 && c[0] == 0) : c[0] == 0);
      d3 gp = p, gv = v;
      qt gq = q;
      if (on) {
        const d3 om = mk(0., 0., ang[s]);
        gv = rotate_vector(v, om);
        gp = m + rotate_vector(p - m, om);
        gq = rotate_quaternion(q, om);
      }
      const long long k = (long long)s * n + i;
      st3(gpos, k, gp);
      st3(gvel, k, gv);
      gquat[4 * k] = gq.q0; gquat[4 * k + 1] = gq.q1; gquat[4 * k + 2] = gq.q2; gquat[4 * k + 3] = gq.q3;
    }
  }
}

// ---------------------------------------------------------------------------
// Narrowphase.
// Trilinear value: interpolateLevelSetFunctionValue (LSParticleContactDetectionKernel.cuh:4-32).
static inline double tri_value(double x, double y, double z, const double* c) {
  const double wx0 = 1.0 - x, wx1 = x, wy0 = 1.0 - y, wy1 = y, wz0 = 1.0 - z, wz1 = z;
  return c[0] * wx0 * wy0 * wz0 + c[1] * wx1 * wy0 * wz0 + c[2] * wx0 * wy1 * wz0 + c[3] * wx1 * wy1 * wz0 +
         c[4] * wx0 * wy0 * wz1 + c[5] * wx1 * wy0 * wz1 + c[6] * wx0 * wy1 * wz1 + c[7] * wx1 * wy1 * wz1;
}
// Gradient in grid units: interpolateLevelSetFunctionGradient (…cuh:34-77).
static inline d3 tri_grad(double x, double y, double z, const double* c) {
  const double wx0 = 1.0 - x, wx1 = x, wy0 = 1.0 - y, wy1 = y, wz0 = 1.0 - z, wz1 = z;
  double gx = (c[1] - c[0]) * wy0 * wz0 + (c[3] - c[2]) * wy1 * wz0 + (c[5] - c[4]) * wy0 * wz1 + (c[7] - c[6]) * wy1 * wz1;
  double gy = (c[2] - c[0]) * wx0 * wz0 + (c[3] - c[1]) * wx1 * wz0 + (c[6] - c[4]) * wx0 * wz1 + (c[7] - c[5]) * wx1 * wz1;
  double gz = (c[4] - c[0]) * wx0 * wy0 + (c[5] - c[1]) * wx1 * wy0 + (c[6] - c[2]) * wx0 * wy1 + (c[7] - c[3]) * wx1 * wy1;
  return mk(gx, gy, gz);
}

// Node-vs-body SDF test (…cu:59-115 / :355-409). Returns true when the node is
// inside the body's grid and overlap = -phi >= 0; fills the fractions and corners.
static inline bool sdf_test(const OraBodies* B, int j, d3 wpos, double* ov, double* fx, double* fy, double* fz,
                            double* corners) {
  const d3 rel = wpos - ld3(B->pos, j);
  const qt qB = ldq(B->quat, j);
  const d3 l = rotate_inv(rel, qB);
  const d3 o = ld3(B->origin, j);
  const double ih = B->invh[j];
  const int nx = B->gsize[3 * j], ny = B->gsize[3 * j + 1], nz = B->gsize[3 * j + 2];
  const double gx = (l.x - o.x) * ih, gy = (l.y - o.y) * ih, gz = (l.z - o.z) * ih;
  const int i0 = (int)std::floor(gx), j0 = (int)std::floor(gy), k0 = (int)std::floor(gz);
  if (i0 < 0 || j0 < 0 || k0 < 0) return false;
  if (i0 >= nx - 1 || j0 >= ny - 1 || k0 >= nz - 1) return false;
  const int i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
  *fx = gx - (double)i0; *fy = gy - (double)j0; *fz = gz - (double)k0;
  const double* s = B->sdf + B->sdf_off[j];
  corners[0] = s[lin3(i0, j0, k0, nx, ny)];
  corners[1] = s[lin3(i1, j0, k0, nx, ny)];
  corners[2] = s[lin3(i0, j1, k0, nx, ny)];
  corners[3] = s[lin3(i1, j1, k0, nx, ny)];
  corners[4] = s[lin3(i0, j0, k1, nx, ny)];
  corners[5] = s[lin3(i1, j0, k1, nx, ny)];
  corners[6] = s[lin3(i0, j1, k1, nx, ny)];
  corners[7] = s[lin3(i1, j1, k1, nx, ny)];
  if (B->sdf_scale) {
    const double sc = B->sdf_scale[j];
    for (int c = 0; c < 8; ++c) corners[c] = sc * corners[c];
  }
  *ov = -tri_value(*fx, *fy, *fz, corners);
  return *ov >= 0.;
}

// Visits the candidate bodies of one node in the reference's order: 27-cell walk
// z, y, x with edge clamping (…cu:35-57), then sorted occupants of each cell.
// mode 0 applies the particle-particle filters idxA < idxB and |r| <= rad_B (…cu:58-61).
template <class F>
static inline void walk(int mode, const OraBodies* B, const OraGrid* g, int idxA, d3 w, F&& visit) {
  int c[3];
  cell_of(w, g->min, g->inv, c);
  int s[3] = {-1, -1, -1}, e[3] = {1, 1, 1};
  for (int a = 0; a < 3; ++a) {
    if (c[a] <= 0) { c[a] = 0; s[a] = 0; }
    if (c[a] >= g->size[a] - 1) { c[a] = g->size[a] - 1; e[a] = 0; }
  }
  for (int zz = s[2]; zz <= e[2]; zz++)
    for (int yy = s[1]; yy <= e[1]; yy++)
      for (int xx = s[0]; xx <= e[0]; xx++) {
        const int h = lin3(c[0] + xx, c[1] + yy, c[2] + zz, g->size[0], g->size[1]);
        const int st = g->start[h];
        if (st == -1) continue;
        const int en = g->end[h];
        for (int i = st; i < en; i++) {
          const int idxB = g->idx[i];
          if (mode == 0) {
            if (idxA >= idxB) continue;
            const d3 r = w - ld3(B->pos, idxB);
            const double rb = B->radius[idxB];
            if (len2(r) > rb * rb) continue;
          }
          visit(idxB);
        }
      }
}

static inline d3 node_world(const OraNodes* nd, const double* ppos, const double* pquat, int p, long long k) {
  d3 local = ld3(nd->node_local, nd->node_src[p] + k);
  if (nd->node_scale) local = nd->node_scale[p] * local;
  return rotate(ldq(pquat, p), local) + ld3(ppos, p);
}

// countLevelSetBoundaryNode{,FixedParticle}InteractionsKernel (…cu:4-122, :299-416).
// Writes count[node id] for the nodes of particles p0..p1-1.
ORA_API void ora_detect_count(int mode, const OraNodes* nd, const double* ppos, const double* pquat, const OraBodies* B,
                      const OraGrid* g, int p0, int p1, int* count) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int p = p0; p < p1; ++p) {
    const long long nb = nd->node_base[p], ne = nd->node_base[p + 1];
    for (long long id = nb; id < ne; ++id) {
      const d3 w = node_world(nd, ppos, pquat, p, id - nb);
      int cnt = 0;
      walk(mode, B, g, p, w, [&](int j) {
        double ov, fx, fy, fz, cr[8];
        if (sdf_test(B, j, w, &ov, &fx, &fy, &fz, cr)) cnt++;
      });
      count[id] = cnt;
    }
  }
}

// writeLevelSetBoundaryNode{,FixedParticle}InteractionsKernel (…cu:124-297, :418-590).
// `prefix` is the inclusive scan of this step's counts, `prefix_old` the one of
// the previous step (history carried over by a linear search of the node's old
// partners, …cu:280-289).
ORA_API void ora_detect_write(int mode, const OraNodes* nd, const double* ppos, const double* pquat, const OraBodies* B,
                      const OraGrid* g, int p0, int p1, const int* prefix, const int* prefix_old,
                      const int* partner_old, const double* spring_old, int flags, double* spring, double* point,
                      double* normal, double* overlap, long long* node_out, int* partner_out, int* owner_out) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int p = p0; p < p1; ++p) {
    const long long nb = nd->node_base[p], ne = nd->node_base[p + 1];
    for (long long id = nb; id < ne; ++id) {
      int base_w = 0, base_old = 0;
      if (id > 0) { base_w = prefix[id - 1]; base_old = prefix_old[id - 1]; }
      const int end_w = prefix[id];
      if (end_w - base_w == 0) continue;
      const int end_old = prefix_old[id];
      const d3 w = node_world(nd, ppos, pquat, p, id - nb);
      int cnt = 0;
      walk(mode, B, g, p, w, [&](int j) {
        double ov, fx, fy, fz, cr[8];
        if (!sdf_test(B, j, w, &ov, &fx, &fy, &fz, cr)) return;
        const long long k = base_w + cnt;
        const double gxw = (flags & ORA_FIX_GRADIENT) ? fx : (double)(int)fx;
        d3 n = tri_grad(gxw, fy, fz, cr);
        n = rotate(ldq(B->quat, j), n);
        n = normalize(n);
        st3(point, k, w + 0.5 * ov * n);
        st3(normal, k, n);
        overlap[k] = ov;
        node_out[k] = id;
        partner_out[k] = j;
        owner_out[k] = p;
        d3 ss = mk(0., 0., 0.);
        for (int q = base_old; q < end_old; q++)
          if (j == partner_old[q]) { ss = ld3(spring_old, q); break; }
        st3(spring, k, ss);
        cnt++;
      });
    }
  }
}

// ---------------------------------------------------------------------------
// Contact forces.
static inline double sqrt_damp(double v, int flags) {
  return (flags & ORA_FIX_SQRTF) ? std::sqrt(v) : (double)sqrtf((float)v);
}

// integrateSlidingSpring (contactKernel.cuh:4-34).
static inline d3 sliding_spring(d3 prev, d3 sv, d3 n, d3 fn, double mu, double k, double c, double dt) {
  d3 spring = mk(0., 0., 0.);
  if (mu > 0. && k > 0.) {
    d3 p1 = prev - dot(prev, n) * n;
    const double a1 = len(p1);
    if (!is_zero(a1)) p1 *= len(prev) / a1;
    spring = p1 + sv * dt;
    d3 fs = -k * spring - c * sv;
    const double afs = len(fs), afn = len(fn);
    if (!is_zero(afs) && afs > mu * afn) {
      double ratio = mu * afn / afs;
      fs *= ratio;
      spring = -(fs + c * sv) / k;
    }
  }
  return spring;
}

// LinearContact (contactKernel.cuh:36-77).
static inline void linear_contact(d3& F, d3& spring, d3 vc, d3 n, double delta, double dt, double kn, double ks,
                                  double mu, double e, double effM, int flags) {
  if (delta > 0.) {
    const double logRes = std::log(e);
    const double diss = -logRes / sqrt_damp(logRes * logRes + M_PI * M_PI, flags);
    const double cn = 2. * diss * sqrt_damp(effM * kn, flags);
    const d3 vn = dot(vc, n) * n;
    const d3 fn = kn * delta * n - cn * vn;
    const double cs = 2. * diss * sqrt_damp(effM * ks, flags);
    const d3 vs = vc - vn;
    spring = sliding_spring(spring, vs, n, fn, mu, ks, cs, dt);
    const d3 fs = -ks * spring - cs * vs;
    F = fn + fs;
  } else {
    spring = mk(0., 0., 0.);
  }
}

static inline void add3(double* arr, int i, d3 v, bool par) {
  if (par) {
#pragma omp atomic
    arr[3 * i] += v.x;
#pragma omp atomic
    arr[3 * i + 1] += v.y;
#pragma omp atomic
    arr[3 * i + 2] += v.z;
  } else {
    arr[3 * i] += v.x; arr[3 * i + 1] += v.y; arr[3 * i + 2] += v.z;
  }
}

// kind 0: particle-particle  addLevelSetParticleContactForceTorqueKernel (contactKernel.cu:46-118)
// kind 1: particle-wall      addFixedLevelSetParticleContactForceTorqueKernel (:120-191)
// kind 2: particle-ghost     addGhostLevelSetParticleContactForceTorqueKernel (:193-271);
//         J holds ghost pos/vel with the real particles' angvel and parameters.
// Contacts are processed in list order; with nthreads > 1 the particle sums use atomics.
ORA_API void ora_contact_force(int kind, long long nc, const int* owner, const int* partner, const double* point,
                       const double* normal, const double* overlap, double* spring, double* en_n, double* en_s,
                       const OraDyn* P, const OraDyn* J, double dt, int flags, double* force, double* torque,
                       int nthreads) {
  const bool par = nthreads > 1;
#pragma omp parallel for if (par) num_threads(par ? nthreads : 1) schedule(static)
  for (long long k = 0; k < nc; ++k) {
    const int i = owner[k];
    const d3 ri = ld3(P->pos, i), vi = ld3(P->vel, i), wi = ld3(P->angvel, i);
    const double invMi = P->invmass[i], kni = P->kn[i], ksi = P->ks[i], mui = P->mu[i], resi = P->res[i];
    const int j = partner[k];
    const d3 rj = ld3(J->pos, j), vj = ld3(J->vel, j), wj = ld3(J->angvel, j);
    const d3 rc = ld3(point, k), n = ld3(normal, k);
    const double delta = overlap[k];
    const d3 vc = vi + cross(wi, rc - ri) - (vj + cross(wj, rc - rj));
    double kn = 0., ks = 0., effM = 0., mu, res;
    if (kind == 1) {
      kn = kni; ks = ksi;
      if (invMi > 0.) effM = 1. / invMi;
      mu = std::fmin(mui, J->mu[j]);
      res = std::fmin(resi, J->res[j]);
    } else {
      const double invMj = J->invmass[j], knj = J->kn[j], ksj = J->ks[j];
      if (kni > 0. && knj > 0.) kn = kni * knj / (kni + knj);
      if (ksi > 0. && ksj > 0.) ks = ksi * ksj / (ksi + ksj);
      if (invMi > 0. || invMj > 0.) effM = 1. / (invMi + invMj);
      res = std::fmin(resi, J->res[j]);
      mu = std::fmin(mui, J->mu[j]);
    }
    d3 F = mk(0., 0., 0.);
    d3 s = ld3(spring, k);
    linear_contact(F, s, vc, n, delta, dt, kn, ks, mu, res, effM, flags);
    st3(spring, k, s);
    if (en_n) en_n[k] = 0.5 * delta * delta * kn;
    if (en_s) en_s[k] = 0.5 * len2(s) * ks;
    add3(force, i, F, par);
    add3(torque, i, cross(rc - ri, F), par);
    if (kind == 0 || (kind == 2 && i != j)) {
      add3(force, j, -F, par);
      add3(torque, j, cross(rc - rj, -F), par);
    }
  }
}

// VBond + addBondedForceTorqueKernel (contactKernel.cuh:138-199, contactKernel.cu:273-351).
// Per-bond arrays: ids (2), B[4], radius, L0, tensile, cohesion, mu, local frames
// n1,n2,n3,pos for master (12) and slave (12). `state` per bond:
// Un, Us, Ub, Ut, sigma_max, tau_max, point(3).
ORA_API void ora_bond_force(int nb, const int* ids, const double* Bk, const double* geo, const double* frames,
                    int* bonded, double* state, const double* ppos, const double* pquat, double* force,
                    double* torque) {
  for (int k = 0; k < nb; ++k) {
    double* st = state + 9 * k;
    if (bonded[k] == 0) {
      for (int a = 0; a < 6; ++a) st[a] = 0.;
      continue;
    }
    const int i = ids[2 * k], j = ids[2 * k + 1];
    const qt qi = ldq(pquat, i), qj = ldq(pquat, j);
    const double* fr = frames + 24 * k;
    const d3 n1i = rotate(qi, ld3(fr, 0)), n2i = rotate(qi, ld3(fr, 1)), n3i = rotate(qi, ld3(fr, 2));
    const d3 n1j = rotate(qj, ld3(fr, 4)), n2j = rotate(qj, ld3(fr, 5)), n3j = rotate(qj, ld3(fr, 6));
    const d3 ri = ld3(ppos, i), rj = ld3(ppos, j);
    const d3 rbi = rotate(qi, ld3(fr, 3)) + ri;
    const d3 rbj = rotate(qj, ld3(fr, 7)) + rj;
    const d3 bp = 0.5 * (rbi + rbj);
    st[6] = bp.x; st[7] = bp.y; st[8] = bp.z;
    const double B1 = Bk[4 * k], B2 = Bk[4 * k + 1], B3 = Bk[4 * k + 2], B4 = Bk[4 * k + 3];
    const double Rb = geo[5 * k], D0 = geo[5 * k + 1], ten = geo[5 * k + 2], coh = geo[5 * k + 3], fmu = geo[5 * k + 4];
    d3 F = mk(0., 0., 0.), Mij = mk(0., 0., 0.), Mji = mk(0., 0., 0.);
    int ok = 1;
    const d3 rbij = rbi - rbj;
    const double D = len(rbij);
    if (!is_zero(D)) {
      const d3 nij = normalize(rbij);
      const d3 e = -nij;
      st[0] = 0.5 * B1 * (D - D0) * (D - D0);
      st[1] = B2 * (0.5 * dot((n1j - n1i), e) - 0.25 * dot(n1i, n1j) + 0.75);
      st[2] = (0.25 * B2 + B3 + 0.5 * B4) * (dot(n1i, n1j) + 1.);
      st[3] = -0.5 * B4 * (dot(n1i, n1j) + dot(n2i, n2j) + dot(n3i, n3j) - 1);
      F = B1 * (D - D0) * e + B2 / (2 * D) * ((n1j - n1i) - dot((n1j - n1i), e) * e);
      const d3 MTB = B3 * cross(n1j, n1i) - 0.5 * B4 * (cross(n2j, n2i) + cross(n3j, n3i));
      Mij = -0.5 * B2 * cross(e, n1i) + MTB;
      Mji = 0.5 * B2 * cross(e, n1j) - MTB;
      const double fnb = dot(F, nij);
      const d3 fsb = F - fnb * nij;
      const double tt = dot(MTB, nij);
      const d3 tb = MTB - tt * nij;
      const double A = Rb * Rb * M_PI;
      const double I = A * Rb * Rb / 4.;
      const double J2 = 2 * I;
      st[4] = -fnb / A + len(tb) / I * Rb;
      st[5] = len(fsb) / A + std::fabs(tt) / J2 * Rb;
      if (ten > 0. && st[4] > ten) ok = 0;
      else if (coh > 0. && st[5] > coh - fmu * st[4]) ok = 0;
    }
    bonded[k] = ok;
    add3(force, i, F, false);
    add3(torque, i, Mij + cross(rbi - ri, F), false);
    add3(force, j, -F, false);
    add3(torque, j, Mji + cross(rbj - rj, -F), false);
  }
}

// ---------------------------------------------------------------------------
// Integration: particleVelocityAngularVelocityIntegrationKernel (particleIntegrationKernel.cu:3-24).
ORA_API void ora_kick(int n, double* vel, double* angvel, const double* force, const double* torque, const double* invmass,
              const double* quat, const double* invI, const double* g, double h) {
  const d3 grav = mk(g[0], g[1], g[2]);
  for (int i = 0; i < n; ++i) {
    const double im = invmass[i];
    if (is_zero(im)) continue;
    d3 v = ld3(vel, i);
    v += (ld3(force, i) * im + grav) * h;
    st3(vel, i, v);
    const double* I = invI + 6 * i;
    const sm Iw = rotate_inv_inertia(ldq(quat, i), sm{I[0], I[1], I[2], I[3], I[4], I[5]});
    d3 w = ld3(angvel, i);
    w += mul(Iw, ld3(torque, i)) * h;
    st3(angvel, i, w);
  }
}

// particlePositionOrientationIntegrationKernel (particleIntegrationKernel.cu:26-40).
ORA_API void ora_drift(int n, double* pos, double* quat, const double* vel, const double* angvel, double dt) {
  for (int i = 0; i < n; ++i) {
    d3 p = ld3(pos, i);
    p += dt * ld3(vel, i);
    st3(pos, i, p);
    qt q = integrate_q(ldq(quat, i), ld3(angvel, i), dt);
    quat[4 * i] = q.q0; quat[4 * i + 1] = q.q1; quat[4 * i + 2] = q.q2; quat[4 * i + 3] = q.q3;
  }
}

// ---------------------------------------------------------------------------
// Mass properties of a level-set body by smoothed Heaviside integration over
// the SDF grid (LSSolver.h:66-135). out: mass, centroid[3], inertia[6] (local,
// about the centroid), inverse inertia[6].
ORA_API void ora_mass_props(const double* sdf, int nx, int ny, int nz, const double* origin, double h, double density,
                    double* out) {
  auto H = [](double phi, double eps) -> double {
    if (eps <= 0.0) return (phi > 0.0) ? 0.0 : 1.0;
    if (phi < -eps) return 1.0;
    if (phi > eps) return 0.0;
    const double x = -phi / eps;
    return 0.5 * (1.0 + x + std::sin(M_PI * x) / M_PI);
  };
  double mass = 0.;
  const double mg = density * h * h * h;
  for (int x = 0; x < nx; x++)
    for (int y = 0; y < ny; y++)
      for (int z = 0; z < nz; z++) mass += H(sdf[lin3(x, y, z, nx, ny)] / h, 1.5);
  mass *= mg;
  d3 c = mk(0., 0., 0.);
  sm I{0, 0, 0, 0, 0, 0};
  if (mass > 0.) {
    for (int x = 0; x < nx; x++)
      for (int y = 0; y < ny; y++)
        for (int z = 0; z < nz; z++) {
          const double Hv = H(sdf[lin3(x, y, z, nx, ny)] / h, 1.5);
          c.x += Hv * (origin[0] + double(x) * h);
          c.y += Hv * (origin[1] + double(y) * h);
          c.z += Hv * (origin[2] + double(z) * h);
        }
    c *= mg / mass;
    for (int x = 0; x < nx; x++)
      for (int y = 0; y < ny; y++)
        for (int z = 0; z < nz; z++) {
          const double Hv = H(sdf[lin3(x, y, z, nx, ny)] / h, 1.5);
          const d3 r = mk(origin[0], origin[1], origin[2]) + h * mk(double(x), double(y), double(z)) - c;
          I.xx += Hv * (r.y * r.y + r.z * r.z) * mg;
          I.yy += Hv * (r.x * r.x + r.z * r.z) * mg;
          I.zz += Hv * (r.y * r.y + r.x * r.x) * mg;
          I.xy -= Hv * r.x * r.y * mg;
          I.xz -= Hv * r.x * r.z * mg;
          I.yz -= Hv * r.y * r.z * mg;
        }
  }
  const sm inv = mass > 0. ? inverse(I) : sm{0, 0, 0, 0, 0, 0};
  out[0] = mass;
  out[1] = c.x; out[2] = c.y; out[3] = c.z;
  out[4] = I.xx; out[5] = I.yy; out[6] = I.zz; out[7] = I.xy; out[8] = I.xz; out[9] = I.yz;
  out[10] = inv.xx; out[11] = inv.yy; out[12] = inv.zz; out[13] = inv.xy; out[14] = inv.xz; out[15] = inv.yz;
}

// ---------------------------------------------------------------------------
// Level-set grid of a closed triangle mesh: LevelSetObject::Base::buildGrid
// (FunDEM/kernel/helper/LevelSetObjectGenerator.h:122-224) over
// TriangleMeshParticle::evaluateImplicitFunctionValueAndGradient (:888-914).
// Closest point on a triangle by the Voronoi-region tests of Ericson,
// "Real-Time Collision Detection" (2005) 5.1.5 (closestPointOnTriangle,
// :454-500); the nearest triangle by a scan in index order (the reference's BVH
// finds the same distance); inside by the solid-angle sum of Van Oosterom and
// Strackee (1983) in triangle order (:758-802).
static d3 closest_on_triangle(d3 p, d3 a, d3 b, d3 c) {
  const d3 ab = b - a, ac = c - a, ap = p - a;
  const double d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) return a;
  const d3 bp = p - b;
  const double d3v = dot(ab, bp), d4 = dot(ac, bp);
  if (d3v >= 0.0 && d4 <= d3v) return b;
  const double vc = d1 * d4 - d3v * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3v <= 0.0) return a + (d1 / (d1 - d3v)) * ab;
  const d3 cp = p - c;
  const double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return c;
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return a + (d2 / (d2 - d6)) * ac;
  const double va = d3v * d6 - d5 * d4;
  if (va <= 0.0 && (d4 - d3v) >= 0.0 && (d5 - d6) >= 0.0) return b + ((d4 - d3v) / ((d4 - d3v) + (d5 - d6))) * (c - b);
  const double denom = 1.0 / (va + vb + vc);
  const double v = vb * denom, w = vc * denom;
  return a + ab * v + ac * w;
}

static double solid_angle(d3 p, d3 a, d3 b, d3 c) {
  const d3 r0 = a - p, r1 = b - p, r2 = c - p;
  const double l0 = len(r0), l1 = len(r1), l2 = len(r2);
  if (l0 < 1e-30 || l1 < 1e-30 || l2 < 1e-30) return 0.0;
  const double num = dot(r0, cross(r1, r2));
  const double den = l0 * l1 * l2 + dot(r0, r1) * l2 + dot(r1, r2) * l0 + dot(r2, r0) * l1;
  return 2.0 * std::atan2(num, den);
}

ORA_API void ora_mesh_grid(const double* verts, const int* tris, int nt, const double* origin, int nx, int ny, int nz,
                           double h, int positive_inside, double* out) {
  const long long n = (long long)nx * ny * nz;
#pragma omp parallel for schedule(dynamic, 64)
  for (long long i = 0; i < n; ++i) {
    const int ix = (int)(i % nx), iy = (int)((i / nx) % ny), iz = (int)(i / ((long long)nx * ny));
    const d3 p = mk(origin[0] + double(ix) * h, origin[1] + double(iy) * h, origin[2] + double(iz) * h);
    double best = 1.7976931348623157e308, sum = 0.0;
    d3 cp = mk(0., 0., 0.);
    for (int t = 0; t < nt; ++t) {
      const d3 a = ld3(verts, tris[3 * t]), b = ld3(verts, tris[3 * t + 1]), c = ld3(verts, tris[3 * t + 2]);
      const d3 x = closest_on_triangle(p, a, b, c);
      const double dd = len2(p - x);
      if (dd < best) { best = dd; cp = x; }
      sum += solid_angle(p, a, b, c);
    }
    const double d = len(p - cp);
    const bool inside = std::fabs(sum / (4.0 * 3.14159265358979323846)) > 0.5;
    double value = inside ? -d : d;
    d3 g = mk(0., 0., 0.);
    if (d > 1e-30) {
      const d3 u = (p - cp) / d;
      g = inside ? -u : u;
    }
    if (positive_inside) { value = -value; g = -g; }
    const double gn = len(g);
    out[i] = gn > 1e-12 ? value / gn : (value <= 0.0 ? -1.0 : 1.0) * 0.5 * h;
  }
}

// Host-side helpers used by the orchestration layer.
ORA_API void ora_rotate(int n, const double* quat, const double* v, double* out) {
  for (int i = 0; i < n; ++i) st3(out, i, rotate(ldq(quat, i), ld3(v, i)));
}
ORA_API void ora_normalize_quat(int n, double* quat) {
  for (int i = 0; i < n; ++i) {
    qt q = normalize(ldq(quat, i));
    quat[4 * i] = q.q0; quat[4 * i + 1] = q.q1; quat[4 * i + 2] = q.q2; quat[4 * i + 3] = q.q3;
  }
}
ORA_API int ora_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
ORA_API void ora_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}


