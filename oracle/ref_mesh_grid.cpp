// Golden-vector driver for the level-set grid builder — TEST INFRASTRUCTURE ONLY.
//
// Compiled by oracle/build_ref.sh against the reference's own host header
// FunDEM/kernel/helper/LevelSetObjectGenerator.h (read where it lies in the
// reference tree, never copied) into oracle/_ref/mesh_grid_ref. It runs the
// reference's generator classes on the host and writes their output, so that
// tests/golden/make_mesh_grid_golden.py can store it as fixtures. Nothing of
// the product links or runs it.
//
// Usage:
//   mesh_grid_ref super RX RY RZ EE EN LEVEL SPACING PAD OUT
//       LevelSetObject::Superellipsoid(RX, RY, RZ, EE, EN, LEVEL): its mesh,
//       its own buildGrid(SPACING, PAD) (analytic F / |grad F|), and the grid
//       of a TriangleMeshParticle built from that mesh (mesh distance with the
//       solid-angle sign).
//   mesh_grid_ref mesh IN SPACING PAD OUT
//       TriangleMeshParticle from the mesh in IN (text: nv nt, then nv
//       vertex rows, then nt index rows) and its buildGrid(SPACING, PAD).
//
// OUT (text, %.17g): sections "mesh nv nt" + rows, "grid nx ny nz ox oy oz h"
// + values in the reference's linear order ix + nx (iy + ny iz).
#include "helper/LevelSetObjectGenerator.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

static void write_mesh(FILE* f, const std::vector<double3>& v, const std::vector<int3>& t) {
  std::fprintf(f, "mesh %zu %zu\n", v.size(), t.size());
  for (const auto& p : v) std::fprintf(f, "%.17g %.17g %.17g\n", p.x, p.y, p.z);
  for (const auto& q : t) std::fprintf(f, "%d %d %d\n", q.x, q.y, q.z);
}

static void write_grid(FILE* f, const char* name, const LevelSetObject::GridInfo& g) {
  std::fprintf(f, "grid %s %d %d %d %.17g %.17g %.17g %.17g\n", name, g.gridNodeSize.x, g.gridNodeSize.y,
               g.gridNodeSize.z, g.gridOrigin.x, g.gridOrigin.y, g.gridOrigin.z, g.gridNodeSpacing);
  for (double v : g.gridNodeSignedDistance) std::fprintf(f, "%.17g\n", v);
}

int main(int argc, char** argv) {
  if (argc >= 11 && std::strcmp(argv[1], "super") == 0) {
    const double rx = std::atof(argv[2]), ry = std::atof(argv[3]), rz = std::atof(argv[4]);
    const double ee = std::atof(argv[5]), en = std::atof(argv[6]);
    const int level = std::atoi(argv[7]);
    const double h = std::atof(argv[8]);
    const int pad = std::atoi(argv[9]);
    LevelSetObject::Superellipsoid s(rx, ry, rz, ee, en, level);
    s.buildGrid(h, pad);
    LevelSetObject::TriangleMeshParticle m(s.vertexPosition(), s.triangleVertexIndex());
    m.buildGrid(h, pad);
    FILE* f = std::fopen(argv[10], "w");
    if (!f) return 2;
    write_mesh(f, s.vertexPosition(), s.triangleVertexIndex());
    write_grid(f, "analytic", s.gridInfo());
    write_grid(f, "mesh", m.gridInfo());
    std::fclose(f);
    return 0;
  }
  if (argc >= 6 && std::strcmp(argv[1], "mesh") == 0) {
    FILE* in = std::fopen(argv[2], "r");
    if (!in) return 2;
    size_t nv = 0, nt = 0;
    if (std::fscanf(in, "%zu %zu", &nv, &nt) != 2) return 3;
    std::vector<double3> v(nv);
    std::vector<int3> t(nt);
    for (auto& p : v)
      if (std::fscanf(in, "%lf %lf %lf", &p.x, &p.y, &p.z) != 3) return 3;
    for (auto& q : t)
      if (std::fscanf(in, "%d %d %d", &q.x, &q.y, &q.z) != 3) return 3;
    std::fclose(in);
    LevelSetObject::TriangleMeshParticle m(v, t);
    m.buildGrid(std::atof(argv[3]), std::atoi(argv[4]));
    FILE* f = std::fopen(argv[5], "w");
    if (!f) return 2;
    write_mesh(f, v, t);
    write_grid(f, "mesh", m.gridInfo());
    std::fclose(f);
    return 0;
  }
  std::fprintf(stderr, "usage: mesh_grid_ref super RX RY RZ EE EN LEVEL SPACING PAD OUT | mesh IN SPACING PAD OUT\n");
  return 1;
}
