// Frame output: the VTU files of the reference's LSSolver::output (FunDEM/kernel/LSSolver.h:637-665),
// produced on the GPU.
//
// The reference downloads every array, converts it element by element on one
// host core and base64-encodes it there (LSParticle::outputVTU :311-506,
// outputParticleVTU :508-654, SolidInteraction::outputVTU :154-317,
// VBondedInteraction::outputVTU :262-448); the surface-node mesh alone is
// 12 bytes per node and array. Here every array streams through the GPU in
// chunks: a packing kernel computes the chunk's values from the device state
// (node world positions and velocities as the reference's host loop computes
// them: p + rotate(q, local), v + w x (p_node - p), then cast to float), a
// second kernel base64-encodes the chunk (the reference's inline-binary form:
// an 8-byte little-endian byte count, then the data, one continuous base64
// stream, the partial 3-byte group carried to the next chunk), and the encoded
// chunk is copied to one of two pinned host buffers, so that the file write of
// one chunk overlaps the packing and copy of the next. Small host-side arrays
// (contacts, bonds, walls) take the same encoder after a host-to-device copy.
// The XML around the arrays is the reference's, so files written here and by
// the reference have the same layout, array names and types.
//
// Compiled with --fmad=false: products and sums round as the reference's host
// arithmetic does, so FP64 node positions agree before the cast to float.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "kernels.h"

namespace lsdem {
namespace {

constexpr size_t kChunkBytes = (size_t)32 << 20;  // raw bytes per chunk (multiple of 12 and 16)
constexpr size_t kEncBytes = (kChunkBytes + 16) / 3 * 4 + 16;

__device__ __forceinline__ char b64c(unsigned v) {
  return v < 26 ? (char)('A' + v) : v < 52 ? (char)('a' + v - 26) : v < 62 ? (char)('0' + v - 52) : v == 62 ? '+' : '/';
}

// One base64 group (3 stream bytes -> 4 characters) per thread. The stream is
// carry[0 .. cn) followed by data[0 .. nb); groups past the stream's end are
// padded with '=' (only in the last chunk). The bytes after the last whole group
// of a chunk that is not the last go to carry_out.
__global__ void k_b64(const uint8_t* __restrict__ carry, int cn, const uint8_t* __restrict__ data, size_t nb,
                      size_t groups, bool last, char* __restrict__ out, uint8_t* __restrict__ carry_out) {
  const size_t len = (size_t)cn + nb;
  const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g == 0 && !last) {
    for (size_t i = 3 * groups; i < len; ++i) carry_out[i - 3 * groups] = i < (size_t)cn ? carry[i] : data[i - cn];
  }
  if (g >= groups) return;
  unsigned b[3];
  for (int k = 0; k < 3; ++k) {
    const size_t i = 3 * g + k;
    b[k] = i < (size_t)cn ? carry[i] : (i < len ? data[i - cn] : 0u);
  }
  const unsigned v = (b[0] << 16) | (b[1] << 8) | b[2];
  out[4 * g] = b64c((v >> 18) & 63);
  out[4 * g + 1] = b64c((v >> 12) & 63);
  out[4 * g + 2] = 3 * g + 1 < len ? b64c((v >> 6) & 63) : '=';
  out[4 * g + 3] = 3 * g + 2 < len ? b64c(v & 63) : '=';
}

LD int owner_of(const long long* __restrict__ base, int n, long long e) {
  int lo = 0, hi = n - 1;  // last p with base[p] <= e
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (base[mid] <= e) lo = mid; else hi = mid - 1;
  }
  return lo;
}

struct NodeSrc {
  const double3* pos;
  const double3* vel;
  const double3* angvel;
  const Quat* quat;
  const long long* base;    // n + 1: first node of each particle (caller order)
  const int* shape;
  const double* scale;
  const double3* tnode;     // template nodes, caller order
  const long long* toff;    // first template node of each shape
  int n;
};

// field 0: node world position, 1: node velocity, 2: particle id
__global__ void k_pack_nodes(NodeSrc s, long long e0, long long e1, int field, void* __restrict__ out) {
  const long long e = e0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= e1) return;
  const int p = owner_of(s.base, s.n, e);
  const long long k = e - e0;
  if (field == 2) { reinterpret_cast<int32_t*>(out)[k] = p; return; }
  const double3 local = s.tnode[s.toff[s.shape[p]] + (e - s.base[p])] * s.scale[p];
  const double3 x = s.pos[p];
  const double3 pw = x + rotate(s.quat[p], local);
  float* o = reinterpret_cast<float*>(out) + 3 * k;
  if (field == 0) {
    o[0] = (float)pw.x; o[1] = (float)pw.y; o[2] = (float)pw.z;
  } else {
    const double3 vw = s.vel[p] + cross(s.angvel[p], pw - x);
    o[0] = (float)vw.x; o[1] = (float)vw.y; o[2] = (float)vw.z;
  }
}

struct TriSrc {
  const long long* tbase;   // n + 1: first output triangle of each particle
  const long long* base;    // n + 1: first node of each particle
  const int* tset;          // triangle set of each particle (-1: none)
  const long long* soff;    // first triangle of each set in `tri`
  const int* tri;           // 3 ints per triangle, local node indices
  int n;
};

// field 0: connectivity (3 per triangle), 1: offsets 3 (i + 1), 2: types (5 = triangle)
__global__ void k_pack_tris(TriSrc s, long long e0, long long e1, int field, void* __restrict__ out) {
  const long long e = e0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= e1) return;
  const long long k = e - e0;
  if (field == 1) { reinterpret_cast<int32_t*>(out)[k] = (int32_t)(3 * (e + 1)); return; }
  if (field == 2) { reinterpret_cast<uint8_t*>(out)[k] = 5; return; }
  const int p = owner_of(s.tbase, s.n, e);
  const int* t = s.tri + 3 * (s.soff[s.tset[p]] + (e - s.tbase[p]));
  const int b = (int)s.base[p];
  int32_t* o = reinterpret_cast<int32_t*>(out) + 3 * k;
  o[0] = t[0] + b; o[1] = t[1] + b; o[2] = t[2] + b;
}

// field 0: position, 1: velocity, 2: angular velocity (float3), 3: orientation (float4), 4: radius
__global__ void k_pack_particles(NodeSrc s, const double* __restrict__ radius, long long e0, long long e1, int field,
                                 void* __restrict__ out) {
  const long long e = e0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= e1) return;
  const long long k = e - e0;
  float* o = reinterpret_cast<float*>(out);
  if (field == 3) {
    const Quat q = s.quat[e];
    o[4 * k] = (float)q.q0; o[4 * k + 1] = (float)q.q1; o[4 * k + 2] = (float)q.q2; o[4 * k + 3] = (float)q.q3;
  } else if (field == 4) {
    o[k] = (float)radius[e];
  } else {
    const double3 v = field == 0 ? s.pos[e] : field == 1 ? s.vel[e] : s.angvel[e];
    o[3 * k] = (float)v.x; o[3 * k + 1] = (float)v.y; o[3 * k + 2] = (float)v.z;
  }
}

void ck(cudaError_t e) {
  if (e != cudaSuccess) throw VtuError{cudaGetErrorString(e)};
}

template <class T>
T* dalloc(size_t n) {
  T* p = nullptr;
  ck(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
  return p;
}

}  // namespace

// Buffers and uploaded layout of one solver's writer (kept between frames).
struct VtuCtx {
  cudaStream_t st = nullptr;
  uint8_t* d_elem = nullptr;
  char* d_enc[2] = {nullptr, nullptr};
  uint8_t* d_carry[2] = {nullptr, nullptr};
  char* h_pin[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  // layout (re-uploaded when it changes)
  long long layout = -1;
  long long* d_base = nullptr;
  int* d_shape = nullptr;
  double* d_scale = nullptr;
  double3* d_tnode = nullptr;
  long long* d_toff = nullptr;
  long long* d_tbase = nullptr;
  int* d_tset = nullptr;
  long long* d_soff = nullptr;
  int* d_tri = nullptr;
  long long n_tris = 0;
  ~VtuCtx() {
    for (void* p : {(void*)d_elem, (void*)d_enc[0], (void*)d_enc[1], (void*)d_carry[0], (void*)d_carry[1],
                    (void*)d_base, (void*)d_shape, (void*)d_scale, (void*)d_tnode, (void*)d_toff, (void*)d_tbase,
                    (void*)d_tset, (void*)d_soff, (void*)d_tri})
      if (p) cudaFree(p);
    for (char* p : h_pin)
      if (p) cudaFreeHost(p);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
  }
};

void vtu_free(VtuCtx* c) { delete c; }

namespace {

// Writes one binary DataArray payload: base64 of [u64 byte count][nelem * esize bytes],
// the bytes of elements [e0, e1) produced into d_elem by gen(e0, e1).
template <class Gen>
void emit(VtuCtx& c, FILE* f, long long nelem, size_t esize, Gen&& gen) {
  const size_t total = (size_t)nelem * esize;
  uint8_t hdr[8];
  for (int k = 0; k < 8; ++k) hdr[k] = (uint8_t)(((uint64_t)total >> (8 * k)) & 0xff);
  ck(cudaMemcpyAsync(c.d_carry[0], hdr, 8, cudaMemcpyHostToDevice, c.st));
  int cn = 8, cur = 0, buf = 0;
  size_t pending = 0;  // bytes of h_pin[buf ^ 1] still to write
  const long long per = (long long)(kChunkBytes / esize);
  long long e0 = 0;
  do {
    const long long e1 = std::min(nelem, e0 + per);
    if (e1 > e0) gen(e0, e1);
    const size_t nb = (size_t)(e1 - e0) * esize;
    const bool last = e1 == nelem;
    const size_t len = (size_t)cn + nb;
    const size_t groups = last ? (len + 2) / 3 : len / 3;
    if (groups > 0) {
      const unsigned blocks = (unsigned)((groups + 255) / 256);
      k_b64<<<blocks, 256, 0, c.st>>>(c.d_carry[cur], cn, c.d_elem, nb, groups, last, c.d_enc[buf], c.d_carry[cur ^ 1]);
      ck(cudaGetLastError());
      ck(cudaMemcpyAsync(c.h_pin[buf], c.d_enc[buf], 4 * groups, cudaMemcpyDeviceToHost, c.st));
    } else if (!last) {
      ck(cudaMemcpyAsync(c.d_carry[cur ^ 1], c.d_carry[cur], (size_t)cn, cudaMemcpyDeviceToDevice, c.st));
    }
    ck(cudaEventRecord(c.ev[buf], c.st));
    if (pending) {  // the previous chunk, while this one is packed, encoded and copied
      ck(cudaEventSynchronize(c.ev[buf ^ 1]));
      if (std::fwrite(c.h_pin[buf ^ 1], 1, pending, f) != pending) throw VtuError{"write error"};
    }
    pending = 4 * groups;
    cn = last ? 0 : (int)(len - 3 * groups);
    cur ^= 1;
    buf ^= 1;
    e0 = e1;
  } while (e0 < nelem);
  ck(cudaEventSynchronize(c.ev[buf ^ 1]));
  if (pending && std::fwrite(c.h_pin[buf ^ 1], 1, pending, f) != pending) throw VtuError{"write error"};
}

// Host array through the encoder.
template <class T>
void emit_host(VtuCtx& c, FILE* f, const std::vector<T>& v, int ncomp) {
  const long long n = (long long)(v.size() / ncomp);
  const size_t es = sizeof(T) * ncomp;
  emit(c, f, n, es, [&](long long e0, long long e1) {
    ck(cudaMemcpyAsync(c.d_elem, v.data() + (size_t)e0 * ncomp, (size_t)(e1 - e0) * es, cudaMemcpyHostToDevice, c.st));
  });
}

struct File {
  FILE* f = nullptr;
  explicit File(const std::string& path) : f(std::fopen(path.c_str(), "wb")) {
    if (!f) throw VtuError{"Cannot open for writing: " + path};
  }
  ~File() { if (f) std::fclose(f); }
  void put(const std::string& s) {
    if (std::fwrite(s.data(), 1, s.size(), f) != s.size()) throw VtuError{"write error"};
  }
};

std::string head(double time, unsigned long long step) {
  std::ostringstream o;
  o << "<?xml version=\"1.0\"?>\n"
    << "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" "
       "byte_order=\"LittleEndian\" header_type=\"UInt64\">\n"
    << "<UnstructuredGrid>\n"
    << "<FieldData>\n"
    << "<DataArray type=\"Float32\" Name=\"TIME\" NumberOfTuples=\"1\" format=\"ascii\">" << static_cast<float>(time)
    << "</DataArray>\n"
    << "<DataArray type=\"Int32\" Name=\"STEP\" NumberOfTuples=\"1\" format=\"ascii\">" << static_cast<int32_t>(step)
    << "</DataArray>\n"
    << "</FieldData>\n";
  return o.str();
}

const char* kTail = "</PointData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n";

std::string name(const std::string& dir, const char* stem, unsigned long long frame) {
  std::ostringstream o;
  o << dir << "/" << stem << "_";
  o.width(4);
  o.fill('0');
  o << frame << ".vtu";
  return o.str();
}

void mkdir(const std::string& d) {
  std::error_code ec;
  std::filesystem::create_directories(d, ec);
}

void upload_layout(VtuCtx& c, const VtuInput& in) {
  if (c.layout == in.layout) return;
  for (void** p : {(void**)&c.d_base, (void**)&c.d_shape, (void**)&c.d_scale, (void**)&c.d_tnode, (void**)&c.d_toff,
                   (void**)&c.d_tbase, (void**)&c.d_tset, (void**)&c.d_soff, (void**)&c.d_tri})
    if (*p) { cudaFree(*p); *p = nullptr; }
  const int n = in.n;
  c.d_base = dalloc<long long>(n + 1);
  c.d_shape = dalloc<int>(n);
  c.d_scale = dalloc<double>(n);
  ck(cudaMemcpy(c.d_base, in.node_base, sizeof(long long) * (n + 1), cudaMemcpyHostToDevice));
  ck(cudaMemcpy(c.d_shape, in.shape, sizeof(int) * n, cudaMemcpyHostToDevice));
  ck(cudaMemcpy(c.d_scale, in.scale, sizeof(double) * n, cudaMemcpyHostToDevice));
  std::vector<long long> toff(in.tnodes.size() + 1, 0);
  for (size_t k = 0; k < in.tnodes.size(); ++k) toff[k + 1] = toff[k] + (long long)(in.tnodes[k]->size() / 3);
  std::vector<double> tn((size_t)toff.back() * 3);
  for (size_t k = 0; k < in.tnodes.size(); ++k)
    std::copy(in.tnodes[k]->begin(), in.tnodes[k]->end(), tn.begin() + 3 * toff[k]);
  c.d_tnode = dalloc<double3>((size_t)toff.back());
  c.d_toff = dalloc<long long>(toff.size());
  ck(cudaMemcpy(c.d_tnode, tn.data(), tn.size() * sizeof(double), cudaMemcpyHostToDevice));
  ck(cudaMemcpy(c.d_toff, toff.data(), toff.size() * sizeof(long long), cudaMemcpyHostToDevice));
  // triangles: per particle its set's count, prefix over particles
  std::vector<long long> soff(in.tri_sets.size() + 1, 0);
  for (size_t k = 0; k < in.tri_sets.size(); ++k) soff[k + 1] = soff[k] + (long long)(in.tri_sets[k]->size() / 3);
  std::vector<int> tri((size_t)soff.back() * 3);
  for (size_t k = 0; k < in.tri_sets.size(); ++k)
    std::copy(in.tri_sets[k]->begin(), in.tri_sets[k]->end(), tri.begin() + 3 * soff[k]);
  std::vector<long long> tbase(n + 1, 0);
  std::vector<int> tset(n, 0);
  for (int p = 0; p < n; ++p) {
    const int k = in.tri_set ? in.tri_set[p] : -1;
    tset[p] = k < 0 ? 0 : k;
    tbase[p + 1] = tbase[p] + (k < 0 ? 0 : soff[k + 1] - soff[k]);
  }
  c.n_tris = tbase[n];
  c.d_tbase = dalloc<long long>(n + 1);
  c.d_tset = dalloc<int>(n);
  c.d_soff = dalloc<long long>(soff.size());
  c.d_tri = dalloc<int>(tri.size());
  ck(cudaMemcpy(c.d_tbase, tbase.data(), tbase.size() * sizeof(long long), cudaMemcpyHostToDevice));
  ck(cudaMemcpy(c.d_tset, tset.data(), tset.size() * sizeof(int), cudaMemcpyHostToDevice));
  ck(cudaMemcpy(c.d_soff, soff.data(), soff.size() * sizeof(long long), cudaMemcpyHostToDevice));
  if (!tri.empty()) ck(cudaMemcpy(c.d_tri, tri.data(), tri.size() * sizeof(int), cudaMemcpyHostToDevice));
  c.layout = in.layout;
}

inline unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256); }

std::string arr(const char* type, const char* nm, int ncomp) {
  std::ostringstream o;
  o << "<DataArray type=\"" << type << "\" Name=\"" << nm << "\" ";
  if (ncomp > 0) o << "NumberOfComponents=\"" << ncomp << "\" ";
  o << "format=\"binary\">\n";
  return o.str();
}
const char* kEnd = "\n</DataArray>\n";

// Mesh file of a body set (LSParticle::outputVTU, LSParticle.h:311-506): nodes in world
// coordinates, triangles of the connectivity given at insertion, velocity and body id per node.
void write_mesh_particles(VtuCtx& c, const VtuInput& in, const std::string& dir) {
  const long long N = in.node_base[in.n], M = c.n_tris;
  mkdir(dir);
  File f(name(dir, "LSObjectMesh", in.frame));
  std::ostringstream o;
  o << head(in.time, in.step) << "<Piece NumberOfPoints=\"" << N << "\" NumberOfCells=\"" << M << "\">\n"
    << "<Points>\n<DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"binary\">\n";
  f.put(o.str());
  NodeSrc s{in.pos, in.vel, in.angvel, in.quat, c.d_base, c.d_shape, c.d_scale, c.d_tnode, c.d_toff, in.n};
  auto nodes = [&](int field) {
    return [&, field](long long e0, long long e1) {
      k_pack_nodes<<<blocks_for(e1 - e0), 256, 0, c.st>>>(s, e0, e1, field, c.d_elem);
      ck(cudaGetLastError());
    };
  };
  emit(c, f.f, N, 12, nodes(0));
  f.put(std::string(kEnd) + "</Points>\n<Cells>\n<DataArray type=\"Int32\" Name=\"connectivity\" format=\"binary\">\n");
  TriSrc t{c.d_tbase, c.d_base, c.d_tset, c.d_soff, c.d_tri, in.n};
  auto tris = [&](int field) {
    return [&, field](long long e0, long long e1) {
      k_pack_tris<<<blocks_for(e1 - e0), 256, 0, c.st>>>(t, e0, e1, field, c.d_elem);
      ck(cudaGetLastError());
    };
  };
  emit(c, f.f, M, 12, tris(0));
  f.put(std::string(kEnd) + "<DataArray type=\"Int32\" Name=\"offsets\" format=\"binary\">\n");
  emit(c, f.f, M, 4, tris(1));
  f.put(std::string(kEnd) + "<DataArray type=\"UInt8\" Name=\"types\" format=\"binary\">\n");
  emit(c, f.f, M, 1, tris(2));
  f.put(std::string(kEnd) + "</Cells>\n<PointData Vectors=\"velocity\">\n" + arr("Int32", "particleID", 0));
  emit(c, f.f, N, 4, nodes(2));
  f.put(std::string(kEnd) + arr("Float32", "velocity", 3));
  emit(c, f.f, N, 12, nodes(1));
  f.put(std::string(kEnd) + kTail);
}

// Particle file (LSParticle::outputParticleVTU, LSParticle.h:508-654).
void write_particles(VtuCtx& c, const VtuInput& in, const std::string& dir) {
  mkdir(dir);
  File f(name(dir, "Particle", in.frame));
  std::ostringstream o;
  o << head(in.time, in.step) << "<Piece NumberOfPoints=\"" << in.n << "\" NumberOfCells=\"0\">\n"
    << "<Points>\n<DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"binary\">\n";
  f.put(o.str());
  NodeSrc s{in.pos, in.vel, in.angvel, in.quat, c.d_base, c.d_shape, c.d_scale, c.d_tnode, c.d_toff, in.n};
  auto gen = [&](int field) {
    return [&, field](long long e0, long long e1) {
      k_pack_particles<<<blocks_for(e1 - e0), 256, 0, c.st>>>(s, in.radius, e0, e1, field, c.d_elem);
      ck(cudaGetLastError());
    };
  };
  emit(c, f.f, in.n, 12, gen(0));
  f.put(std::string(kEnd) + "</Points>\n<Cells/>\n<PointData Vectors=\"velocity\">\n" + arr("Float32", "velocity", 3));
  emit(c, f.f, in.n, 12, gen(1));
  f.put(std::string(kEnd) + arr("Float32", "angularVelocity", 3));
  emit(c, f.f, in.n, 12, gen(2));
  f.put(std::string(kEnd) + arr("Float32", "orientation", 4));
  emit(c, f.f, in.n, 16, gen(3));
  f.put(std::string(kEnd) + "<DataArray type=\"Float32\" Name=\"radius\" NumberOfComponents=\"1\" format=\"binary\">\n");
  emit(c, f.f, in.n, 4, gen(4));
  f.put(std::string(kEnd) + kTail);
}

// Contact file (SolidInteraction::outputVTU, SolidInteraction.h:154-317): one vertex cell per contact.
void write_contacts(VtuCtx& c, const VtuInput& in, const VtuContacts& k, const std::string& dir) {
  mkdir(dir);
  File f(name(dir, "LSInteraction", in.frame));
  const size_t N = k.en_n.size();
  std::vector<float> pt(3 * N), nm(3 * N), sd(3 * N), en(N), es(N);
  std::vector<int32_t> conn(N), offs(N);
  std::vector<uint8_t> types(N, 1);
  for (size_t i = 0; i < N; ++i) {
    const double3 s = d3(k.spring[3 * i], k.spring[3 * i + 1], k.spring[3 * i + 2]);
    // normalize (myVec.h:121-137, host branch): zero below 1e-20, else times 1 / sqrt
    const double l2 = s.x * s.x + s.y * s.y + s.z * s.z;
    double3 u = d3(0., 0., 0.);
    if (!is_zero(l2)) {
      const double inv = 1.0 / std::sqrt(l2);
      u = d3(s.x * inv, s.y * inv, s.z * inv);
    }
    for (int a = 0; a < 3; ++a) {
      pt[3 * i + a] = (float)k.point[3 * i + a];
      nm[3 * i + a] = (float)k.normal[3 * i + a];
    }
    sd[3 * i] = (float)u.x; sd[3 * i + 1] = (float)u.y; sd[3 * i + 2] = (float)u.z;
    en[i] = (float)k.en_n[i];
    es[i] = (float)k.en_s[i];
    conn[i] = (int32_t)i;
    offs[i] = (int32_t)(i + 1);
  }
  std::ostringstream o;
  o << head(in.time, in.step) << "<Piece NumberOfPoints=\"" << N << "\" NumberOfCells=\"" << N << "\">\n"
    << "<Points>\n<DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"binary\">\n";
  f.put(o.str());
  emit_host(c, f.f, pt, 3);
  f.put(std::string(kEnd) + "</Points>\n<Cells>\n<DataArray type=\"Int32\" Name=\"connectivity\" format=\"binary\">\n");
  emit_host(c, f.f, conn, 1);
  f.put(std::string(kEnd) + "<DataArray type=\"Int32\" Name=\"offsets\" format=\"binary\">\n");
  emit_host(c, f.f, offs, 1);
  f.put(std::string(kEnd) + "<DataArray type=\"UInt8\" Name=\"types\" format=\"binary\">\n");
  emit_host(c, f.f, types, 1);
  f.put(std::string(kEnd) + "</Cells>\n<PointData>\n" + arr("Float32", "contactNormal", 3));
  emit_host(c, f.f, nm, 3);
  f.put(std::string(kEnd) + arr("Float32", "slidingDirection", 3));
  emit_host(c, f.f, sd, 3);
  f.put(std::string(kEnd) + "<DataArray type=\"Float32\" Name=\"normalElasticEnergy\" format=\"binary\">\n");
  emit_host(c, f.f, en, 1);
  f.put(std::string(kEnd) + "<DataArray type=\"Float32\" Name=\"slidingElasticEnergy\" format=\"binary\">\n");
  emit_host(c, f.f, es, 1);
  f.put(std::string(kEnd) + kTail);
}

// Bond file (VBondedInteraction::outputVTU, VBondedInteraction.h:262-448).
void write_bonds(VtuCtx& c, const VtuInput& in, const std::string& dir) {
  const size_t N = in.bond_bonded.size();
  mkdir(dir);
  File f(name(dir, "VBondedInteraction", in.frame));
  std::vector<float> pt(3 * N), un(N), us(N), ub(N), ut(N), sn(N), ss(N);
  std::vector<int32_t> conn(N), offs(N), mid(N), sid(N), act(N);
  std::vector<uint8_t> types(N, 1);
  for (size_t i = 0; i < N; ++i) {
    const double* st = &in.bond_state[9 * i];
    pt[3 * i] = (float)st[6]; pt[3 * i + 1] = (float)st[7]; pt[3 * i + 2] = (float)st[8];
    un[i] = (float)st[0]; us[i] = (float)st[1]; ub[i] = (float)st[2]; ut[i] = (float)st[3];
    sn[i] = (float)st[4]; ss[i] = (float)st[5];
    conn[i] = (int32_t)i;
    offs[i] = (int32_t)(i + 1);
    mid[i] = in.bond_ids[2 * i];
    sid[i] = in.bond_ids[2 * i + 1];
    act[i] = in.bond_bonded[i];
  }
  std::ostringstream o;
  o << head(in.time, in.step) << "<Piece NumberOfPoints=\"" << N << "\" NumberOfCells=\"" << N << "\">\n"
    << "<Points>\n<DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"binary\">\n";
  f.put(o.str());
  emit_host(c, f.f, pt, 3);
  f.put(std::string(kEnd) + "</Points>\n<Cells>\n<DataArray type=\"Int32\" Name=\"connectivity\" format=\"binary\">\n");
  emit_host(c, f.f, conn, 1);
  f.put(std::string(kEnd) + "<DataArray type=\"Int32\" Name=\"offsets\" format=\"binary\">\n");
  emit_host(c, f.f, offs, 1);
  f.put(std::string(kEnd) + "<DataArray type=\"UInt8\" Name=\"types\" format=\"binary\">\n");
  emit_host(c, f.f, types, 1);
  f.put(std::string(kEnd) + "</Cells>\n<PointData Scalars=\"activated\">\n" +
        "<DataArray type=\"Int32\" Name=\"masterObjectID\" format=\"binary\">\n");
  emit_host(c, f.f, mid, 1);
  f.put(std::string(kEnd) + "<DataArray type=\"Int32\" Name=\"slaveObjectID\" format=\"binary\">\n");
  emit_host(c, f.f, sid, 1);
  f.put(std::string(kEnd) + "<DataArray type=\"Int32\" Name=\"activated\" format=\"binary\">\n");
  emit_host(c, f.f, act, 1);
  const char* names[6] = {"normalElasticEnergy", "shearElasticEnergy", "bendingElasticEnergy", "torsionElasticEnergy",
                          "maxNormalStress", "maxShearStress"};
  const std::vector<float>* vals[6] = {&un, &us, &ub, &ut, &sn, &ss};
  for (int k = 0; k < 6; ++k) {
    f.put(std::string(kEnd) + "<DataArray type=\"Float32\" Name=\"" + names[k] + "\" format=\"binary\">\n");
    emit_host(c, f.f, *vals[k], 1);
  }
  f.put(std::string(kEnd) + kTail);
}

// Wall mesh file: the walls' vertices in world coordinates and their triangles, written
// by the same mesh writer as the particles (LSParticle::outputVTU on the wall set).
void write_walls(VtuCtx& c, const VtuInput& in, const std::string& dir) {
  mkdir(dir);
  File f(name(dir, "LSObjectMesh", in.frame));
  std::vector<float> pt, vel;
  std::vector<int32_t> id, conn, offs;
  std::vector<uint8_t> types;
  int base = 0;
  for (int w = 0; w < in.nw; ++w) {
    const std::vector<double>& v = *in.wall_verts[w];
    const double3 x = d3(in.wpos[3 * w], in.wpos[3 * w + 1], in.wpos[3 * w + 2]);
    const Quat q{in.wquat[4 * w], in.wquat[4 * w + 1], in.wquat[4 * w + 2], in.wquat[4 * w + 3]};
    const double3 wv = d3(in.wvel[3 * w], in.wvel[3 * w + 1], in.wvel[3 * w + 2]);
    const double3 ww = d3(in.wangvel[3 * w], in.wangvel[3 * w + 1], in.wangvel[3 * w + 2]);
    for (size_t i = 0; i < v.size() / 3; ++i) {
      const double3 pw = x + rotate(q, d3(v[3 * i], v[3 * i + 1], v[3 * i + 2]));
      const double3 vw = wv + cross(ww, pw - x);
      pt.insert(pt.end(), {(float)pw.x, (float)pw.y, (float)pw.z});
      vel.insert(vel.end(), {(float)vw.x, (float)vw.y, (float)vw.z});
      id.push_back(w);
    }
    if (in.wall_tris[w])
      for (size_t t = 0; t < in.wall_tris[w]->size(); ++t) {
        conn.push_back((*in.wall_tris[w])[t] + base);
        if (t % 3 == 2) {
          offs.push_back((int32_t)conn.size());
          types.push_back(5);
        }
      }
    base += (int)(v.size() / 3);
  }
  std::ostringstream o;
  o << head(in.time, in.step) << "<Piece NumberOfPoints=\"" << id.size() << "\" NumberOfCells=\"" << offs.size()
    << "\">\n<Points>\n<DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"binary\">\n";
  f.put(o.str());
  emit_host(c, f.f, pt, 3);
  f.put(std::string(kEnd) + "</Points>\n<Cells>\n<DataArray type=\"Int32\" Name=\"connectivity\" format=\"binary\">\n");
  emit_host(c, f.f, conn, 3);
  f.put(std::string(kEnd) + "<DataArray type=\"Int32\" Name=\"offsets\" format=\"binary\">\n");
  emit_host(c, f.f, offs, 1);
  f.put(std::string(kEnd) + "<DataArray type=\"UInt8\" Name=\"types\" format=\"binary\">\n");
  emit_host(c, f.f, types, 1);
  f.put(std::string(kEnd) + "</Cells>\n<PointData Vectors=\"velocity\">\n" + arr("Int32", "particleID", 0));
  emit_host(c, f.f, id, 1);
  f.put(std::string(kEnd) + arr("Float32", "velocity", 3));
  emit_host(c, f.f, vel, 3);
  f.put(std::string(kEnd) + kTail);
}

}  // namespace

void vtu_write(VtuCtx*& cp, const VtuInput& in) {
  if (!cp) {
    std::unique_ptr<VtuCtx> c(new VtuCtx);
    ck(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    c->d_elem = dalloc<uint8_t>(kChunkBytes);
    for (int k = 0; k < 2; ++k) {
      c->d_enc[k] = dalloc<char>(kEncBytes);
      c->d_carry[k] = dalloc<uint8_t>(16);
      ck(cudaMallocHost(&c->h_pin[k], kEncBytes));
      ck(cudaEventCreateWithFlags(&c->ev[k], cudaEventDisableTiming));
    }
    cp = c.release();
  }
  VtuCtx& c = *cp;
  // the state arrays belong to the solver's stream: order this writer's stream after it
  cudaEvent_t ready;
  ck(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  ck(cudaEventRecord(ready, in.solver_stream));
  ck(cudaStreamWaitEvent(c.st, ready, 0));
  cudaEventDestroy(ready);
  const std::string& d = in.dir;
  if (in.n > 0) {
    upload_layout(c, in);
    write_mesh_particles(c, in, d + "/LSParticle");
    write_particles(c, in, d + "/LSParticle");
  }
  write_contacts(c, in, in.pp, d + "/LSParticleInteraction");
  if (!in.bond_bonded.empty()) write_bonds(c, in, d + "/LSParticleInteraction");
  if (in.nw > 0) write_walls(c, in, d + "/Wall");
  write_contacts(c, in, in.pw, d + "/LSParticle-WallInteraction");
  ck(cudaStreamSynchronize(c.st));
}

}  // namespace lsdem
