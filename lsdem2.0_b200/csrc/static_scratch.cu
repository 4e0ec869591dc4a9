// Cell sort with no device allocation: lsdem_cell_sort_static.
//
// Some callers of this library cannot allocate device memory when they call
// it: latency-critical loops in which an allocation may block or synchronise
// the device, and host applications whose device memory is owned by their own
// pool allocator or held to a fixed budget. This entry point gives them the
// broadphase cell sort (cell keys, stable sorted order, per-cell ranges) with
// all of its scratch memory in one file-scope device array of fixed size, so a
// call allocates and frees nothing: the caller passes the inputs and outputs.
//
// Limits: at most kMaxBodies bodies and kMaxCells cells per call (4.2 MB of
// scratch, held by every GPU that loads the library until the process exits).
//
// Host code cannot name the device array's address directly: the symbol seen
// by host code is a host-side stand-in. The first call on each device looks the
// device address up with cudaGetSymbolAddress while that device is current,
// so that first call should come before any stream capture. The address is kept
// for the life of the process: after cudaDeviceReset on a device, the library's
// device array may sit elsewhere, so this entry point must not be called on that
// device again in the same process. Every call shares
// the array and it keeps the last call's contents; each call clears what must
// start at zero. Calls that overlap on the GPU (for example on two streams at
// once) race on the shared array.
#include <cstdio>
#include <mutex>

#include "../../include/lsdem_b200.h"
#include "kernels.h"

namespace lsdem {
namespace {

constexpr int kMaxBodies = 1 << 18;
constexpr int kMaxCells = 1 << 18;
constexpr int kMaxDevices = 64;

// Scratch of one bucket sort, in ints: counts, fill and offsets (cells + 3
// each), scan partial sums, list of large buckets, its counter, and a copy
// buffer of one entry per body; each part starts on a 64-int (256 B) boundary.
constexpr size_t align64(size_t v) { return (v + 63) / 64 * 64; }
constexpr size_t kBuckets = (size_t)kMaxCells + 3;
constexpr size_t kScanTmp = kBuckets / 4096 + 4;
constexpr size_t kBig = (size_t)kMaxBodies / 65 + 1;
constexpr size_t kScratchInts =
    3 * align64(kBuckets) + align64(kScanTmp) + align64(kBig) + align64(1) + align64(kMaxBodies);

static __device__ __align__(256) int g_scratch[kScratchInts];

std::mutex g_mu;
int* g_addr[kMaxDevices] = {nullptr};

__global__ void k_cell_keys(const double3* __restrict__ pos, int n, GridP g, int* __restrict__ key) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) key[i] = hash_key(pos[i], g);
}

}  // namespace
}  // namespace lsdem

extern "C" int lsdem_cell_sort_static(const void* pos_dev, int n, const double* min3, const double* max3,
                                      const double* inv3, const int* size3, int* key_dev, int* sorted_idx_dev,
                                      int* sorted_key_dev, int* cell_start_dev, int* cell_end_dev, void* stream) {
  using namespace lsdem;
  if (n < 0 || !min3 || !max3 || !inv3 || !size3 || (n > 0 && (!pos_dev || !key_dev || !sorted_idx_dev)) ||
      !cell_start_dev || !cell_end_dev) {
    fprintf(stderr, "lsdem_cell_sort_static: null or negative argument\n");
    return LSDEM_ERR_ARG;
  }
  // each factor is checked before the product, which then cannot overflow
  const bool sizes_ok = size3[0] >= 1 && size3[1] >= 1 && size3[2] >= 1 && size3[0] <= kMaxCells &&
                        size3[1] <= kMaxCells && size3[2] <= kMaxCells;
  const long long ncells = sizes_ok ? (long long)size3[0] * size3[1] * size3[2] : -1;
  if (!sizes_ok || ncells > kMaxCells || n > kMaxBodies) {
    fprintf(stderr,
            "lsdem_cell_sort_static: %d bodies / %lld cells exceed the fixed scratch (at most %d bodies and %d "
            "cells)\n",
            n, ncells, kMaxBodies, kMaxCells);
    return LSDEM_ERR_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return LSDEM_ERR_NODEVICE;
  int* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
      if (e != cudaSuccess || !p) {
        fprintf(stderr, "lsdem_cell_sort_static: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
        return LSDEM_ERR_CUDA;
      }
      g_addr[dev] = (int*)p;
    }
    base = g_addr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  GridP g;
  g.mn = make_double3(min3[0], min3[1], min3[2]);
  g.mx = make_double3(max3[0], max3[1], max3[2]);
  g.inv = make_double3(inv3[0], inv3[1], inv3[2]);
  g.size = make_int3(size3[0], size3[1], size3[2]);
  g.ncells = (int)ncells;
  int* p = base;
  BucketScratch w;
  w.counts = p; p += align64(kBuckets);
  w.fill = p; p += align64(kBuckets);
  w.offs = p; p += align64(kBuckets);
  w.scan_tmp = p; p += align64(kScanTmp);
  w.big_list = p; p += align64(kBig);
  w.big_count = p; p += align64(1);
  w.tmp = p;
  if (n > 0) k_cell_keys<<<(n + 255) / 256, 256, 0, st>>>((const double3*)pos_dev, n, g, key_dev);
  // bucket_sort clears counts, fill and the large-bucket counter itself
  bucket_sort(key_dev, n, (int)ncells, w, sorted_idx_dev, sorted_key_dev, cell_start_dev, cell_end_dev, st);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "lsdem_cell_sort_static: %s\n", cudaGetErrorString(e));
    return LSDEM_ERR_CUDA;
  }
  return LSDEM_OK;
}
