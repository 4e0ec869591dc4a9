// Device-wide prefix sums and the stable cell bucket sort of the broadphase.
//
// Replaces the reference's thrust::inclusive_scan / thrust::sort_by_key +
// findStartAndEnd (FunDEM/kernel/CUDAKernelFunction/myUtility/buildHashStartEnd.cu:18-66,
// :69-137, :139-178). Cell keys are small integers, so instead of a radix sort
// the particles are bucketed by key (histogram -> exclusive scan -> scatter)
// and each bucket is put back into ascending particle order, which yields
// exactly the order of a stable sort by key. Memory traffic per particle:
// key read three times, index written twice, plus 8 B per cell.
#include <algorithm>

#include "kernels.h"

namespace lsdem {

static constexpr int SCAN_THREADS = 1024;
static constexpr int SCAN_ITEMS = 4;
static constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

// Launches given a gate flag return at once when it is zero (the step keeps the
// last sort's results, which are still in place).
__device__ __forceinline__ bool idle(const int* gate) { return gate && *gate == 0; }

template <typename T>
__device__ T block_exclusive_scan(T v, T* smem_warp, T* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    T w = (lane < (int)(blockDim.x >> 5)) ? smem_warp[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    smem_warp[lane] = w;
  }
  __syncthreads();
  T warp_off = warp > 0 ? smem_warp[warp - 1] : T(0);
  if (total) *total = smem_warp[(blockDim.x >> 5) - 1];
  __syncthreads();
  return warp_off + x - v;
}

template <typename T>
__global__ void k_scan_tile_sums(const T* __restrict__ in, long long n, T* __restrict__ sums, const int* gate) {
  if (idle(gate)) return;
  __shared__ T sw[32];
  long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
  T s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k)
    if (base + k < n) s += in[base + k];
  T tot;
  block_exclusive_scan<T>(s, sw, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Exclusive scan of `n` tile sums in place by a single block, chunk by chunk.
template <typename T>
__global__ void k_scan_sums(T* sums, long long n, const int* gate) {
  if (idle(gate)) return;
  __shared__ T sw[32];
  T carry = 0;
  for (long long c = 0; c < n; c += SCAN_TILE) {
    long long base = c + (long long)threadIdx.x * SCAN_ITEMS;
    T v[SCAN_ITEMS];
    T s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
      v[k] = (base + k < n) ? sums[base + k] : T(0);
      s += v[k];
    }
    T tot;
    T ex = block_exclusive_scan<T>(s, sw, &tot);
    T run = carry + ex;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
      if (base + k < n) sums[base + k] = run;
      run += v[k];
    }
    carry += tot;
    __syncthreads();
  }
}

template <typename T>
__global__ void k_scan_apply(const T* __restrict__ in, T* __restrict__ out, long long n, const T* __restrict__ sums,
                             int inclusive, const int* gate) {
  if (idle(gate)) return;
  __shared__ T sw[32];
  long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
  T v[SCAN_ITEMS];
  T s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    v[k] = (base + k < n) ? in[base + k] : T(0);
    s += v[k];
  }
  T ex = block_exclusive_scan<T>(s, sw, nullptr);
  T run = sums[blockIdx.x] + ex;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    if (base + k < n) {
      if (inclusive) { run += v[k]; out[base + k] = run; }
      else { out[base + k] = run; run += v[k]; }
    }
  }
}

size_t scan_temp_elems(long long n) { return (size_t)((n + SCAN_TILE - 1) / SCAN_TILE) + 1; }

template <typename T>
void scan_impl(const T* in, T* out, long long n, T* tmp, bool inclusive, cudaStream_t s, const int* gate) {
  if (n <= 0) return;
  long long tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  k_scan_tile_sums<T><<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(in, n, tmp, gate);
  k_scan_sums<T><<<1, SCAN_THREADS, 0, s>>>(tmp, tiles, gate);
  k_scan_apply<T><<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(in, out, n, tmp, inclusive ? 1 : 0, gate);
}

void scan_i32(const int* in, int* out, long long n, int* tmp, bool inclusive, cudaStream_t s, const int* gate) {
  scan_impl<int>(in, out, n, tmp, inclusive, s, gate);
}
void scan_i64(const long long* in, long long* out, long long n, long long* tmp, bool inclusive, cudaStream_t s) {
  scan_impl<long long>(in, out, n, tmp, inclusive, s, nullptr);
}

// ---------------------------------------------------------------------------
// Bucket sort by cell key.
// Bucket of a key: 0 for -1 (outside the domain), 1 + key for a cell, and a
// last bucket for keys >= ncells (a centre rounding onto the upper domain face),
// which, as in the reference, sort after every cell, by key, and belong to none.
__device__ __forceinline__ int bucket_of(int k, int ncells) { return k < 0 ? 0 : (k >= ncells ? ncells + 1 : k + 1); }

__global__ void k_bucket_clear(int* __restrict__ counts, int* __restrict__ fill, int m, int* __restrict__ big_count,
                               const int* gate) {
  if (idle(gate)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) { counts[i] = 0; fill[i] = 0; }
  if (i == 0) big_count[0] = big_count[1] = 0;  // buckets for k_bucket_big, for k_bucket_mid
}

__global__ void k_bucket_hist(const int* __restrict__ key, int n, int ncells, int* __restrict__ counts, const int* gate) {
  if (idle(gate)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  atomicAdd(&counts[bucket_of(key[i], ncells)], 1);
}

__global__ void k_bucket_scatter(const int* __restrict__ key, int n, int ncells, const int* __restrict__ offs,
                                 int* __restrict__ fill, int* __restrict__ sorted_idx, const int* gate) {
  if (idle(gate)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = bucket_of(key[i], ncells);
  // a special bucket longer than a warp can rank is placed in index order by k_special_buckets
  if ((b == 0 || b == ncells + 1) && offs[b + 1] - offs[b] > 64) return;
  int p = offs[b] + atomicAdd(&fill[b], 1);
  sorted_idx[p] = i;
}

// Bodies outside every cell (bucket 0: key -1; last bucket: key past the last
// cell) can be numerous, e.g. bodies that left a non-periodic domain. A special
// bucket of up to 64 members is scattered and ranked like any other; a longer
// one is placed directly in ascending index order by one block walking the
// bodies in tiles: two block-wide scans of the membership flags give each
// member its rank. Exits at once when neither bucket is longer than 64.
__global__ void k_special_buckets(const int* __restrict__ key, int n, int ncells, const int* __restrict__ offs,
                                  int* __restrict__ sorted_idx, const int* gate) {
  if (idle(gate)) return;
  __shared__ int sw[32];
  const int L = ncells + 1;
  const int n0 = offs[1] - offs[0], nL = offs[L + 1] - offs[L];
  if (n0 <= 64 && nL <= 64) return;
  int base0 = offs[0], baseL = offs[L];
  for (int t0 = 0; t0 < n; t0 += blockDim.x) {
    const int i = t0 + threadIdx.x;
    const int b = i < n ? bucket_of(key[i], ncells) : -1;
    const int f0 = b == 0 && n0 > 64, fL = b == L && nL > 64;
    int tot0, totL;
    const int r0 = block_exclusive_scan<int>(f0, sw, &tot0);
    const int rL = block_exclusive_scan<int>(fL, sw, &totL);
    if (f0) sorted_idx[base0 + r0] = i;
    if (fL) sorted_idx[baseL + rL] = i;
    base0 += tot0;
    baseL += totL;
  }
}

// (key, index) order: a stable sort by key puts the keys past the last cell, which
// share the last bucket, in ascending key and then index order.
__device__ __forceinline__ bool key_idx_less(int ka, int a, int kb, int b) { return ka < kb || (ka == kb && a < b); }

// Compare-exchange of two (key, index) entries.
__device__ __forceinline__ void cx(int& ka, int& a, int& kb, int& b) {
  if (key_idx_less(kb, b, ka, a)) {
    const int t = a, tk = ka;
    a = b; ka = kb;
    b = t; kb = tk;
  }
}

// Cell ranges [start, end) of every cell (-1 when empty; findStartAndEnd,
// buildHashStartEnd.cu:47-67) and the stable order inside each bucket (the
// scatter leaves members in arbitrary order), one thread per bucket: a bucket of up
// to 8 members is put in order in registers by an odd-even transposition network
// (by particle index; the last bucket, whose keys differ, by key, then index);
// buckets of 9 to 64 members are listed for k_bucket_mid (in tmp, which k_bucket_big
// uses only after it), longer ones for k_bucket_big, except the -1 bucket, which
// k_special_buckets has put in index order.
__global__ void k_bucket_fix(const int* __restrict__ key, const int* __restrict__ offs, int nbuckets, int ncells,
                             int* __restrict__ sorted_idx, int* __restrict__ start, int* __restrict__ end,
                             int* __restrict__ big_list, int* __restrict__ big_count, int* __restrict__ mid_list,
                             const int* gate) {
  if (idle(gate)) return;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbuckets) return;
  const int s = offs[b], e = offs[b + 1], L = e - s;
  if (b > 0 && b <= ncells) {
    start[b - 1] = L > 0 ? s : -1;
    end[b - 1] = L > 0 ? e : -1;
  }
  if (L <= 1) return;
  if (b == 0 && L > 64) return;  // placed in index order by k_special_buckets
  if (L > 64) {
    // the last bucket was put in index order by k_special_buckets; k_bucket_big
    // re-ranks it by key
    big_list[atomicAdd(&big_count[0], 1)] = b;
    return;
  }
  if (L > 8) {
    mid_list[atomicAdd(&big_count[1], 1)] = b;
    return;
  }
  const bool bykey = b == ncells + 1;
  int v[8], k[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    v[j] = j < L ? sorted_idx[s + j] : 0x7fffffff;
    k[j] = (j < L && bykey) ? key[v[j]] : (j < L ? 0 : 0x7fffffff);
  }
#pragma unroll
  for (int r = 0; r < 8; ++r) {
#pragma unroll
    for (int j = r & 1; j + 1 < 8; j += 2) cx(k[j], v[j], k[j + 1], v[j + 1]);
  }
#pragma unroll
  for (int j = 0; j < 8; ++j)
    if (j < L) sorted_idx[s + j] = v[j];
}

// One warp per listed bucket of 9 to 64 members: ranked by particle index in registers
// (the last bucket by key, then index).
__global__ void k_bucket_mid(const int* __restrict__ key, const int* __restrict__ offs, int ncells,
                             const int* __restrict__ mid_list, const int* __restrict__ big_count,
                             int* __restrict__ sorted_idx, const int* gate) {
  if (idle(gate)) return;
  const int lane = threadIdx.x & 31;
  const int nmid = big_count[1];
  for (int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < nmid; q += (gridDim.x * blockDim.x) >> 5) {
    const int b = mid_list[q];
    const int s = offs[b], L = offs[b + 1] - s;
    const int v0 = lane < L ? sorted_idx[s + lane] : 0x7fffffff;
    const int v1 = lane + 32 < L ? sorted_idx[s + 32 + lane] : 0x7fffffff;
    int r0 = 0, r1 = 0;
    if (b == ncells + 1) {
      const int k0 = lane < L ? key[v0] : 0x7fffffff, k1 = lane + 32 < L ? key[v1] : 0x7fffffff;
      for (int j = 0; j < 32; ++j) {
        const int u0 = __shfl_sync(0xffffffffu, v0, j), u1 = __shfl_sync(0xffffffffu, v1, j);
        const int w0 = __shfl_sync(0xffffffffu, k0, j), w1 = __shfl_sync(0xffffffffu, k1, j);
        r0 += key_idx_less(w0, u0, k0, v0) + key_idx_less(w1, u1, k0, v0);
        r1 += key_idx_less(w0, u0, k1, v1) + key_idx_less(w1, u1, k1, v1);
      }
    } else {
      for (int j = 0; j < 32; ++j) {
        const int u0 = __shfl_sync(0xffffffffu, v0, j), u1 = __shfl_sync(0xffffffffu, v1, j);
        r0 += (u0 < v0) + (u1 < v0);
        r1 += (u0 < v1) + (u1 < v1);
      }
    }
    __syncwarp();
    if (lane < L) sorted_idx[s + r0] = v0;
    if (lane + 32 < L) sorted_idx[s + r1] = v1;
  }
}
// One block per bucket longer than 64: rank of each member by index (by key, then
// index, in the last bucket, whose keys differ).
__global__ void k_bucket_big(const int* __restrict__ key, const int* __restrict__ offs, int ncells,
                             const int* __restrict__ big_list, const int* __restrict__ big_count,
                             int* __restrict__ sorted_idx, int* __restrict__ tmp, const int* gate) {
  if (idle(gate) || (int)blockIdx.x >= *big_count) return;
  const int b = big_list[blockIdx.x];
  const int s = offs[b], e = offs[b + 1], L = e - s;
  for (int k = threadIdx.x; k < L; k += blockDim.x) tmp[s + k] = sorted_idx[s + k];
  __syncthreads();
  if (b == ncells + 1) {
    for (int k = threadIdx.x; k < L; k += blockDim.x) {
      const int v = tmp[s + k], kv = key[v];
      int r = 0;
      for (int m = 0; m < L; ++m) {
        const int u = tmp[s + m];
        r += key_idx_less(key[u], u, kv, v);
      }
      sorted_idx[s + r] = v;
    }
    return;
  }
  for (int k = threadIdx.x; k < L; k += blockDim.x) {
    const int v = tmp[s + k];
    int r = 0;
    for (int m = 0; m < L; ++m) r += tmp[s + m] < v;
    sorted_idx[s + r] = v;
  }
}

__global__ void k_sorted_keys(const int* __restrict__ key, const int* __restrict__ sorted_idx, int n,
                              int* __restrict__ sorted_key, const int* gate) {
  if (idle(gate)) return;
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) sorted_key[p] = key[sorted_idx[p]];
}

void bucket_sort(const int* key, int n, int ncells, BucketScratch& w, int* sorted_idx, int* sorted_key, int* start,
                 int* end, cudaStream_t s, const int* gate) {
  const int nb = ncells + 2;  // bucket 0: key -1, 1..ncells: cells, ncells+1: keys past the last cell
  k_bucket_clear<<<(nb + 1 + 255) / 256, 256, 0, s>>>(w.counts, w.fill, nb + 1, w.big_count, gate);
  if (n > 0) k_bucket_hist<<<(n + 255) / 256, 256, 0, s>>>(key, n, ncells, w.counts, gate);
  // exclusive scan over nb + 1 entries: offs[nb] = n
  scan_i32(w.counts, w.offs, nb + 1, w.scan_tmp, false, s, gate);
  if (n > 0) {
    k_bucket_scatter<<<(n + 255) / 256, 256, 0, s>>>(key, n, ncells, w.offs, w.fill, sorted_idx, gate);
    k_special_buckets<<<1, 1024, 0, s>>>(key, n, ncells, w.offs, sorted_idx, gate);
  }
  k_bucket_fix<<<(unsigned)((nb + 255) / 256), 256, 0, s>>>(key, w.offs, nb, ncells, sorted_idx, start, end,
                                                            w.big_list, w.big_count, w.tmp, gate);
  // at most n / 9 buckets have 9 to 64 members: one warp each, grid-stride
  const int max_mid = n / 9 + 1;
  const int mid_blocks = std::min((max_mid + 7) / 8, 148 * 16);
  if (n > 8) k_bucket_mid<<<mid_blocks, 256, 0, s>>>(key, w.offs, ncells, w.tmp, w.big_count, sorted_idx, gate);
  // at most n / 65 buckets can exceed 64 members
  int max_big = n / 65 + 1;
  k_bucket_big<<<max_big, 256, 0, s>>>(key, w.offs, ncells, w.big_list, w.big_count, sorted_idx, w.tmp, gate);
  if (sorted_key && n > 0) k_sorted_keys<<<(n + 255) / 256, 256, 0, s>>>(key, sorted_idx, n, sorted_key, gate);
}

}  // namespace lsdem
