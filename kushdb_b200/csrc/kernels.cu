// Static (nvcc-compiled, sm_100a) kernels used by every query: stable LSD
// radix sort of (uint64 key, uint32 value) pairs, the order-by tie-break key,
// and gathers.
//
// ORDER BY in the reference materialises the child into a runtime::Vector and
// runs a top-down merge sort whose merge takes the right element on ties
// (runtime/vector.cc:45-110, comparator order_by_translator.cc:54-75).  Here
// the same order is produced by stable radix passes: first on a "tie path"
// key that encodes where that merge sort leaves equal rows, then on each sort
// key from the least to the most significant.
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "engine.h"

namespace kdb {
namespace {

constexpr int kSortBlock = 256;
constexpr int kSortTile = 4096;  // items per block per pass
constexpr int kSortWarps = kSortBlock / 32;

__global__ void __launch_bounds__(kSortBlock) RadixHistogram(const uint64_t* __restrict__ keys,
                                                             int64_t n, int shift,
                                                             uint32_t* __restrict__ hist,
                                                             int nblocks) {
  __shared__ uint32_t h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  int64_t base = static_cast<int64_t>(blockIdx.x) * kSortTile;
  int64_t end = min(base + kSortTile, n);
  for (int64_t i = base + threadIdx.x; i < end; i += blockDim.x)
    atomicAdd(&h[(keys[i] >> shift) & 0xff], 1u);
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[d * nblocks + blockIdx.x] = h[d];
}

// Exclusive scan of `count` uint32 in place (one block of 1024 threads).
__global__ void __launch_bounds__(1024) ExclusiveScanSmall(uint32_t* __restrict__ a,
                                                           int64_t count) {
  __shared__ uint32_t partial[1024];
  int t = threadIdx.x;
  int64_t per = (count + blockDim.x - 1) / blockDim.x;
  int64_t b = t * per, e = min(b + per, count);
  uint32_t s = 0;
  for (int64_t i = b; i < e; i++) s += a[i];
  partial[t] = s;
  __syncthreads();
  if (t == 0) {
    uint32_t run = 0;
    for (int i = 0; i < static_cast<int>(blockDim.x); i++) {
      uint32_t x = partial[i];
      partial[i] = run;
      run += x;
    }
  }
  __syncthreads();
  uint32_t run = partial[t];
  for (int64_t i = b; i < e; i++) {
    uint32_t x = a[i];
    a[i] = run;
    run += x;
  }
}

// Stable scatter: each block walks its tile in chunks of blockDim items in
// order; ranks inside a chunk come from a warp match plus per-warp digit
// counts prefixed in warp order.
__global__ void __launch_bounds__(kSortBlock) RadixScatter(
    const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint64_t* __restrict__ kout,
    uint32_t* __restrict__ vout, int64_t n, int shift, const uint32_t* __restrict__ offsets,
    int nblocks) {
  __shared__ uint32_t base[256];
  __shared__ uint32_t total[256];
  __shared__ uint32_t wcnt[kSortWarps][256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = threadIdx.x; d < 256; d += blockDim.x) base[d] = offsets[d * nblocks + blockIdx.x];
  int64_t tile = static_cast<int64_t>(blockIdx.x) * kSortTile;
  int64_t end = min(tile + kSortTile, n);
  for (int64_t c = tile; c < end; c += blockDim.x) {
    for (int i = threadIdx.x; i < kSortWarps * 256; i += blockDim.x) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    int64_t i = c + threadIdx.x;
    bool valid = i < end;
    uint64_t k = valid ? kin[i] : 0;
    uint32_t v = valid ? vin[i] : 0;
    uint32_t digit = valid ? static_cast<uint32_t>((k >> shift) & 0xff) : 256u;
    unsigned peers = __match_any_sync(0xffffffffu, digit);
    uint32_t rank = __popc(peers & ((1u << lane) - 1));
    if (valid && rank == 0) wcnt[warp][digit] = __popc(peers);
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) {
      uint32_t run = 0;
      for (int w = 0; w < kSortWarps; w++) {
        uint32_t x = wcnt[w][d];
        wcnt[w][d] = run;
        run += x;
      }
      total[d] = run;
    }
    __syncthreads();
    if (valid) {
      uint32_t dst = base[digit] + wcnt[warp][digit] + rank;
      kout[dst] = k;
      vout[dst] = v;
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) base[d] += total[d];
    __syncthreads();
  }
}

// Stable sort of at most kSmallSort pairs in one block: an element's rank is
// the number of smaller keys plus the equal keys before it.
constexpr int kSmallSort = 2048;

__global__ void __launch_bounds__(1024) SmallRankSort(uint64_t* __restrict__ keys,
                                                      uint32_t* __restrict__ vals, int n,
                                                      uint64_t mask) {
  __shared__ uint64_t sk[kSmallSort];
  __shared__ uint64_t sfull[kSmallSort];
  __shared__ uint32_t sv[kSmallSort];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    sfull[i] = keys[i];
    sk[i] = keys[i] & mask;
    sv[i] = vals[i];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    uint64_t k = sk[i];
    int r = 0;
    for (int j = 0; j < n; j++) r += (sk[j] < k) || (sk[j] == k && j < i);
    keys[r] = sfull[i];
    vals[r] = sv[i];
  }
}

__global__ void CopyPairs(const uint64_t* __restrict__ ks, const uint32_t* __restrict__ vs,
                          uint64_t* __restrict__ kd, uint32_t* __restrict__ vd, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    kd[i] = ks[i];
    vd[i] = vs[i];
  }
}

}  // namespace

// Sorts (keys, vals) by the low `key_bits` bits of keys, stably.
void Context::RadixSortPairs(uint64_t* keys, uint32_t* vals, int64_t n, Arena& arena,
                             int key_bits) {
  if (n <= 1 || dry) return;
  if (n > 0xffffffffLL) throw Error(-5, "sort of more than 2^32 rows");
  if (n <= kSmallSort) {
    uint64_t mask = key_bits >= 64 ? ~0ULL : ((1ULL << key_bits) - 1);
    TimedStart("sort small");
    SmallRankSort<<<1, 1024, 0, stream>>>(keys, vals, static_cast<int>(n), mask);
    TimedStop();
    kernel_launches++;
    KDB_CUDA(cudaGetLastError());
    return;
  }
  int nblocks = static_cast<int>((n + kSortTile - 1) / kSortTile);
  uint64_t* k2 = arena.AllocT<uint64_t>(n);
  uint32_t* v2 = arena.AllocT<uint32_t>(n);
  uint32_t* hist = arena.AllocT<uint32_t>(static_cast<size_t>(nblocks) * 256);
  uint64_t* ka = keys;
  uint32_t* va = vals;
  uint64_t* kb = k2;
  uint32_t* vb = v2;
  int passes = (key_bits + 7) / 8;
  for (int p = 0; p < passes; p++) {
    int shift = 8 * p;
    TimedStart("sort histogram");
    RadixHistogram<<<nblocks, kSortBlock, 0, stream>>>(ka, n, shift, hist, nblocks);
    TimedStop();
    TimedStart("sort scan");
    ExclusiveScanSmall<<<1, 1024, 0, stream>>>(hist, static_cast<int64_t>(nblocks) * 256);
    TimedStop();
    TimedStart("sort scatter");
    RadixScatter<<<nblocks, kSortBlock, 0, stream>>>(ka, va, kb, vb, n, shift, hist, nblocks);
    TimedStop();
    kernel_launches += 3;
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  KDB_CUDA(cudaGetLastError());
  if (ka != keys) {
    TimedStart("sort copy");
    CopyPairs<<<GridFor(n, 256), 256, 0, stream>>>(ka, va, keys, vals, n);
    TimedStop();
    kernel_launches++;
    KDB_CUDA(cudaGetLastError());
  }
}

}  // namespace kdb
