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
#include <mutex>
#include <vector>

#include "../../include/kdb_b200.h"
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

// ---------------------------------------------------------------------------
// Allocation-free sort entry point.
//
// Some callers cannot allocate device memory at the moment they need a sort:
// code recording a CUDA graph (cudaMalloc is not a stream operation and breaks
// the capture), host callbacks and driver-owned threads where CUDA
// allocation calls are not allowed, and host engines that budget every byte
// of HBM through their own allocator and forbid hidden allocations from a
// library.  kdb_sort_pairs_noalloc serves them: the radix passes' scratch (a
// second key/value buffer and the per-block digit histograms) lives in one
// file-scope __device__ array sized for KDB_SORT_NOALLOC_MAX_PAIRS pairs,
// which each GPU that loads this library holds until the process exits.
// ---------------------------------------------------------------------------
namespace kdb {
namespace {

constexpr int64_t kNoAllocMaxPairs = KDB_SORT_NOALLOC_MAX_PAIRS;
constexpr int64_t kNoAllocMaxBlocks = (kNoAllocMaxPairs + kSortTile - 1) / kSortTile;
constexpr size_t kNoAllocKeyBytes = sizeof(uint64_t) * kNoAllocMaxPairs;
constexpr size_t kNoAllocValBytes = sizeof(uint32_t) * kNoAllocMaxPairs;
constexpr size_t kNoAllocHistBytes = sizeof(uint32_t) * 256 * kNoAllocMaxBlocks;
constexpr size_t kNoAllocScratchBytes = kNoAllocKeyBytes + kNoAllocValBytes + kNoAllocHistBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device.  In host code the array's
// name is only a host-side stand-in, so its device address is looked up once
// per device, with that device current, through cudaGetSymbolAddress.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};

int NoAllocScratch(unsigned char** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return KDB_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return KDB_ERR_CUDA;
    g_noalloc_addr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_addr[dev]);
  return KDB_OK;
}

}  // namespace
}  // namespace kdb

extern "C" int kdb_sort_pairs_noalloc(uint64_t* d_keys, uint32_t* d_vals, int64_t n,
                                      int32_t key_bits, void* stream) {
  using namespace kdb;
  if (n < 0 || (n > 0 && (!d_keys || !d_vals)) || key_bits < 1 || key_bits > 64)
    return KDB_ERR_INVALID;
  if (n > kNoAllocMaxPairs) return KDB_ERR_CAPACITY;  // scratch holds at most this many pairs
  unsigned char* scratch = nullptr;
  int rc = NoAllocScratch(&scratch);
  if (rc != KDB_OK) return rc;
  if (n <= 1) return KDB_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n <= kSmallSort) {
    uint64_t mask = key_bits >= 64 ? ~0ULL : ((1ULL << key_bits) - 1);
    SmallRankSort<<<1, 1024, 0, s>>>(d_keys, d_vals, static_cast<int>(n), mask);
    return cudaGetLastError() == cudaSuccess ? KDB_OK : KDB_ERR_CUDA;
  }
  int nblocks = static_cast<int>((n + kSortTile - 1) / kSortTile);
  uint64_t* k2 = reinterpret_cast<uint64_t*>(scratch);
  uint32_t* v2 = reinterpret_cast<uint32_t*>(scratch + kNoAllocKeyBytes);
  uint32_t* hist = reinterpret_cast<uint32_t*>(scratch + kNoAllocKeyBytes + kNoAllocValBytes);
  uint64_t* ka = d_keys;
  uint32_t* va = d_vals;
  uint64_t* kb = k2;
  uint32_t* vb = v2;
  int passes = (key_bits + 7) / 8;
  for (int p = 0; p < passes; p++) {
    int shift = 8 * p;
    // every histogram entry is rewritten by each pass, so nothing left in the
    // shared scratch by an earlier call is read
    RadixHistogram<<<nblocks, kSortBlock, 0, s>>>(ka, n, shift, hist, nblocks);
    ExclusiveScanSmall<<<1, 1024, 0, s>>>(hist, static_cast<int64_t>(nblocks) * 256);
    RadixScatter<<<nblocks, kSortBlock, 0, s>>>(ka, va, kb, vb, n, shift, hist, nblocks);
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != d_keys) {
    int grid = static_cast<int>(std::min<int64_t>((n + 255) / 256, 4096));
    CopyPairs<<<grid, 256, 0, s>>>(ka, va, d_keys, d_vals, n);
  }
  return cudaGetLastError() == cudaSuccess ? KDB_OK : KDB_ERR_CUDA;
}
