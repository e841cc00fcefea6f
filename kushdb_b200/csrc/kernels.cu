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

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "../../include/kdb_b200.h"
#include "engine.h"

namespace kdb {
namespace {

constexpr int kSortBlock = 256;
constexpr int kSortTile = 4096;  // items per block per pass
constexpr int kSortWarps = kSortBlock / 32;
static_assert(kSortBlock == 256, "one thread per radix digit");
constexpr int64_t kPlanMinRows = 1 << 15;  // below this a counting read costs more than it saves

__global__ void __launch_bounds__(kSortBlock) RadixHistogram(const uint64_t* __restrict__ keys,
                                                             int64_t n, int shift, int tile,
                                                             uint32_t* __restrict__ hist,
                                                             int nblocks) {
  __shared__ uint32_t h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  int64_t base = static_cast<int64_t>(blockIdx.x) * tile;
  int64_t end = min(base + tile, n);
  const int lane = threadIdx.x & 31;
  // one shared-memory atomic per distinct digit in a warp: a skewed key
  // column (many equal keys) would otherwise serialise the block on one counter
  for (int64_t c = base; c < end; c += blockDim.x) {
    const int64_t i = c + threadIdx.x;
    const uint32_t d = i < end ? static_cast<uint32_t>((keys[i] >> shift) & 0xff) : 256u;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    if (d < 256u && lane == __ffs(peers) - 1) atomicAdd(&h[d], static_cast<uint32_t>(__popc(peers)));
  }
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[d * nblocks + blockIdx.x] = h[d];
}

// Digit counts of every 8-bit pass at once (order independent), so passes
// whose digit is the same for every key can be skipped.
__global__ void __launch_bounds__(kSortBlock) RadixDigitCounts(const uint64_t* __restrict__ keys, int64_t n,
                                                               int passes, uint32_t* __restrict__ counts) {
  __shared__ uint32_t h[8][256];
  for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&h[0][0])[i] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  // whole warps step together so that equal digits in a warp add once
  for (int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x); c < n; c += stride) {
    const int64_t i = c + threadIdx.x;
    const bool valid = i < n;
    const uint64_t k = valid ? keys[i] : 0;
    for (int p = 0; p < passes; p++) {
      const uint32_t d = valid ? static_cast<uint32_t>((k >> (8 * p)) & 0xff) : 256u;
      const unsigned peers = __match_any_sync(0xffffffffu, d);
      if (d < 256u && lane == __ffs(peers) - 1) atomicAdd(&h[p][d], static_cast<uint32_t>(__popc(peers)));
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) {
    const uint32_t c = (&h[0][0])[i];
    if (c) atomicAdd(counts + i, c);
  }
}

// Exclusive scan in place by one block of 1024 threads: each thread owns
// kPer contiguous elements of a tile (moved with 16-byte vector loads and
// stores), scans them in registers, the thread sums are scanned with warp
// shuffles, and a carry runs from tile to tile.  With `total`, the sum of all
// elements is also written to total[0].  `a` must be 16-byte aligned.
template <typename T, int kPer>
__device__ __forceinline__ void BlockScanTiles(T* __restrict__ a, int64_t count, T* __restrict__ total) {
  static_assert((kPer * sizeof(T)) % 16 == 0, "whole vectors per thread");
  constexpr int kVec = static_cast<int>(kPer * sizeof(T) / 16);
  constexpr int64_t kTile = 1024LL * kPer;
  __shared__ T warp_sum[32];
  __shared__ T carry;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (t == 0) carry = 0;
  for (int64_t base = 0; base < count; base += kTile) {
    const int64_t i0 = base + static_cast<int64_t>(t) * kPer;
    const bool full = i0 + kPer <= count;
    T v[kPer];
    if (full) {
      const uint4* src = reinterpret_cast<const uint4*>(a + i0);
      uint4 q[kVec];
#pragma unroll
      for (int k = 0; k < kVec; k++) q[k] = src[k];
      memcpy(v, q, sizeof(v));
    } else {
#pragma unroll
      for (int j = 0; j < kPer; j++) v[j] = i0 + j < count ? a[i0 + j] : T(0);
    }
    T s = 0;
#pragma unroll
    for (int j = 0; j < kPer; j++) s += v[j];
    T incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const T w = warp_sum[lane];
      T wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += y;
      }
      warp_sum[lane] = wi - w;
    }
    __syncthreads();
    T run = carry + warp_sum[warp] + incl - s;
    T out[kPer];
#pragma unroll
    for (int j = 0; j < kPer; j++) {
      out[j] = run;
      run += v[j];
    }
    if (full) {
      uint4 q[kVec];
      memcpy(q, out, sizeof(out));
      uint4* dst = reinterpret_cast<uint4*>(a + i0);
#pragma unroll
      for (int k = 0; k < kVec; k++) dst[k] = q[k];
    } else {
#pragma unroll
      for (int j = 0; j < kPer; j++)
        if (i0 + j < count) a[i0 + j] = out[j];
    }
    __syncthreads();
    if (t == 1023) carry = run;
  }
  __syncthreads();
  if (total && t == 0) total[0] = carry;
}

__global__ void __launch_bounds__(1024) ExclusiveScanSmall(uint32_t* __restrict__ a, int64_t count) {
  BlockScanTiles<uint32_t, 16>(a, count, nullptr);
}

// Exclusive scan of n uint64 in place, total written to a[n].
__global__ void __launch_bounds__(1024) ExclusiveScanU64(uint64_t* __restrict__ a, int64_t n) {
  BlockScanTiles<unsigned long long, 8>(reinterpret_cast<unsigned long long*>(a), n,
                                           reinterpret_cast<unsigned long long*>(a) + n);
}

// The same with the count read on the device (*n_ptr); nothing is done when
// it exceeds `cap` (the array's capacity).
__global__ void __launch_bounds__(1024) ExclusiveScanU64Bounded(uint64_t* __restrict__ a,
                                                                const uint64_t* __restrict__ n_ptr, int64_t cap) {
  const int64_t n = static_cast<int64_t>(*n_ptr);
  if (n > cap) return;
  BlockScanTiles<unsigned long long, 8>(reinterpret_cast<unsigned long long*>(a), n,
                                           reinterpret_cast<unsigned long long*>(a) + n);
}

// Stable scatter: each block walks its tile in chunks of blockDim items in
// order; ranks inside a chunk come from a warp match plus per-warp digit
// counts prefixed in warp order.
// Exclusive prefix of the 256 values v (one per thread of a 256-thread
// block) through warp shuffles; `ws` is 8 words of shared scratch.
__device__ __forceinline__ uint32_t BlockExclusive256(uint32_t v, uint32_t* ws) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) ws[warp] = incl;
  __syncthreads();
  uint32_t before = 0;
  for (int w = 0; w < warp; w++) before += ws[w];
  __syncthreads();
  return before + incl - v;
}

// Per digit (one block each): exclusive scan of the digit's per-block counts
// hist[d][0..nblocks) in place, the digit's total into totals[d].
// With `zero_next`, also clears the same digit's row of the next pass's
// counts (which the scatter then fills).
__global__ void __launch_bounds__(kSortBlock) RadixRowScan(uint32_t* __restrict__ hist, int nblocks,
                                                           uint32_t* __restrict__ totals,
                                                           uint32_t* __restrict__ zero_next) {
  __shared__ uint32_t ws[kSortWarps];
  uint32_t* row = hist + static_cast<int64_t>(blockIdx.x) * nblocks;
  if (zero_next)
    for (int i = threadIdx.x; i < nblocks; i += kSortBlock) zero_next[static_cast<int64_t>(blockIdx.x) * nblocks + i] = 0;
  const int per = (nblocks + kSortBlock - 1) / kSortBlock;
  const int b0 = min(static_cast<int>(threadIdx.x) * per, nblocks), e = min(b0 + per, nblocks);
  uint32_t s = 0;
  for (int i = b0; i < e; i++) s += row[i];
  uint32_t run = BlockExclusive256(s, ws);
  if (threadIdx.x == kSortBlock - 1) totals[blockIdx.x] = run + s;
  for (int i = b0; i < e; i++) {
    const uint32_t x = row[i];
    row[i] = run;
    run += x;
  }
}

// `offsets` holds each (digit, block) start: global when `totals` is null
// (one scan over all counts), else relative to the digit, whose start is the
// exclusive prefix of `totals`.  With `next_hist`, every element also counts
// itself in the next pass's per-tile histogram at its destination (the next
// pass needs no histogram launch).
__global__ void __launch_bounds__(kSortBlock) RadixScatter(
    const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint64_t* __restrict__ kout,
    uint32_t* __restrict__ vout, int64_t n, int shift, int tile, const uint32_t* __restrict__ offsets,
    int nblocks, const uint32_t* __restrict__ totals, uint32_t* __restrict__ next_hist, int next_shift) {
  __shared__ uint32_t base[256];
  __shared__ uint32_t total[256];
  __shared__ uint32_t wcnt[kSortWarps][256];
  __shared__ uint32_t ws[kSortWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  {
    const int d = threadIdx.x;  // kSortBlock == 256: one digit per thread
    const uint32_t digit_start = totals ? BlockExclusive256(totals[d], ws) : 0u;
    base[d] = offsets[d * nblocks + blockIdx.x] + digit_start;
  }
  const int64_t first = static_cast<int64_t>(blockIdx.x) * tile;
  const int64_t end = min(first + tile, n);
  for (int64_t c = first; c < end; c += blockDim.x) {
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
    const uint32_t dst = valid ? base[digit] + wcnt[warp][digit] + rank : 0u;
    if (valid) {
      kout[dst] = k;
      vout[dst] = v;
    }
    if (next_hist) {
      // one global atomic per distinct (next digit, destination tile) in the
      // warp: equal keys land in consecutive slots of one tile, and a hot key
      // would otherwise queue thousands of atomics on one counter
      const uint32_t slot = valid ? (dst / static_cast<uint32_t>(tile)) * 256u +
                                        static_cast<uint32_t>((k >> next_shift) & 0xff)
                                  : 0xffffffffu;
      const unsigned grp = __match_any_sync(0xffffffffu, slot);
      if (valid && lane == __ffs(grp) - 1)
        atomicAdd(&next_hist[static_cast<int64_t>(slot & 0xffu) * nblocks + (slot >> 8)],
                  static_cast<uint32_t>(__popc(grp)));
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

// Result download: copies up to kMaxPackSegs device segments into one
// contiguous staging buffer (16-byte aligned offsets), so the host reads the
// whole result with a single copy instead of one per column.
__global__ void PackSegments(PackSegs a, char* __restrict__ dst) {
  const PackSeg& g = a.seg[blockIdx.y];
  const uint64_t nvec = g.bytes / 16;
  const bool aligned = (reinterpret_cast<uintptr_t>(g.src) & 15) == 0;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i * 16 < g.bytes;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    if (aligned && i < nvec) {
      reinterpret_cast<uint4*>(dst + g.off)[i] = reinterpret_cast<const uint4*>(g.src)[i];
    } else {
      for (uint64_t b = i * 16; b < g.bytes && b < i * 16 + 16; b++) dst[g.off + b] = g.src[b];
    }
  }
}

// ---- merge sort of unique (key, tie) pairs ---------------------------------
// ORDER BY on one numeric key: the key and the reference merge sort's tie
// rank together are unique, so any correct sort gives the reference order;
// for mid-size inputs a block sort plus log2(n / tile) merge-path passes
// take far fewer launches than 8-bit radix passes.
struct SortItem {
  uint64_t key;
  uint32_t tie;
  uint32_t val;
};
static_assert(sizeof(SortItem) == 16, "SortItem layout");

__device__ __forceinline__ bool ItemLess(const SortItem& a, const SortItem& b) {
  return a.key < b.key || (a.key == b.key && a.tie < b.tie);
}

constexpr int kMergeTile = 2048;  // largest tile of a block sort or a merge pass

// Shared-memory tiles hold one pad item after every 8, so that the 8
// consecutive items of consecutive threads fall in different banks.
__device__ __forceinline__ int Padded(int i) { return i + (i >> 3); }
template <int TILE>
__host__ __device__ constexpr int PaddedTile() { return TILE + TILE / 8; }

// Number of items of A among the first `diag` outputs of merging A and B,
// where B's item goes first on equal items.  `at`/`bt` read A[i] and B[j].
template <typename AT, typename BT>
__device__ __forceinline__ int MergePathSplit(AT at, int a_len, BT bt, int b_len, int diag) {
  int lo = diag - b_len > 0 ? diag - b_len : 0, hi = diag < a_len ? diag : a_len;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ItemLess(at(mid), bt(diag - 1 - mid))) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// The same split for runs in global memory, searched by a whole warp: each
// step tests 32 evenly spaced candidates, so a run of 2^20 items takes four
// dependent rounds of loads instead of twenty.  Every lane returns the split.
__device__ int64_t WarpMergePathSplit(const SortItem* __restrict__ A, int64_t a_len,
                                      const SortItem* __restrict__ B, int64_t b_len, int64_t diag) {
  const int lane = threadIdx.x & 31;
  int64_t lo = diag - b_len > 0 ? diag - b_len : 0, hi = diag < a_len ? diag : a_len;
  // A[i] is among the first `diag` outputs exactly for i < split, i.e. where
  // A[i] < B[diag - 1 - i]; that test is true on a prefix of [lo, hi)
  while (hi - lo > 32) {
    const int64_t step = (hi - lo + 31) / 32;
    const int64_t p = lo + lane * step;
    const bool before = p < hi && ItemLess(A[p], B[diag - 1 - p]);
    const int k = __popc(__ballot_sync(0xffffffffu, before));
    if (k == 0) return lo;
    const int64_t next_hi = lo + k * step;
    lo = lo + (k - 1) * step + 1;
    hi = next_hi < hi ? next_hi : hi;
  }
  const int64_t p = lo + lane;
  const bool before = p < hi && ItemLess(A[p], B[diag - 1 - p]);
  return lo + __popc(__ballot_sync(0xffffffffu, before));
}

__device__ __forceinline__ void CompareSwap(SortItem& a, SortItem& b) {
  if (ItemLess(b, a)) {
    const SortItem t = a;
    a = b;
    b = t;
  }
}

// Batcher's odd-even merge sort networks for 2, 4 and 8 items (1, 5 and 19
// comparators).
template <int N>
__device__ __forceinline__ void SortNetwork(SortItem (&x)[N]) {
  static_assert(N == 2 || N == 4 || N == 8, "sort network size");
  if constexpr (N == 2) {
    CompareSwap(x[0], x[1]);
  } else if constexpr (N == 4) {
    CompareSwap(x[0], x[1]); CompareSwap(x[2], x[3]);
    CompareSwap(x[0], x[2]); CompareSwap(x[1], x[3]);
    CompareSwap(x[1], x[2]);
  } else {
    CompareSwap(x[0], x[1]); CompareSwap(x[2], x[3]); CompareSwap(x[4], x[5]); CompareSwap(x[6], x[7]);
    CompareSwap(x[0], x[2]); CompareSwap(x[1], x[3]); CompareSwap(x[4], x[6]); CompareSwap(x[5], x[7]);
    CompareSwap(x[1], x[2]); CompareSwap(x[5], x[6]);
    CompareSwap(x[0], x[4]); CompareSwap(x[1], x[5]); CompareSwap(x[2], x[6]); CompareSwap(x[3], x[7]);
    CompareSwap(x[2], x[4]); CompareSwap(x[3], x[5]);
    CompareSwap(x[1], x[2]); CompareSwap(x[3], x[4]); CompareSwap(x[5], x[6]);
  }
}

// Sorts each tile of TILE items of `in` into `out` (which may be `in`):
// every thread sorts ITEMS items in registers, then rounds of merge path in
// shared memory double the sorted runs from ITEMS to TILE items.  Missing
// items of the last tile are maximal padding and never written.
// Tiles above 2048 items keep their items in dynamic shared memory.
template <int TILE, int ITEMS>
__global__ void __launch_bounds__(TILE / ITEMS) BlockSortItems(const SortItem* in, SortItem* out, int64_t n) {
  constexpr int kThreads = TILE / ITEMS;
  constexpr bool kDynamic = TILE > 2048;
  extern __shared__ __align__(16) unsigned char sort_dyn[];
  __shared__ SortItem s_static[kDynamic ? 1 : PaddedTile<TILE>()];
  SortItem* s = kDynamic ? reinterpret_cast<SortItem*>(sort_dyn) : s_static;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * TILE;
  const int cnt = static_cast<int>(n - base < TILE ? n - base : TILE);
  for (int i = threadIdx.x; i < TILE; i += kThreads)
    s[Padded(i)] = i < cnt ? in[base + i] : SortItem{~0ULL, ~0u, ~0u};
  __syncthreads();
  const int d = threadIdx.x * ITEMS;
  SortItem x[ITEMS];
#pragma unroll
  for (int k = 0; k < ITEMS; k++) x[k] = s[Padded(d + k)];
  SortNetwork<ITEMS>(x);
  for (int run = ITEMS; run < TILE; run <<= 1) {
    __syncthreads();
#pragma unroll
    for (int k = 0; k < ITEMS; k++) s[Padded(d + k)] = x[k];
    __syncthreads();
    const int pb = d & ~(2 * run - 1);
    auto at = [&](int i) -> const SortItem& { return s[Padded(pb + i)]; };
    auto bt = [&](int j) -> const SortItem& { return s[Padded(pb + run + j)]; };
    int i = MergePathSplit(at, run, bt, run, d - pb);
    int j = d - pb - i;
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
      const bool take_a = j >= run || (i < run && ItemLess(at(i), bt(j)));
      x[k] = take_a ? at(i++) : bt(j++);
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < ITEMS; k++) s[Padded(d + k)] = x[k];
  __syncthreads();
  for (int i = threadIdx.x; i < cnt; i += kThreads) out[base + i] = s[Padded(i)];
}

// One merge pass: sorted runs of `w` (a multiple of TILE) items merge
// pairwise into runs of 2w.  Each block makes one tile of TILE
// outputs: two warps find the tile's first and last merge-path splits in
// global memory, the block stages the tile's inputs in shared memory with
// coalesced loads, and every thread merges ITEMS outputs from there.
template <int TILE, int ITEMS>
__global__ void __launch_bounds__(TILE / ITEMS) MergeItems(const SortItem* __restrict__ in,
                                                           SortItem* __restrict__ out, int64_t n, int64_t w) {
  constexpr int kThreads = TILE / ITEMS;
  __shared__ SortItem s[PaddedTile<TILE>()];
  __shared__ int64_t split[2];
  const int64_t o0 = static_cast<int64_t>(blockIdx.x) * TILE;
  const int64_t base = o0 / (2 * w) * (2 * w);
  const int64_t a_len = w < n - base ? w : n - base;
  const int64_t b0 = base + w;
  const int64_t b_len = b0 < n ? (w < n - b0 ? w : n - b0) : 0;
  const int64_t pair_end = base + a_len + b_len;
  const int64_t o1 = o0 + TILE < pair_end ? o0 + TILE : pair_end;
  const SortItem* A = in + base;
  const SortItem* B = in + b0;
  const int warp = threadIdx.x >> 5;
  if (warp < 2) {
    const int64_t sp = WarpMergePathSplit(A, a_len, B, b_len, (warp == 0 ? o0 : o1) - base);
    if ((threadIdx.x & 31) == 0) split[warp] = sp;
  }
  __syncthreads();
  const int64_t ia = split[0], jb = o0 - base - split[0];
  const int na = static_cast<int>(split[1] - split[0]);
  const int cnt = static_cast<int>(o1 - o0);
  const int nb = cnt - na;
  for (int i = threadIdx.x; i < cnt; i += kThreads)
    s[Padded(i)] = i < na ? A[ia + i] : B[jb + i - na];
  __syncthreads();
  const int d = threadIdx.x * ITEMS;
  SortItem x[ITEMS];
  if (d < cnt) {
    auto at = [&](int i) -> const SortItem& { return s[Padded(i)]; };
    auto bt = [&](int j) -> const SortItem& { return s[Padded(na + j)]; };
    int i = MergePathSplit(at, na, bt, nb, d);
    int j = d - i;
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
      if (d + k < cnt) {
        const bool take_a = j >= nb || (i < na && ItemLess(at(i), bt(j)));
        x[k] = take_a ? at(i++) : bt(j++);
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < ITEMS; k++)
    if (d + k < cnt) s[Padded(d + k)] = x[k];
  __syncthreads();
  for (int i = threadIdx.x; i < cnt; i += kThreads) out[o0 + i] = s[Padded(i)];
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

namespace {
// lengths of a TEXT .kdb image's slots (validated on the host) into toff[r]
__global__ void KdbTextLengths(const char* __restrict__ raw, int64_t n, int64_t* __restrict__ toff) {
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int32_t len;
    memcpy(&len, raw + 8 + 16 * r, 4);
    toff[r] = len;
  }
}
// one warp per string: its bytes from the image to the column's byte array
__global__ void KdbTextGather(const char* __restrict__ raw, int64_t n, const int64_t* __restrict__ toff,
                              char* __restrict__ chars) {
  const int lane = threadIdx.x & 31;
  for (int64_t r = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5; r < n;
       r += (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5) {
    uint64_t o;
    memcpy(&o, raw + 8 + 16 * r + 8, 8);
    const int64_t b = toff[r], len = toff[r + 1] - b;
    for (int64_t i = lane; i < len; i += 32) chars[b + i] = raw[o + i];
  }
}
}  // namespace

namespace {
__global__ void SpinDelay(long long cycles) {
  const long long t0 = clock64();
  while (clock64() - t0 < cycles) {
  }
}
}  // namespace

void Context::DelayStream(double us) {
  if (dry || us <= 0) return;
  // SM clock cycles at up to 2 GHz; at most 2 ms
  const long long cycles = static_cast<long long>(std::min(us, 2000.0) * 2000.0);
  SpinDelay<<<1, 1, 0, stream>>>(cycles);
  KDB_CUDA(cudaGetLastError());
}

void Context::DecodeKdbText(const char* d_raw, int64_t n, int64_t* toff, char* tchars) {
  if (dry || n <= 0) return;
  TimedStart("text decode");
  KdbTextLengths<<<GridFor(n, 256), 256, 0, stream>>>(d_raw, n, toff);
  kernel_launches++;
  TimedStop();
  ScanU64(reinterpret_cast<uint64_t*>(toff), n, "text decode offsets");
  TimedStart("text decode");
  KdbTextGather<<<GridFor(n * 32, 256), 256, 0, stream>>>(d_raw, n, toff, tchars);
  kernel_launches++;
  TimedStop();
  KDB_CUDA(cudaGetLastError());
}

void Context::PackToHost(const PackSegs& segs, size_t total, void* host) {
  if (dry || segs.n == 0) return;
  uint64_t most = 0;
  for (int i = 0; i < segs.n; i++) most = std::max<uint64_t>(most, segs.seg[i].bytes);
  const int gx = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((most / 16 + 255) / 256, 64)));
  // A small result is gathered by the kernel straight into the pinned host
  // block (mapped into the device's address space): no device stage and no
  // copy to launch and wait for after the kernel.
  constexpr size_t kDirect = size_t(64) << 10;
  void* mapped = nullptr;
  // The lookup is skipped while an earlier error is pending, so that clearing
  // the lookup's own failure below can never swallow someone else's error.
  if (total <= kDirect && !OptStr("KDB_NO_MAPPED_RESULT") &&
      cudaPeekAtLastError() == cudaSuccess) {
    if (cudaHostGetDevicePointer(&mapped, host, 0) != cudaSuccess) {
      cudaGetLastError();
      mapped = nullptr;
    }
  }
  if (mapped) {
    PackSegments<<<dim3(gx, segs.n), 256, 0, stream>>>(segs, static_cast<char*>(mapped));
    kernel_launches++;
    KDB_CUDA(cudaGetLastError());
    return;
  }
  if (total > dev_stage_bytes_) {
    if (dev_stage_) cudaFreeAsync(dev_stage_, stream);
    dev_stage_bytes_ = std::max<size_t>(total, 1 << 20);
    KDB_CUDA(cudaMallocAsync(&dev_stage_, dev_stage_bytes_, stream));
  }
  char* dst = static_cast<char*>(dev_stage_);
  PackSegments<<<dim3(gx, segs.n), 256, 0, stream>>>(segs, dst);
  kernel_launches++;
  KDB_CUDA(cudaGetLastError());
  KDB_CUDA(cudaMemcpyAsync(host, dst, total, cudaMemcpyDeviceToHost, stream));
}

// Launch shapes of the two sort kernels: tile size and items per thread.
struct SortShape {
  int tile, items;
};

template <int TILE, int ITEMS>
void LaunchBlockSort(const SortItem* in, SortItem* out, int64_t n, cudaStream_t s) {
  const int dyn = TILE > 2048 ? static_cast<int>(sizeof(SortItem)) * PaddedTile<TILE>() : 0;
  // set once, on the first (uncaptured) launch; replays reuse the attribute
  static const bool attr = dyn == 0 || cudaFuncSetAttribute(BlockSortItems<TILE, ITEMS>,
                                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                           dyn) == cudaSuccess;
  (void)attr;
  BlockSortItems<TILE, ITEMS><<<static_cast<unsigned>((n + TILE - 1) / TILE), TILE / ITEMS, dyn, s>>>(in, out, n);
}
template <int TILE, int ITEMS>
void LaunchMerge(const SortItem* in, SortItem* out, int64_t n, int64_t w, cudaStream_t s) {
  MergeItems<TILE, ITEMS><<<static_cast<unsigned>((n + TILE - 1) / TILE), TILE / ITEMS, 0, s>>>(in, out, n, w);
}

// option KDB_SORT_SHAPE="bt,bi,mt,mi" overrides the shapes (tuning)
void SortShapes(const Context& ctx, SortShape* block, SortShape* merge) {
  // measured on the 134k-item ORDER BY of the Q3-shape query: smaller
  // merge tiles give a pass more blocks (latency-bound searches and staging)
  *block = {1024, 2};
  *merge = {256, 2};
  if (const char* e = ctx.OptStr("KDB_SORT_SHAPE")) {
    int v[4];
    if (std::sscanf(e, "%d,%d,%d,%d", &v[0], &v[1], &v[2], &v[3]) == 4) {
      *block = {v[0], v[1]};
      *merge = {v[2], v[3]};
    }
  }
}

// ---------------------------------------------------------------------------
// Sample sort of 16-byte items by (key, tie): splitters are quantiles of a
// strided sample (sorted in one block), one pass sends every item to its
// bucket, and one CTA per bucket sorts it in shared memory (bitonic) and
// writes it at the bucket's offset.  (key, tie) pairs are unique, so the
// buckets stay balanced whatever the key distribution; a bucket larger than
// kBucketCap makes the caller fall back to the merge sort.
// ---------------------------------------------------------------------------
namespace {

constexpr int kSampleOver = 8;       // samples per bucket
constexpr int kMaxBuckets = 1024;
constexpr int kBucketCap = 8192;     // items a bucket may hold (128 KiB of shared memory)

// (key, tie, val): the order of ItemLess, refined by the value so that the
// padding items (all ones; real values are rows below 2^31) sort last
__device__ __forceinline__ bool ItemLess3(const SortItem& a, const SortItem& b) {
  if (a.key != b.key) return a.key < b.key;
  if (a.tie != b.tie) return a.tie < b.tie;
  return a.val < b.val;
}

__device__ __forceinline__ void CmpSwap(SortItem* s, int i, int j, bool up) {
  SortItem a = s[i], b = s[j];
  if (ItemLess3(b, a) == up) {
    s[i] = b;
    s[j] = a;
  }
}

// bitonic sort of s[0..m) in shared memory, m a power of two
__device__ void BitonicSort(SortItem* s, int m) {
  for (int k = 2; k <= m; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int l = i ^ j;
        if (l > i) CmpSwap(s, i, l, (i & k) == 0);
      }
      __syncthreads();
    }
}

__device__ __forceinline__ SortItem MaxItem() {
  SortItem m;
  m.key = ~0ULL;
  m.tie = 0xffffffffu;
  m.val = 0xffffffffu;
  return m;
}

// one block: the strided sample, sorted; splitter j = sample[(j + 1) * over]
__global__ void SampleSplitters(const SortItem* __restrict__ items, int64_t n, int buckets,
                                SortItem* __restrict__ splitters) {
  extern __shared__ SortItem smp[];
  const int m = buckets * kSampleOver;  // a power of two
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const int64_t at = (static_cast<int64_t>(i) * n) / m;
    smp[i] = items[at];
  }
  __syncthreads();
  BitonicSort(smp, m);
  for (int j = threadIdx.x; j + 1 < buckets; j += blockDim.x) splitters[j] = smp[(j + 1) * kSampleOver];
}

__device__ __forceinline__ int BucketOf(const SortItem& x, const SortItem* spl, int buckets) {
  int lo = 0, hi = buckets - 1;  // first splitter greater than x, in [0, buckets - 1]
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ItemLess(x, spl[mid])) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

__global__ void SampleBucketCount(const SortItem* __restrict__ items, int64_t n, int buckets,
                                  const SortItem* __restrict__ splitters, uint16_t* __restrict__ bucket_of,
                                  unsigned* __restrict__ counts) {
  __shared__ SortItem spl[kMaxBuckets];
  __shared__ unsigned cnt[kMaxBuckets];
  for (int j = threadIdx.x; j < buckets; j += blockDim.x) {
    if (j + 1 < buckets) spl[j] = splitters[j];
    cnt[j] = 0;
  }
  __syncthreads();
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int b = BucketOf(items[i], spl, buckets);
    bucket_of[i] = static_cast<uint16_t>(b);
    atomicAdd(&cnt[b], 1u);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < buckets; j += blockDim.x)
    if (cnt[j]) atomicAdd(&counts[j], cnt[j]);
}

// one block: exclusive offsets of the bucket counts (offs[buckets] = n),
// cursors zeroed, the largest bucket into *largest
__global__ void SampleBucketOffsets(const unsigned* __restrict__ counts, int buckets, unsigned* __restrict__ offs,
                                    unsigned* __restrict__ cursor, unsigned* __restrict__ largest) {
  __shared__ unsigned s[kMaxBuckets];
  for (int j = threadIdx.x; j < buckets; j += blockDim.x) s[j] = counts[j];
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned run = 0, big = 0;
    for (int j = 0; j < buckets; j++) {
      const unsigned c = s[j];
      offs[j] = run;
      run += c;
      big = c > big ? c : big;
    }
    offs[buckets] = run;
    *largest = big;
  }
  for (int j = threadIdx.x; j < buckets; j += blockDim.x) cursor[j] = 0;
}

__global__ void SampleScatter(const SortItem* __restrict__ items, int64_t n, const uint16_t* __restrict__ bucket_of,
                              const unsigned* __restrict__ offs, unsigned* __restrict__ cursor,
                              SortItem* __restrict__ out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int b = bucket_of[i];
    out[offs[b] + atomicAdd(&cursor[b], 1u)] = items[i];
  }
}

// one block per bucket: sort it in shared memory, write it in place in dst
__global__ void SampleBucketSort(const SortItem* __restrict__ src, const unsigned* __restrict__ offs,
                                 SortItem* __restrict__ dst) {
  extern __shared__ SortItem sb[];
  const unsigned b0 = offs[blockIdx.x], cnt = offs[blockIdx.x + 1] - b0;
  if (cnt == 0) return;
  int m = 1;
  while (m < static_cast<int>(cnt)) m <<= 1;
  for (int i = threadIdx.x; i < m; i += blockDim.x) sb[i] = i < static_cast<int>(cnt) ? src[b0 + i] : MaxItem();
  __syncthreads();
  BitonicSort(sb, m);
  for (int i = threadIdx.x; i < static_cast<int>(cnt); i += blockDim.x) dst[b0 + i] = sb[i];
}

}  // namespace

// ---------------------------------------------------------------------------
// Range-bucket sort of 16-byte items by (key, tie): the keys' minimum and
// maximum split the key range into kRangeBuckets equal-width buckets (a
// bucket index never decreases with the key), one pass counts them, one
// block scans the counts, one pass scatters every item into its bucket's
// range, and then every item finds its final slot itself: its bucket's
// start plus the number of items in the same bucket that order before it.
// With many narrow buckets each item compares itself with a few dozen
// others, all in parallel (no per-bucket sort whose largest bucket sets the
// time).  Equal keys share a bucket, so many ties (or a very skewed range)
// make a bucket larger than kRangeBucketCap; the caller then uses the merge
// sort.
// ---------------------------------------------------------------------------
namespace {

constexpr int kRangeBuckets = 16384;
constexpr int kRangeThreads = 1024;
constexpr unsigned kRangeBucketCap = 1024;  // items one bucket may hold

__global__ void __launch_bounds__(kRangeThreads) RangeMinMax(const SortItem* __restrict__ items, int64_t n,
                                                             unsigned long long* __restrict__ mm) {
  __shared__ unsigned long long slo[kRangeThreads / 32], shi[kRangeThreads / 32];
  unsigned long long lo = ~0ULL, hi = 0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const unsigned long long k = items[i].key;
    lo = k < lo ? k : lo;
    hi = k > hi ? k : hi;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo, o), b = __shfl_xor_sync(0xffffffffu, hi, o);
    lo = a < lo ? a : lo;
    hi = b > hi ? b : hi;
  }
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    slo[warp] = lo;
    shi[warp] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < nw; w++) {
      lo = slo[w] < lo ? slo[w] : lo;
      hi = shi[w] > hi ? shi[w] : hi;
    }
    atomicMin(&mm[0], lo);
    atomicMax(&mm[1], hi);
  }
}

__device__ __forceinline__ unsigned RangeBucket(unsigned long long k, unsigned long long lo, unsigned long long range) {
  // (k - lo) / (range + 1) * B in doubles: rounding keeps it monotonic
  const double f = static_cast<double>(k - lo) / (static_cast<double>(range) + 1.0);
  const int b = static_cast<int>(f * kRangeBuckets);
  return b < 0 ? 0u : (b >= kRangeBuckets ? static_cast<unsigned>(kRangeBuckets - 1) : static_cast<unsigned>(b));
}

// bucket counts (global; few items per bucket, so the atomics rarely meet)
__global__ void RangeCount(const SortItem* __restrict__ items, int64_t n, const unsigned long long* __restrict__ mm,
                           uint16_t* __restrict__ bucket_of, unsigned* __restrict__ counts) {
  const unsigned long long lo = mm[0], range = mm[1] - mm[0];
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const unsigned b = RangeBucket(items[i].key, lo, range);
    bucket_of[i] = static_cast<uint16_t>(b);
    atomicAdd(&counts[b], 1u);
  }
}

// one block: exclusive bucket offsets (offs[B] = total), each bucket's
// cursor set to its offset, the largest bucket into *largest
__global__ void __launch_bounds__(kRangeThreads) RangeOffsets(const unsigned* __restrict__ counts,
                                                              unsigned* __restrict__ offs,
                                                              unsigned* __restrict__ cursor,
                                                              unsigned* __restrict__ largest) {
  constexpr int kPer = kRangeBuckets / kRangeThreads;
  __shared__ unsigned ws[32], wmax[32];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  static_assert(kPer % 4 == 0, "whole 16-byte vectors per thread");
  unsigned c[kPer], tot = 0, mx = 0;
  // a thread's buckets as 16-byte vectors (a warp reads 2 KiB contiguously)
#pragma unroll
  for (int q = 0; q < kPer / 4; q++) {
    const uint4 v = reinterpret_cast<const uint4*>(counts + t * kPer)[q];
    c[4 * q] = v.x;
    c[4 * q + 1] = v.y;
    c[4 * q + 2] = v.z;
    c[4 * q + 3] = v.w;
  }
#pragma unroll
  for (int q = 0; q < kPer; q++) {
    tot += c[q];
    mx = c[q] > mx ? c[q] : mx;
  }
  unsigned incl = tot;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
    const unsigned z = __shfl_xor_sync(0xffffffffu, mx, o);
    mx = z > mx ? z : mx;
  }
  if (lane == 31) ws[warp] = incl;
  if (lane == 0) wmax[warp] = mx;
  __syncthreads();
  if (warp == 0) {
    unsigned v = ws[lane], m = wmax[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
      const unsigned z = __shfl_xor_sync(0xffffffffu, m, o);
      m = z > m ? z : m;
    }
    ws[lane] = v;  // inclusive per warp
    if (lane == 0) *largest = m;
  }
  __syncthreads();
  unsigned run = (warp ? ws[warp - 1] : 0u) + incl - tot;
#pragma unroll
  for (int q = 0; q < kPer / 4; q++) {
    uint4 v;
    v.x = run;
    v.y = v.x + c[4 * q];
    v.z = v.y + c[4 * q + 1];
    v.w = v.z + c[4 * q + 2];
    run = v.w + c[4 * q + 3];
    reinterpret_cast<uint4*>(offs + t * kPer)[q] = v;
    reinterpret_cast<uint4*>(cursor + t * kPer)[q] = v;
  }
  if (t == kRangeThreads - 1) offs[kRangeBuckets] = run;
}

// every item into its bucket's range (in any order within the bucket)
__global__ void RangeScatter(const SortItem* __restrict__ items, int64_t n, const uint16_t* __restrict__ bucket_of,
                             unsigned* __restrict__ cursor, SortItem* __restrict__ out, uint16_t* __restrict__ out_bucket) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const unsigned b = bucket_of[i];
    const unsigned pos = atomicAdd(&cursor[b], 1u);
    out[pos] = items[i];
    out_bucket[pos] = static_cast<uint16_t>(b);
  }
}

// every item to its bucket's start plus the number of its bucket's items
// that order before it ((key, tie) pairs are unique: distinct slots).  With
// `ties`, an item whose key another item of its bucket shares (and, under
// `tie_mask`, the same masked tie bits) counts into *ties: equal keys always
// share a bucket, so this finds every tie of the sorted sequence.
__global__ void RangeRank(const SortItem* __restrict__ src, const uint16_t* __restrict__ bucket, int64_t n,
                          const unsigned* __restrict__ offs, SortItem* __restrict__ dst,
                          unsigned long long* __restrict__ ties, uint32_t tie_mask) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const SortItem x = src[i];
    const unsigned b = bucket[i], b0 = offs[b], b1 = offs[b + 1];
    unsigned r = b0;
    bool tie = false;
    for (unsigned j = b0; j < b1; j++) {
      const SortItem y = src[j];
      r += ItemLess(y, x) ? 1u : 0u;
      tie |= j != static_cast<unsigned>(i) && y.key == x.key && ((y.tie ^ x.tie) & tie_mask) == 0;
    }
    dst[r] = x;
    if (ties && tie) atomicAdd(ties, 1ULL);
  }
}

}  // namespace

bool Context::RangeSortItems(void* items_v, int64_t n, Arena& arena, unsigned long long* ties, uint32_t tie_mask,
                             const unsigned long long* key_range) {
  if (n <= 1 || dry) return true;
  if (n > 0x7fffffffLL) return false;
  SortItem* items = static_cast<SortItem*>(items_v);
  SortItem* tmp = reinterpret_cast<SortItem*>(arena.Alloc(sizeof(SortItem) * n));
  uint16_t* bof = reinterpret_cast<uint16_t*>(arena.Alloc(sizeof(uint16_t) * n));
  uint16_t* tbof = reinterpret_cast<uint16_t*>(arena.Alloc(sizeof(uint16_t) * n));
  unsigned long long* mm = key_range ? nullptr : arena.AllocT<unsigned long long>(2);
  const unsigned long long* range = key_range ? key_range : mm;
  unsigned* counts = arena.AllocT<unsigned>(kRangeBuckets);
  unsigned* offs = arena.AllocT<unsigned>(kRangeBuckets + 1);
  unsigned* cursor = arena.AllocT<unsigned>(kRangeBuckets);
  unsigned* largest = arena.AllocT<unsigned>(1);
  // a fallback to the merge sort drops these passes from the recording
  const auto mark = RecordMark();
  if (mm) {
    Memset(mm, 0xff, sizeof(unsigned long long));
    Memset(mm + 1, 0, sizeof(unsigned long long));
  }
  Memset(counts, 0, sizeof(unsigned) * kRangeBuckets);
  const int mm_grid = static_cast<int>(std::min<int64_t>((n + kRangeThreads - 1) / kRangeThreads, 32));
  const int grid = GridFor(n, 256);
  TimedStart("sort range");
  if (mm) Issue([=](cudaStream_t s) { RangeMinMax<<<mm_grid, kRangeThreads, 0, s>>>(items, n, mm); });
  Issue([=](cudaStream_t s) { RangeCount<<<grid, 256, 0, s>>>(items, n, range, bof, counts); });
  Issue([=](cudaStream_t s) { RangeOffsets<<<1, kRangeThreads, 0, s>>>(counts, offs, cursor, largest); });
  TimedStop();
  KDB_CUDA(cudaGetLastError());
  // the bucket sizes decide (at recording; a replay runs on the same data)
  unsigned big = 0;
  D2H(&big, largest, sizeof(big));
  if (big > kRangeBucketCap) {
    RecordTruncate(mark);
    return false;
  }
  TimedStart("sort buckets");
  Issue([=](cudaStream_t s) { RangeScatter<<<grid, 256, 0, s>>>(items, n, bof, cursor, tmp, tbof); });
  Issue([=](cudaStream_t s) { RangeRank<<<grid, 256, 0, s>>>(tmp, tbof, n, offs, items, ties, tie_mask); });
  TimedStop();
  KDB_CUDA(cudaGetLastError());
  return true;
}

bool Context::SampleSortItems(void* items_v, int64_t n, Arena& arena) {
  if (n <= 1 || dry) return true;
  if (n > 0x7fffffffLL) return false;
  // buckets: a power of two near n / 512, at most kMaxBuckets
  int buckets = 2;
  while (buckets < kMaxBuckets && static_cast<int64_t>(buckets) * 512 < n) buckets <<= 1;
  SortItem* items = static_cast<SortItem*>(items_v);
  SortItem* spl = reinterpret_cast<SortItem*>(arena.Alloc(sizeof(SortItem) * buckets));
  SortItem* tmp = reinterpret_cast<SortItem*>(arena.Alloc(sizeof(SortItem) * n));
  uint16_t* bof = reinterpret_cast<uint16_t*>(arena.Alloc(sizeof(uint16_t) * n));
  unsigned* counts = arena.AllocT<unsigned>(buckets);
  unsigned* offs = arena.AllocT<unsigned>(buckets + 1);
  unsigned* cursor = arena.AllocT<unsigned>(buckets);
  unsigned* largest = arena.AllocT<unsigned>(1);
  Memset(counts, 0, sizeof(unsigned) * buckets);
  const size_t smem_sample = sizeof(SortItem) * buckets * kSampleOver;
  const int grid = GridFor(n, 256);
  TimedStart("sort sample");
  if (smem_sample > 48 * 1024)
    KDB_CUDA(cudaFuncSetAttribute(SampleSplitters, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem_sample)));
  const int b = buckets;
  Issue([=](cudaStream_t s) { SampleSplitters<<<1, 1024, smem_sample, s>>>(items, n, b, spl); });
  Issue([=](cudaStream_t s) { SampleBucketCount<<<grid, 256, 0, s>>>(items, n, b, spl, bof, counts); });
  Issue([=](cudaStream_t s) { SampleBucketOffsets<<<1, 256, 0, s>>>(counts, b, offs, cursor, largest); });
  TimedStop();
  KDB_CUDA(cudaGetLastError());
  unsigned big = 0;
  D2H(&big, largest, sizeof(big));
  if (big > static_cast<unsigned>(kBucketCap)) return false;  // skewed sample: the merge sort takes it
  int m = 1;
  while (m < static_cast<int>(big)) m <<= 1;
  const size_t smem_bucket = sizeof(SortItem) * std::max(m, 1);
  TimedStart("sort buckets");
  Issue([=](cudaStream_t s) { SampleScatter<<<grid, 256, 0, s>>>(items, n, bof, offs, cursor, tmp); });
  if (smem_bucket > 48 * 1024)
    KDB_CUDA(cudaFuncSetAttribute(SampleBucketSort, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem_bucket)));
  Issue([=](cudaStream_t s) { SampleBucketSort<<<b, 512, smem_bucket, s>>>(tmp, offs, items); });
  TimedStop();
  KDB_CUDA(cudaGetLastError());
  return true;
}

void Context::MergeSortItems(void* items, int64_t n, Arena& arena) {
  if (n <= 1 || dry) return;
  if (n > 0x7fffffffLL) throw Error(-5, "merge sort of more than 2^31 items");
  SortShape bs, ms;
  SortShapes(*this, &bs, &ms);
  auto block_sort = [&]() -> void (*)(const SortItem*, SortItem*, int64_t, cudaStream_t) {
    switch (bs.tile * 16 + bs.items) {
      case 8192 * 16 + 8: return LaunchBlockSort<8192, 8>;
      case 4096 * 16 + 4: return LaunchBlockSort<4096, 4>;
      case 4096 * 16 + 8: return LaunchBlockSort<4096, 8>;
      case 2048 * 16 + 2: return LaunchBlockSort<2048, 2>;
      case 2048 * 16 + 4: return LaunchBlockSort<2048, 4>;
      case 2048 * 16 + 8: return LaunchBlockSort<2048, 8>;
      case 1024 * 16 + 2: return LaunchBlockSort<1024, 2>;
      case 1024 * 16 + 4: return LaunchBlockSort<1024, 4>;
      case 512 * 16 + 2: return LaunchBlockSort<512, 2>;
      default: throw Error(-5, "unsupported block sort shape");
    }
  }();
  auto merge = [&]() -> void (*)(const SortItem*, SortItem*, int64_t, int64_t, cudaStream_t) {
    switch (ms.tile * 16 + ms.items) {
      case 2048 * 16 + 8: return LaunchMerge<2048, 8>;
      case 2048 * 16 + 4: return LaunchMerge<2048, 4>;
      case 2048 * 16 + 2: return LaunchMerge<2048, 2>;
      case 1024 * 16 + 4: return LaunchMerge<1024, 4>;
      case 1024 * 16 + 8: return LaunchMerge<1024, 8>;
      case 512 * 16 + 4: return LaunchMerge<512, 4>;
      case 512 * 16 + 2: return LaunchMerge<512, 2>;
      case 256 * 16 + 2: return LaunchMerge<256, 2>;
      default: throw Error(-5, "unsupported merge shape");
    }
  }();
  // a merge tile must divide every run width
  if (ms.tile > bs.tile) throw Error(-5, "merge tile larger than the block sort tile");
  SortItem* a = static_cast<SortItem*>(items);
  SortItem* b = reinterpret_cast<SortItem*>(arena.Alloc(sizeof(SortItem) * n));
  int passes = 0;
  for (int64_t w = bs.tile; w < n; w <<= 1) passes++;
  // with an odd number of merge passes the block sort writes into the
  // scratch buffer, so that the last pass ends in `items` (no copy back)
  SortItem* src = a;
  SortItem* dst = passes % 2 ? b : a;
  TimedStart("sort block");
  Issue([=](cudaStream_t s) { block_sort(src, dst, n, s); });
  TimedStop();
  SortItem* cur = dst;
  SortItem* other = cur == a ? b : a;
  for (int64_t w = bs.tile; w < n; w <<= 1) {
    const SortItem* in = cur;
    SortItem* out = other;
    TimedStart("sort merge");
    Issue([=](cudaStream_t s) { merge(in, out, n, w, s); });
    TimedStop();
    std::swap(cur, other);
  }
  KDB_CUDA(cudaGetLastError());
}

void Context::ScanU64Bounded(uint64_t* a, const uint64_t* n_ptr, int64_t cap, const char* tag) {
  if (dry) return;
  TimedStart(tag);
  Issue([=](cudaStream_t s) { ExclusiveScanU64Bounded<<<1, 1024, 0, s>>>(a, n_ptr, cap); });
  TimedStop();
  KDB_CUDA(cudaGetLastError());
}

void Context::ScanU64(uint64_t* a, int64_t n, const char* tag) {
  if (dry) return;
  TimedStart(tag);
  Issue([=](cudaStream_t s) { ExclusiveScanU64<<<1, 1024, 0, s>>>(a, n); });
  TimedStop();
  KDB_CUDA(cudaGetLastError());
}

// Sorts (keys, vals) by the low `key_bits` bits of keys, stably.
void Context::RadixSortPairs(uint64_t* keys, uint32_t* vals, int64_t n, Arena& arena,
                             int key_bits) {
  if (n <= 1 || dry) return;
  if (n > 0xffffffffLL) throw Error(-5, "sort of more than 2^32 rows");
  if (n <= kSmallSort) {
    uint64_t mask = key_bits >= 64 ? ~0ULL : ((1ULL << key_bits) - 1);
    TimedStart("sort small");
    Issue([=](cudaStream_t s) { SmallRankSort<<<1, 1024, 0, s>>>(keys, vals, static_cast<int>(n), mask); });
    TimedStop();
    KDB_CUDA(cudaGetLastError());
    return;
  }
  // tiles small enough that every SM gets about two blocks, at most 4096
  // items (a multiple of the block size)
  int64_t tile = (n + 2 * num_sms - 1) / (2 * num_sms);
  tile = std::min<int64_t>(kSortTile, std::max<int64_t>(kSortBlock, (tile + kSortBlock - 1) / kSortBlock * kSortBlock));
  const int nblocks = static_cast<int>((n + tile - 1) / tile);
  const int itile = static_cast<int>(tile);
  uint64_t* k2 = arena.AllocT<uint64_t>(n);
  uint32_t* v2 = arena.AllocT<uint32_t>(n);
  uint32_t* hist = arena.AllocT<uint32_t>(static_cast<size_t>(nblocks) * 256);
  uint32_t* hist2 = arena.AllocT<uint32_t>(static_cast<size_t>(nblocks) * 256);
  uint32_t* totals = arena.AllocT<uint32_t>(256);
  uint64_t* ka = keys;
  uint32_t* va = vals;
  uint64_t* kb = k2;
  uint32_t* vb = v2;
  const int passes = (key_bits + 7) / 8;
  // skip passes whose digit is constant (one counting read of the keys)
  std::vector<bool> needed(passes, true);
  if (passes > 1 && n >= kPlanMinRows) {
    uint32_t* counts = arena.AllocT<uint32_t>(8 * 256);
    Memset(counts, 0, sizeof(uint32_t) * 8 * 256);
    TimedStart("sort digit counts");
    const int grid = GridFor(n, kSortBlock);
    Issue([=](cudaStream_t s) { RadixDigitCounts<<<grid, kSortBlock, 0, s>>>(ka, n, passes, counts); });
    TimedStop();
    std::vector<uint32_t> h(static_cast<size_t>(passes) * 256);
    D2H(h.data(), counts, sizeof(uint32_t) * h.size());
    for (int p = 0; p < passes; p++)
      for (int d = 0; d < 256; d++)
        if (h[p * 256 + d] == static_cast<uint64_t>(n)) needed[p] = false;
  }
  // Passes: one histogram launch for the first; each scatter counts the
  // next pass's histogram as it writes.
  std::vector<int> plist;
  for (int p = 0; p < passes; p++)
    if (needed[p]) plist.push_back(p);
  if (!plist.empty()) {
    const int shift0 = 8 * plist[0];
    TimedStart("sort histogram");
    Issue([=](cudaStream_t s) { RadixHistogram<<<nblocks, kSortBlock, 0, s>>>(ka, n, shift0, itile, hist, nblocks); });
    TimedStop();
  }
  uint32_t* cur = hist;
  uint32_t* other = hist2;
  for (size_t q = 0; q < plist.size(); q++) {
    const int shift = 8 * plist[q];
    const bool more = q + 1 < plist.size();
    const int next_shift = more ? 8 * plist[q + 1] : 0;
    uint32_t* next = more ? other : nullptr;
    TimedStart("sort scan");
    Issue([=](cudaStream_t s) { RadixRowScan<<<256, kSortBlock, 0, s>>>(cur, nblocks, totals, next); });
    TimedStop();
    TimedStart("sort scatter");
    Issue([=](cudaStream_t s) {
      RadixScatter<<<nblocks, kSortBlock, 0, s>>>(ka, va, kb, vb, n, shift, itile, cur, nblocks, totals, next,
                                                  next_shift);
    });
    TimedStop();
    std::swap(cur, other);
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  KDB_CUDA(cudaGetLastError());
  if (ka != keys) {
    TimedStart("sort copy");
    const int grid = GridFor(n, 256);
    Issue([=](cudaStream_t s) { CopyPairs<<<grid, 256, 0, s>>>(ka, va, keys, vals, n); });
    TimedStop();
    KDB_CUDA(cudaGetLastError());
  }
}

}  // namespace kdb

// ---------------------------------------------------------------------------
// Allocation-free sort entry point.
//
// Some callers cannot allocate device memory at the moment they need a sort:
// host callbacks and driver-owned threads where CUDA allocation calls are
// not allowed, and host engines that budget every byte
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
// per device, with that device current, through cudaGetSymbolAddress.  The
// cached address belongs to the device's primary context as it was at the
// first call: after cudaDeviceReset the module is loaded again and the cache
// would be stale, so resetting a device after this entry point has run on it
// is not supported.
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
  // An error already pending on this thread belongs to the caller's earlier
  // work: leave it in place and launch nothing, so the final check below
  // only ever reports (and clears) this call's own launch errors.
  if (cudaPeekAtLastError() != cudaSuccess) return KDB_ERR_CUDA;
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
    RadixHistogram<<<nblocks, kSortBlock, 0, s>>>(ka, n, shift, kSortTile, hist, nblocks);
    ExclusiveScanSmall<<<1, 1024, 0, s>>>(hist, static_cast<int64_t>(nblocks) * 256);
    RadixScatter<<<nblocks, kSortBlock, 0, s>>>(ka, va, kb, vb, n, shift, kSortTile, hist, nblocks, nullptr,
                                                nullptr, 0);
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != d_keys) {
    int grid = static_cast<int>(std::min<int64_t>((n + 255) / 256, 4096));
    CopyPairs<<<grid, 256, 0, s>>>(ka, va, d_keys, d_vals, n);
  }
  return cudaGetLastError() == cudaSuccess ? KDB_OK : KDB_ERR_CUDA;
}
