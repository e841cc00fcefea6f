// Per-operator entry points: hand-written sm_100a kernels behind the
// operator-granularity part of the C ABI (include/kdb_b200.h, "per-operator
// boundary").  They work on HBM-resident base columns and device selection
// vectors, one operator per call, the way the reference's generated code
// calls one runtime structure at a time:
//
//   kdb_hash_build / kdb_hash_probe   runtime::HashTable::{Create,Insert,
//                                      GetBucket} (runtime/hash_table.cc:13-67)
//                                      as driven by hash_join_translator.cc:
//                                      79-139 (NULL build keys skipped, every
//                                      duplicate kept, a probe row meets its
//                                      bucket's rows in build order)
//   kdb_agg_create/update/finalize    runtime::AggregateHashTable + the proxy
//                                      aggregators (aggregate_hash_table.cc:
//                                      187-333, aggregator.cc:28-296)
//   kdb_index_build / kdb_index_get   MemoryColumnIndex / ColumnIndex
//                                      (memory_column_index.cc:17-121,
//                                      column_index.cc:67-144)
//
// Hash join (kernel b).  A build side whose table fits comfortably in L2 is
// one open-addressing table probed straight from the probe column.  A larger
// build side is radix partitioned by the top bits of the key hash into P
// sub-tables of at most ~128 KiB each: both sides are scattered into
// partition order, then one CTA per partition copies its sub-table into
// shared memory with a TMA bulk copy (cp.async.bulk, completion on an
// mbarrier) and streams its probe tuples through shared memory in
// double-buffered bulk-copied tiles, so every probe is a shared-memory
// access instead of a random HBM sector.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "capi_internal.h"
#include "operators.h"

namespace cg = cooperative_groups;

namespace kdb {
namespace ops {
namespace {

constexpr int kBlock = 256;
constexpr int kPartBlock = 1024;                 // threads of a partitioned build / probe CTA
constexpr int kMaxPartBits = 13;                 // at most 8192 sub-tables
constexpr size_t kSmemTableMax = 128 << 10;      // a sub-table built in shared memory
constexpr size_t kTableBuf = 64 << 10;           // a probe-side sub-table buffer (two of them)
constexpr int kProbeTile = 2048;                 // probe tuples per bulk-copied tile
constexpr uint32_t kWaitLimit = 1u << 24;        // bounded mbarrier waits
constexpr int kErrWait = 1;                      // device error word: a wait gave up
constexpr int kErrFull = 2;                      // a table ran out of empty slots
constexpr unsigned kOutStage = 4096;             // pairs a partitioned-probe CTA stages
constexpr unsigned kFlatStage = 2048;            // pairs a flat-probe CTA stages
constexpr int kTupCap = 3072;                    // probe tuples per partition buffer (warp-level probe)
constexpr int kWarpStage = 64;                   // pairs a warp stages before one global append

// ---- keys --------------------------------------------------------------------
struct KeyCol {
  const void* data;
  const int8_t* nulls;
  int width;  // 1, 2, 4 or 8 bytes (signed)
};

__device__ __forceinline__ int64_t LoadKey(const KeyCol& c, int64_t r) {
  switch (c.width) {
    case 1: return static_cast<const int8_t*>(c.data)[r];
    case 2: return static_cast<const int16_t*>(c.data)[r];
    case 4: return static_cast<const int32_t*>(c.data)[r];
    default: return static_cast<const int64_t*>(c.data)[r];
  }
}

__device__ __forceinline__ bool KeyNull(const KeyCol& c, int64_t r) {
  return c.nulls != nullptr && c.nulls[r] != 0;
}

// murmur3's 32-bit finaliser over the 64-bit value folded to 32 bits: equal
// values of any integer width hash alike.
__host__ __device__ __forceinline__ uint32_t Hash32(uint64_t v) {
  uint32_t x = static_cast<uint32_t>(v) + static_cast<uint32_t>(v >> 32) * 0x9e3779b9u;
  x ^= x >> 16;
  x *= 0x85ebca6bu;
  x ^= x >> 13;
  x *= 0xc2b2ae35u;
  x ^= x >> 16;
  return x;
}

__device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }

__device__ __forceinline__ int64_t RowAt(const int32_t* sel, int64_t i) { return sel ? sel[i] : i; }

__device__ __forceinline__ uint32_t PartOf(uint32_t h, int bits) { return bits ? h >> (32 - bits) : 0u; }

// Table slots.  Keys of at most 32 bits share one 64-bit word with the row:
// {key << 32 | row + 1}, claimed with one CAS (0 = empty).  64-bit keys use
// a 16-byte slot {key, row + 1} whose row word is claimed first; the key is
// read only by probes, which run after the build has finished.
// Staged tuples (partition order) use the same layouts.
template <bool WIDE>
struct Slot;
template <>
struct Slot<false> {
  using T = unsigned long long;
  __device__ static T Make(int64_t key, int64_t row) {
    return (static_cast<T>(static_cast<uint32_t>(key)) << 32) | static_cast<T>(row + 1);
  }
  __device__ static int64_t Key(T s) { return static_cast<int32_t>(s >> 32); }
  __device__ static int64_t Row(T s) { return static_cast<int64_t>(s & 0xffffffffULL) - 1; }
  __device__ static bool Empty(T s) { return s == 0; }
  // claims slot `p` for `v` when it is empty
  __device__ static bool Claim(T* p, T v) { return atomicCAS(p, 0ULL, v) == 0ULL; }
};
template <>
struct Slot<true> {
  using T = ulonglong2;
  __device__ static T Make(int64_t key, int64_t row) {
    T s;
    s.x = static_cast<unsigned long long>(key);
    s.y = static_cast<unsigned long long>(row + 1);
    return s;
  }
  __device__ static int64_t Key(T s) { return static_cast<int64_t>(s.x); }
  __device__ static int64_t Row(T s) { return static_cast<int64_t>(s.y) - 1; }
  __device__ static bool Empty(T s) { return s.y == 0; }
  __device__ static bool Claim(T* p, T v) {
    if (atomicCAS(&p->y, 0ULL, v.y) != 0ULL) return false;
    p->x = v.x;
    return true;
  }
};

// ---- TMA bulk copies (1-D, global -> shared, completion on an mbarrier) -----
__device__ __forceinline__ uint32_t SmemAddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void BarInit(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(SmemAddr(bar)) : "memory");
}
// Orders this thread's generic-proxy accesses to shared memory before later
// async-proxy (bulk copy) accesses, and makes barrier inits visible to it.
__device__ __forceinline__ void FenceProxyAsync() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Issued by one thread: expects `bytes` on `bar` and starts the copy.
// dst, src and bytes are multiples of 16.
__device__ __forceinline__ void BulkLoad(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(SmemAddr(bar)), "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          SmemAddr(dst)),
      "l"(src), "r"(bytes), "r"(SmemAddr(bar))
      : "memory");
}
// Several copies completing on one barrier phase: one thread announces their
// total bytes (the phase's one arrival), then starts each copy.
__device__ __forceinline__ void BarExpect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(SmemAddr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void BulkCopy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          SmemAddr(dst)),
      "l"(src), "r"(bytes), "r"(SmemAddr(bar))
      : "memory");
}
// The same as several copies of at most `piece` bytes (a multiple of 16),
// all in flight together.
__device__ __forceinline__ void BulkCopyPieces(void* dst, const void* src, uint32_t bytes, uint64_t* bar,
                                               uint32_t piece) {
  for (uint32_t o = 0; o < bytes; o += piece)
    BulkCopy(static_cast<char*>(dst) + o, static_cast<const char*>(src) + o, bytes - o < piece ? bytes - o : piece,
             bar);
}

// Waits for phase `parity` of `bar` to complete; false when the wait gave up.
__device__ __forceinline__ bool BarWait(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < kWaitLimit; it++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(SmemAddr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Every thread of the block waits; the outcome is made block-uniform (one
// barrier), so a block either goes on together or leaves together.  A wait
// that gave up records the failure and waits once more (bounded), so that no
// copy this block issued is still writing its shared memory when it returns.
__device__ __forceinline__ bool BarWaitAll(uint64_t* bar, uint32_t parity, int* err) {
  const bool ok = BarWait(bar, parity);
  if (!__syncthreads_or(!ok)) return true;
  if (threadIdx.x == 0) {
    atomicOr(err, kErrWait);
    BarWait(bar, parity);
  }
  return false;
}

// ---- partitioning ----------------------------------------------------------
// Per-partition counts of the selected rows with non-NULL keys.
__global__ void PartHistogram(KeyCol key, const int32_t* __restrict__ sel, int64_t n, int bits,
                              unsigned* __restrict__ hist) {
  extern __shared__ unsigned sh_hist[];
  const int parts = 1 << bits;
  for (int i = threadIdx.x; i < parts; i += blockDim.x) sh_hist[i] = 0;
  __syncthreads();
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = RowAt(sel, i);
    if (KeyNull(key, r)) continue;
    atomicAdd(&sh_hist[PartOf(Hash32(static_cast<uint64_t>(LoadKey(key, r))), bits)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < parts; i += blockDim.x)
    if (sh_hist[i]) atomicAdd(&hist[i], sh_hist[i]);
}

// One block: partition p's staged tuples start at stage_off[p] (each
// partition padded to an even count, so every partition starts on a 16-byte
// boundary), its sub-table at slot_off[p] with a power-of-two capacity of at
// least count / load_factor and at least 16 slots (slot_off == nullptr: no
// tables, probe side).  Totals go to stage_off[P] / slot_off[P]; the scatter
// cursors are zeroed.
__global__ void PartOffsets(const unsigned* __restrict__ hist, int parts, double load_factor,
                            unsigned long long* __restrict__ stage_off, unsigned long long* __restrict__ slot_off,
                            unsigned* __restrict__ cursor) {
  __shared__ unsigned long long s_stage[1024], s_slot[1024];
  const int per = (parts + 1023) / 1024;
  unsigned long long my_stage = 0, my_slot = 0;
  for (int k = 0; k < per; k++) {
    const int p = threadIdx.x * per + k;
    if (p >= parts) break;
    const unsigned long long c = hist[p];
    my_stage += (c + 1) & ~1ULL;
    unsigned long long want = static_cast<unsigned long long>(ceil(static_cast<double>(c) / load_factor));
    unsigned long long cap = 16;
    while (cap < want + 1) cap <<= 1;
    my_slot += cap;
  }
  s_stage[threadIdx.x] = my_stage;
  s_slot[threadIdx.x] = my_slot;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {  // inclusive scan of the per-thread sums
    unsigned long long a = threadIdx.x >= d ? s_stage[threadIdx.x - d] : 0;
    unsigned long long b = threadIdx.x >= d ? s_slot[threadIdx.x - d] : 0;
    __syncthreads();
    s_stage[threadIdx.x] += a;
    s_slot[threadIdx.x] += b;
    __syncthreads();
  }
  unsigned long long st = threadIdx.x ? s_stage[threadIdx.x - 1] : 0;
  unsigned long long sl = threadIdx.x ? s_slot[threadIdx.x - 1] : 0;
  for (int k = 0; k < per; k++) {
    const int p = threadIdx.x * per + k;
    if (p >= parts) break;
    const unsigned long long c = hist[p];
    stage_off[p] = st;
    st += (c + 1) & ~1ULL;
    unsigned long long want = static_cast<unsigned long long>(ceil(static_cast<double>(c) / load_factor));
    unsigned long long cap = 16;
    while (cap < want + 1) cap <<= 1;
    if (slot_off) slot_off[p] = sl;
    sl += cap;
    cursor[p] = 0;
  }
  if (threadIdx.x == 1023) {
    stage_off[parts] = s_stage[1023];
    if (slot_off) slot_off[parts] = s_slot[1023];
  }
}

// Writes every selected row with a non-NULL key as a tuple at its
// partition's next staged position.
template <bool WIDE>
__global__ void PartScatter(KeyCol key, const int32_t* __restrict__ sel, int64_t n, int bits,
                            const unsigned long long* __restrict__ stage_off, unsigned* __restrict__ cursor,
                            typename Slot<WIDE>::T* __restrict__ staged) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = RowAt(sel, i);
    if (KeyNull(key, r)) continue;
    const int64_t k = LoadKey(key, r);
    const uint32_t p = PartOf(Hash32(static_cast<uint64_t>(k)), bits);
    const unsigned at = atomicAdd(&cursor[p], 1u);
    staged[stage_off[p] + at] = Slot<WIDE>::Make(k, r);
  }
}

// ---- build -------------------------------------------------------------------
// Inserts into table `tab` of capacity `cap` (a power of two) at the hash's
// low bits, linear probing; false when no empty slot was found.
template <bool WIDE>
__device__ __forceinline__ bool Insert(typename Slot<WIDE>::T* tab, uint64_t cap, uint32_t h,
                                       typename Slot<WIDE>::T v) {
  uint64_t i = h & (cap - 1);
  for (uint64_t step = 0; step < cap; step++) {
    if (Slot<WIDE>::Claim(&tab[i], v)) return true;
    i = (i + 1) & (cap - 1);
  }
  return false;
}

// One table: every selected row with a non-NULL key.
template <bool WIDE>
__global__ void BuildFlat(KeyCol key, const int32_t* __restrict__ sel, int64_t n,
                          typename Slot<WIDE>::T* __restrict__ tab, uint64_t cap, int* err) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = RowAt(sel, i);
    if (KeyNull(key, r)) continue;
    const int64_t k = LoadKey(key, r);
    if (!Insert<WIDE>(tab, cap, Hash32(static_cast<uint64_t>(k)), Slot<WIDE>::Make(k, r))) atomicOr(err, kErrFull);
  }
}

// Persistent CTAs, partitions p = blockIdx.x + i * gridDim.x (empty ones
// skipped: their slots are already zero).  A partition's staged tuples come
// into shared memory in bulk-copied tiles through a two-buffer ring that
// runs one tile ahead, across partition boundaries too; a sub-table that
// fits shared memory is built there with shared-memory CAS and written out
// with coalesced stores, a larger one is built in place in HBM.
template <bool WIDE>
__global__ void __launch_bounds__(kPartBlock) BuildParts(const typename Slot<WIDE>::T* __restrict__ staged,
                                                     const unsigned long long* __restrict__ stage_off,
                                                     const unsigned* __restrict__ hist,
                                                     const unsigned long long* __restrict__ slot_off, int parts,
                                                     typename Slot<WIDE>::T* __restrict__ slots, int* err) {
  using S = Slot<WIDE>;
  using T = typename S::T;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  T* tiles[2] = {reinterpret_cast<T*>(smem), reinterpret_cast<T*>(smem + kProbeTile * sizeof(T))};
  T* stab = reinterpret_cast<T*>(smem + 2 * kProbeTile * sizeof(T));
  if (threadIdx.x == 0) {
    for (int b = 0; b < 2; b++) BarInit(&bar[b]);
    FenceProxyAsync();
  }
  __syncthreads();
  uint32_t issued[2] = {0, 0}, waited[2] = {0, 0};
  auto next_part = [&](int q) {
    for (q += gridDim.x; q < parts && hist[q] == 0; q += gridDim.x) {
    }
    return q;
  };
  auto issue_tile = [&](int q, uint64_t t, int b) {
    const uint64_t count = hist[q], t0 = t * kProbeTile;
    const uint32_t n = static_cast<uint32_t>(umin64(kProbeTile, count - t0));
    FenceProxyAsync();
    BulkLoad(tiles[b], staged + stage_off[q] + t0, (n * sizeof(T) + 15) & ~15u, &bar[b]);
    issued[b]++;
  };
  int p = blockIdx.x;
  if (p < parts && hist[p] == 0) p = next_part(p);
  if (threadIdx.x == 0 && p < parts) issue_tile(p, 0, 0);
  bool failed = false;
  uint64_t j = 0;
  while (p < parts && !failed) {
    const uint64_t cap = slot_off[p + 1] - slot_off[p];
    T* gtab = slots + slot_off[p];
    const bool in_smem = cap * sizeof(T) <= kSmemTableMax;
    T* tab = in_smem ? stab : gtab;
    const uint64_t count = hist[p];
    const uint64_t ntiles = (count + kProbeTile - 1) / kProbeTile;
    const int np = next_part(p);
    if (in_smem) {
      // the previous partition's table was written out before the barrier
      // that ended it
      for (uint64_t i = threadIdx.x; i < cap; i += blockDim.x) tab[i] = T{};
      __syncthreads();
    }
    for (uint64_t t = 0; t < ntiles; t++) {
      const int b = static_cast<int>(j & 1);
      // tile j + 1 into the other buffer, whose reads ended at the barrier
      // that closed item j - 1
      if (threadIdx.x == 0) {
        if (t + 1 < ntiles) issue_tile(p, t + 1, b ^ 1);
        else if (np < parts) issue_tile(np, 0, b ^ 1);
      }
      if (!BarWaitAll(&bar[b], waited[b] & 1, err)) {
        failed = true;
        break;
      }
      waited[b]++;
      const uint32_t nt = static_cast<uint32_t>(umin64(kProbeTile, count - t * kProbeTile));
      for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) {
        const T v = tiles[b][i];
        const int64_t k = S::Key(v);
        if (!Insert<WIDE>(tab, cap, Hash32(static_cast<uint64_t>(k)), v)) atomicOr(err, kErrFull);
      }
      __syncthreads();
      j++;
    }
    if (in_smem && !failed)
      for (uint64_t i = threadIdx.x; i < cap; i += blockDim.x) gtab[i] = tab[i];
    __syncthreads();
    p = np;
  }
  if (failed && threadIdx.x == 0) {
    for (int b = 0; b < 2; b++)
      for (; waited[b] < issued[b]; waited[b]++) BarWait(&bar[b], waited[b] & 1);
  }
}

// ---- probe -------------------------------------------------------------------
// Output pairs go through a per-CTA shared-memory stage: a match takes a
// stage position (one shared-memory atomic per coalesced group) and the CTA
// appends the whole stage to the output with one global atomic.  A match
// that finds the stage full is appended on its own.
template <unsigned N>
struct OutStage {
  static constexpr unsigned kCap = N;
  unsigned long long buf[N];
  unsigned count;  // may pass N; positions from N on went direct
  unsigned long long base;
};

__device__ __forceinline__ unsigned long long PackPair(int64_t probe_row, int64_t build_row) {
  return (static_cast<unsigned long long>(probe_row) << 32) | static_cast<uint32_t>(build_row);
}

// Appends one pair straight to the output through a warp-aggregated counter.
__device__ __forceinline__ void EmitPair(unsigned long long* out, unsigned long long cap,
                                         unsigned long long* counter, unsigned long long v) {
  cg::coalesced_group g = cg::coalesced_threads();
  unsigned long long base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(counter, static_cast<unsigned long long>(g.size()));
  base = g.shfl(base, 0) + g.thread_rank();
  if (base < cap) out[base] = v;
}

template <typename Stage>
__device__ __forceinline__ void StagePair(Stage& st, unsigned long long* out, unsigned long long cap,
                                          unsigned long long* counter, unsigned long long v) {
  cg::coalesced_group g = cg::coalesced_threads();
  unsigned at = 0;
  if (g.thread_rank() == 0) at = atomicAdd(&st.count, g.size());
  at = g.shfl(at, 0) + g.thread_rank();
  if (at < Stage::kCap) st.buf[at] = v;
  else EmitPair(out, cap, counter, v);
}

// Every thread of the CTA calls it: the staged pairs are appended with one
// global atomic and the stage is emptied.
template <typename Stage>
__device__ __forceinline__ void FlushPairs(Stage& st, unsigned long long* out, unsigned long long cap,
                                           unsigned long long* counter) {
  __syncthreads();
  const unsigned n = st.count < Stage::kCap ? st.count : Stage::kCap;
  if (n > 0) {
    if (threadIdx.x == 0) st.base = atomicAdd(counter, static_cast<unsigned long long>(n));
    __syncthreads();
    const unsigned long long base = st.base;
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x)
      if (base + i < cap) out[base + i] = st.buf[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) st.count = 0;
  __syncthreads();
}

template <bool WIDE, typename Stage>
__device__ __forceinline__ void ProbeOne(const typename Slot<WIDE>::T* tab, uint64_t cap, int64_t k,
                                         int64_t probe_row, Stage& st, unsigned long long* out,
                                         unsigned long long out_cap, unsigned long long* counter) {
  using S = Slot<WIDE>;
  uint64_t i = Hash32(static_cast<uint64_t>(k)) & (cap - 1);
  for (uint64_t step = 0; step < cap; step++) {
    const typename S::T s = tab[i];
    if (S::Empty(s)) return;
    if (S::Key(s) == k) StagePair(st, out, out_cap, counter, PackPair(probe_row, S::Row(s)));
    i = (i + 1) & (cap - 1);
  }
}

// One table: every selected probe row looks its key up directly; the CTA
// appends its staged pairs whenever the stage is half full.
template <bool WIDE>
__global__ void __launch_bounds__(kBlock) ProbeFlat(KeyCol key, const int32_t* __restrict__ sel, int64_t n,
                                                    const typename Slot<WIDE>::T* __restrict__ tab, uint64_t cap,
                                                    unsigned long long* __restrict__ out,
                                                    unsigned long long out_cap, unsigned long long* counter) {
  __shared__ OutStage<kFlatStage> st;
  if (threadIdx.x == 0) st.count = 0;
  __syncthreads();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t b0 = blockIdx.x * static_cast<int64_t>(blockDim.x); b0 < n; b0 += stride) {
    const int64_t i = b0 + threadIdx.x;
    if (i < n) {
      const int64_t r = RowAt(sel, i);
      if (!KeyNull(key, r)) ProbeOne<WIDE>(tab, cap, LoadKey(key, r), r, st, out, out_cap, counter);
    }
    // every thread's matches of this round are staged before thread 0 looks
    if (__syncthreads_or(threadIdx.x == 0 && st.count >= kFlatStage / 2)) FlushPairs(st, out, out_cap, counter);
  }
  FlushPairs(st, out, out_cap, counter);
}

// Persistent CTAs, partitions p = blockIdx.x + i * gridDim.x.  A CTA's work
// is the sequence of its partitions' probe tiles (kProbeTile staged tuples
// each); thread 0 keeps one tile ahead in a two-buffer ring and, as a
// partition starts, the NEXT partition's sub-table loading into the other of
// two table buffers, so a partition's table copy overlaps the probing of the
// one before.  Sub-tables larger than a table buffer are probed in HBM.
template <bool WIDE>
__global__ void __launch_bounds__(kPartBlock) ProbeParts(const typename Slot<WIDE>::T* __restrict__ staged,
                                                     const unsigned long long* __restrict__ stage_off,
                                                     const unsigned* __restrict__ hist,
                                                     const typename Slot<WIDE>::T* __restrict__ slots,
                                                     const unsigned long long* __restrict__ slot_off, int parts,
                                                     unsigned long long* __restrict__ out,
                                                     unsigned long long out_cap, unsigned long long* counter,
                                                     int* err) {
  using S = Slot<WIDE>;
  using T = typename S::T;
  extern __shared__ __align__(128) unsigned char smem[];
  // barriers 0-1: tile ring; 2-3: table buffers
  __shared__ __align__(8) uint64_t bar[4];
  __shared__ OutStage<kOutStage> st;
  T* tiles[2] = {reinterpret_cast<T*>(smem), reinterpret_cast<T*>(smem + kProbeTile * sizeof(T))};
  T* tabs[2] = {reinterpret_cast<T*>(smem + 2 * kProbeTile * sizeof(T)),
                reinterpret_cast<T*>(smem + 2 * kProbeTile * sizeof(T) + kTableBuf)};
  if (threadIdx.x == 0) {
    for (int b = 0; b < 4; b++) BarInit(&bar[b]);
    st.count = 0;
    FenceProxyAsync();
  }
  __syncthreads();
  // copies issued / waited per barrier (thread 0 issues, every thread waits
  // in the same order, so `waited` is block-uniform)
  uint32_t issued[4] = {0, 0, 0, 0}, waited[4] = {0, 0, 0, 0};
  auto next_part = [&](int q) {
    for (q += gridDim.x; q < parts && hist[q] == 0; q += gridDim.x) {
    }
    return q;
  };
  auto tab_fits = [&](int q) { return (slot_off[q + 1] - slot_off[q]) * sizeof(T) <= kTableBuf; };
  auto issue_tile = [&](int q, uint64_t t, int b) {
    const uint64_t count = hist[q], t0 = t * kProbeTile;
    const uint32_t n = static_cast<uint32_t>(umin64(kProbeTile, count - t0));
    FenceProxyAsync();
    BulkLoad(tiles[b], staged + stage_off[q] + t0, (n * sizeof(T) + 15) & ~15u, &bar[b]);
    issued[b]++;
  };
  auto issue_tab = [&](int q, int b) {
    FenceProxyAsync();
    BulkLoad(tabs[b], slots + slot_off[q], static_cast<uint32_t>((slot_off[q + 1] - slot_off[q]) * sizeof(T)),
             &bar[2 + b]);
    issued[2 + b]++;
  };
  int p = blockIdx.x;
  if (p < parts && hist[p] == 0) p = next_part(p);
  if (threadIdx.x == 0 && p < parts) {
    if (tab_fits(p)) issue_tab(p, 0);
    issue_tile(p, 0, 0);
  }
  bool failed = false;
  uint64_t j = 0;  // items (tiles) so far
  int tb = 0;      // table buffer of the current partition
  while (p < parts && !failed) {
    const uint64_t cap = slot_off[p + 1] - slot_off[p];
    const uint64_t count = hist[p];
    const uint64_t ntiles = (count + kProbeTile - 1) / kProbeTile;
    const bool fits = tab_fits(p);
    const int np = next_part(p);
    for (uint64_t t = 0; t < ntiles; t++) {
      const int b = static_cast<int>(j & 1);
      if (threadIdx.x == 0) {
        if (t + 1 < ntiles) issue_tile(p, t + 1, b ^ 1);
        else if (np < parts) issue_tile(np, 0, b ^ 1);
        // the next fitting partition's buffer: the other one when this
        // partition holds one, else the free current one
        if (t == 0 && np < parts && tab_fits(np)) issue_tab(np, fits ? tb ^ 1 : tb);
      }
      if (t == 0 && fits) {
        if (!BarWaitAll(&bar[2 + tb], waited[2 + tb] & 1, err)) {
          failed = true;
          break;
        }
        waited[2 + tb]++;
      }
      if (!BarWaitAll(&bar[b], waited[b] & 1, err)) {
        failed = true;
        break;
      }
      waited[b]++;
      const T* tab = fits ? tabs[tb] : slots + slot_off[p];
      const uint32_t nt = static_cast<uint32_t>(umin64(kProbeTile, count - t * kProbeTile));
      for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) {
        const T v = tiles[b][i];
        ProbeOne<WIDE>(tab, cap, S::Key(v), S::Row(v), st, out, out_cap, counter);
      }
      // a barrier: this tile's (and at the partition's end its table's)
      // reads are done before those buffers are refilled; the staged pairs
      // go out once the stage is half full (a tile adds at most kProbeTile
      // pairs per distinct build key)
      if (__syncthreads_or(threadIdx.x == 0 && st.count >= kOutStage / 2)) FlushPairs(st, out, out_cap, counter);
      j++;
    }
    if (fits) tb ^= 1;
    p = np;
  }
  if (failed && threadIdx.x == 0) {
    // every copy still in flight into this CTA's shared memory lands (or
    // its bounded wait gives up) before the CTA leaves
    for (int b = 0; b < 4; b++)
      for (; waited[b] < issued[b]; waited[b]++) BarWait(&bar[b], waited[b] & 1);
  }
  FlushPairs(st, out, out_cap, counter);
}

// Partitioned probe with warp-level consumption (32-bit keys).  A CTA walks
// its partitions through two buffers, each holding a partition's sub-table
// (when it fits) and its probe tuples (up to kTupCap per copy): while one
// partition is probed the next one's copy is in flight.  Inside a
// partition the warps take their tuples without CTA barriers and stage
// their pairs per warp (one global atomic per flush); one CTA barrier per
// partition releases its buffer.
__global__ void __launch_bounds__(kPartBlock) ProbePartsW(const unsigned long long* __restrict__ staged,
                                                          const unsigned long long* __restrict__ stage_off,
                                                          const unsigned* __restrict__ hist,
                                                          const unsigned long long* __restrict__ slots,
                                                          const unsigned long long* __restrict__ slot_off, int parts,
                                                          unsigned long long* __restrict__ out,
                                                          unsigned long long out_cap, unsigned long long* counter,
                                                          int* err, uint32_t piece) {
  using S = Slot<false>;
  using T = S::T;
  constexpr size_t kBuf = kTableBuf + kTupCap * sizeof(T);
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ unsigned long long wst[kPartBlock / 32][kWarpStage];
  __shared__ unsigned wcount[kPartBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    for (int b = 0; b < 2; b++) BarInit(&bar[b]);
    FenceProxyAsync();
  }
  if (lane == 0) wcount[warp] = 0;
  __syncthreads();
  uint32_t issued[2] = {0, 0}, waited[2] = {0, 0};
  auto next_part = [&](int q) {
    for (q += gridDim.x; q < parts && hist[q] == 0; q += gridDim.x) {
    }
    return q;
  };
  auto tab_fits = [&](int q) { return (slot_off[q + 1] - slot_off[q]) * sizeof(T) <= kTableBuf; };
  // partition q's table (when it fits; only with the first chunk) and its
  // tuples from c0 on into buffer b
  auto issue = [&](int q, int b, uint64_t c0) {
    const uint64_t count = hist[q];
    const uint32_t n = static_cast<uint32_t>(umin64(kTupCap, count - c0));
    const uint32_t tb = (n * sizeof(T) + 15) & ~15u;
    const bool with_tab = c0 == 0 && tab_fits(q);
    const uint32_t ab = with_tab ? static_cast<uint32_t>((slot_off[q + 1] - slot_off[q]) * sizeof(T)) : 0u;
    unsigned char* base = smem + b * kBuf;
    FenceProxyAsync();
    BarExpect(&bar[b], ab + tb);
    if (with_tab) BulkCopyPieces(base, slots + slot_off[q], ab, &bar[b], piece);
    BulkCopyPieces(base + kTableBuf, staged + stage_off[q] + c0, tb, &bar[b], piece);
    issued[b]++;
  };
  auto warp_flush = [&]() {
    const unsigned n = wcount[warp] < kWarpStage ? wcount[warp] : kWarpStage;
    unsigned long long base = 0;
    if (lane == 0 && n) base = atomicAdd(counter, static_cast<unsigned long long>(n));
    base = __shfl_sync(0xffffffffu, base, 0);
    for (unsigned i = lane; i < n; i += 32)
      if (base + i < out_cap) out[base + i] = wst[warp][i];
    __syncwarp();
    if (lane == 0) wcount[warp] = 0;
    __syncwarp();
  };
  int p = blockIdx.x;
  if (p < parts && hist[p] == 0) p = next_part(p);
  int pn = p < parts ? next_part(p) : parts;  // the partition in the other buffer
  if (threadIdx.x == 0) {
    if (p < parts) issue(p, 0, 0);
    if (pn < parts) issue(pn, 1, 0);
  }
  bool failed = false;
  int b = 0;
  while (p < parts && !failed) {
    const uint64_t cap = slot_off[p + 1] - slot_off[p];
    const uint64_t count = hist[p];
    const T* tab = tab_fits(p) ? reinterpret_cast<const T*>(smem + b * kBuf) : slots + slot_off[p];
    const T* tup = reinterpret_cast<const T*>(smem + b * kBuf + kTableBuf);
    for (uint64_t c0 = 0; c0 < count && !failed; c0 += kTupCap) {
      if (c0 > 0) {
        // a partition beyond one buffer of tuples: the next chunk into the
        // same buffer once every warp is done with this one
        __syncthreads();
        if (threadIdx.x == 0) issue(p, b, c0);
      }
      if (!BarWaitAll(&bar[b], waited[b] & 1, err)) {
        failed = true;
        break;
      }
      waited[b]++;
      const uint32_t n = static_cast<uint32_t>(umin64(kTupCap, count - c0));
      for (uint32_t i0 = warp * 32; i0 < n; i0 += kPartBlock) {
        const uint32_t i = i0 + lane;
        if (i < n) {
          const T v = tup[i];
          const int64_t k = S::Key(v);
          uint64_t j = Hash32(static_cast<uint64_t>(k)) & (cap - 1);
          for (uint64_t step = 0; step < cap; step++) {
            const T e = tab[j];
            if (S::Empty(e)) break;
            if (S::Key(e) == k) {
              const unsigned long long pair = PackPair(S::Row(v), S::Row(e));
              cg::coalesced_group g = cg::coalesced_threads();
              unsigned at = 0;
              if (g.thread_rank() == 0) at = atomicAdd(&wcount[warp], g.size());
              at = g.shfl(at, 0) + g.thread_rank();
              if (at < static_cast<unsigned>(kWarpStage)) wst[warp][at] = pair;
              else EmitPair(out, out_cap, counter, pair);
            }
            j = (j + 1) & (cap - 1);
          }
        }
        __syncwarp();
        if (wcount[warp] >= kWarpStage / 2) warp_flush();
      }
    }
    if (failed) break;
    // buffer b is free once every warp is done with it
    __syncthreads();
    const int pnn = pn < parts ? next_part(pn) : parts;
    if (threadIdx.x == 0 && pnn < parts) issue(pnn, b, 0);
    p = pn;
    pn = pnn;
    b ^= 1;
  }
  if (failed && threadIdx.x == 0) {
    for (int k = 0; k < 2; k++)
      for (; waited[k] < issued[k]; waited[k]++) BarWait(&bar[k], waited[k] & 1);
  }
  __syncwarp();
  warp_flush();
}

__global__ void SplitPairs(const unsigned long long* __restrict__ pairs, int64_t n, int32_t* __restrict__ probe,
                           int32_t* __restrict__ build) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const unsigned long long v = pairs[i];
    probe[i] = static_cast<int32_t>(v >> 32);
    build[i] = static_cast<int32_t>(v & 0xffffffffULL);
  }
}

int KeyWidth(plan::TypeId t) {
  switch (t) {
    case plan::TypeId::BOOLEAN: return 1;
    case plan::TypeId::SMALLINT: return 2;
    case plan::TypeId::INT:
    case plan::TypeId::DATE:
    case plan::TypeId::ENUM: return 4;
    case plan::TypeId::BIGINT: return 8;
    default: return 0;
  }
}

KeyCol KeyOf(const DevColumn& c) {
  int w = KeyWidth(c.type.id);
  if (!w) throw Error(KDB_ERR_UNSUPPORTED, "hash keys must be integer, date, enum or boolean columns");
  return KeyCol{c.data, c.nulls, w};
}

void CheckErr(Context& c, int* d_err, const char* what) {
  int h = 0;
  c.D2H(&h, d_err, sizeof(int));
  if (h & kErrWait) throw Error(KDB_ERR_TIMEOUT, std::string(what) + ": a bounded device wait gave up");
  if (h & kErrFull) throw Error(KDB_ERR_CAPACITY, std::string(what) + ": hash table full");
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

SelVec::~SelVec() {
  if (ctx && rows) {
    cudaSetDevice(ctx->device);
    cudaFreeAsync(rows, ctx->stream);
  }
}

HashTable::~HashTable() {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (slots) cudaFreeAsync(slots, ctx->stream);
  if (slot_off) cudaFreeAsync(slot_off, ctx->stream);
}

static int64_t SelCount(const Context& c, const std::string& table, const SelVec* sel) {
  if (sel) {
    if (sel->table != table) throw Error(KDB_ERR_INVALID, "selection vector of table " + sel->table + " used on " + table);
    return sel->n;
  }
  auto it = c.tables.find(table);
  if (it == c.tables.end()) throw Error(KDB_ERR_INVALID, "unknown table " + table);
  return std::max<int64_t>(it->second.rows, 0);
}

// ---------------------------------------------------------------------------
// Sort of a table's rows by key columns (ORDER BY outside a plan): one
// stable radix sort of (order key, row) pairs per key column, from the last
// key to the first, each pass keyed by the column's value in the current
// row order.
// ---------------------------------------------------------------------------
namespace {

// The order key of row r: an unsigned 64-bit value whose order is the
// column's ORDER BY order ascending, NULL above every value; descending is
// its complement (NULL then first).
__global__ void SortKeyFill(const void* __restrict__ data, const int8_t* __restrict__ nulls, int kind,
                            const int32_t* __restrict__ rank, const uint32_t* __restrict__ perm, int64_t n,
                            bool desc, uint64_t* __restrict__ keys) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = perm[i];
    uint64_t k;
    if (nulls && nulls[r]) {
      k = ~0ULL;
    } else {
      switch (kind) {
        case 0: k = static_cast<uint64_t>(static_cast<const int8_t*>(data)[r] != 0); break;
        case 1: k = static_cast<uint64_t>(static_cast<int64_t>(static_cast<const int16_t*>(data)[r])) ^ (1ULL << 63); break;
        case 2: k = static_cast<uint64_t>(static_cast<int64_t>(static_cast<const int32_t*>(data)[r])) ^ (1ULL << 63); break;
        case 3: k = static_cast<uint64_t>(static_cast<const int64_t*>(data)[r]) ^ (1ULL << 63); break;
        case 4: {
          const uint64_t b = __double_as_longlong(static_cast<const double*>(data)[r]);
          k = (b >> 63) ? ~b : (b | (1ULL << 63));
          break;
        }
        default: k = static_cast<uint64_t>(rank[static_cast<const int32_t*>(data)[r]]); break;
      }
      // values stay below the NULL key
      if (k == ~0ULL) k = ~0ULL - 1;
    }
    keys[i] = desc ? ~k : k;
  }
}

__global__ void SortPermInit(const int32_t* __restrict__ sel, int64_t n, uint32_t* __restrict__ perm) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    perm[i] = static_cast<uint32_t>(sel ? sel[i] : i);
}

}  // namespace

std::unique_ptr<SelVec> SortRows(Context& c, const std::string& table, const std::vector<std::string>& keys,
                                 const std::vector<bool>& asc, const SelVec* sel) {
  if (c.dry) throw Error(KDB_ERR_UNSUPPORTED, "operators need a device context");
  if (keys.empty() || keys.size() != asc.size()) throw Error(KDB_ERR_INVALID, "one direction per sort key");
  const int64_t n = SelCount(c, table, sel);
  if (n >= (int64_t(1) << 32)) throw Error(KDB_ERR_UNSUPPORTED, "sort of 2^32 rows or more");
  struct KeyCol {
    const DevColumn* col;
    int kind;
  };
  std::vector<KeyCol> kc;
  for (const auto& k : keys) {
    const DevColumn& col = c.Column(table, k);
    int kind;
    switch (col.type.id) {
      case plan::TypeId::BOOLEAN: kind = 0; break;
      case plan::TypeId::SMALLINT: kind = 1; break;
      case plan::TypeId::INT:
      case plan::TypeId::DATE: kind = 2; break;
      case plan::TypeId::BIGINT: kind = 3; break;
      case plan::TypeId::REAL: kind = 4; break;
      case plan::TypeId::ENUM: kind = 5; break;
      default: throw Error(KDB_ERR_UNSUPPORTED, "sort keys must be integer, date, boolean, enum or real columns");
    }
    kc.push_back({&col, kind});
  }
  auto out = std::make_unique<SelVec>();
  out->ctx = &c;
  out->table = table;
  out->n = n;
  KDB_CUDA(cudaMallocAsync(&out->rows, sizeof(int32_t) * std::max<int64_t>(n, 1), c.stream));
  if (n == 0) return out;
  Arena arena(c);
  uint64_t* kbuf = arena.AllocT<uint64_t>(n);
  const int grid = c.GridFor(n, kBlock);
  uint32_t* perm = reinterpret_cast<uint32_t*>(out->rows);
  c.TimedStart("sort rows");
  SortPermInit<<<grid, kBlock, 0, c.stream>>>(sel ? sel->rows : nullptr, n, perm);
  c.kernel_launches++;
  c.TimedStop();
  for (size_t j = keys.size(); j-- > 0;) {
    const DevColumn& col = *kc[j].col;
    const int32_t* rank = kc[j].kind == 5 ? c.Enum(col.type.enum_id).d_rank : nullptr;
    c.TimedStart("sort rows");
    SortKeyFill<<<grid, kBlock, 0, c.stream>>>(col.data, col.nulls, kc[j].kind, rank, perm, n, !asc[j], kbuf);
    c.kernel_launches++;
    c.TimedStop();
    KDB_CUDA(cudaGetLastError());
    // stable: rows with equal keys keep the order of the previous pass
    c.RadixSortPairs(kbuf, perm, n, arena, 64);
  }
  KDB_CUDA(cudaStreamSynchronize(c.stream));
  return out;
}


int PartBitsFor(int64_t n, double lf, int slot_bytes, int32_t fanout) {
  if (fanout == 1) return 0;
  if (fanout > 1) {
    int b = 0;
    while ((1 << b) < fanout) b++;
    if ((1 << b) != fanout || b > kMaxPartBits)
      throw Error(KDB_ERR_INVALID, "fanout must be a power of two of at most 8192");
    return b;
  }
  // automatic: one table while it stays well inside L2 (126 MB), otherwise
  // sub-tables of about 64 KiB (a shared-memory copy per partition)
  double table_bytes = static_cast<double>(n) / lf * 1.5 * slot_bytes;
  if (table_bytes <= 48.0 * (1 << 20)) return 0;
  int b = 0;
  while (b < kMaxPartBits && table_bytes / (1 << b) > 64.0 * 1024) b++;
  return b;
}

std::unique_ptr<HashTable> HashBuild(Context& c, const std::string& table, const std::string& key_column,
                                     const SelVec* sel, double load_factor, int32_t fanout) {
  if (!(load_factor > 0.05 && load_factor <= 0.95)) throw Error(KDB_ERR_INVALID, "load factor must be in (0.05, 0.95]");
  if (c.dry) throw Error(KDB_ERR_UNSUPPORTED, "operators need a device context");
  const DevColumn& col = c.Column(table, key_column);
  const KeyCol key = KeyOf(col);
  const int64_t n = SelCount(c, table, sel);
  const int32_t* srows = sel ? sel->rows : nullptr;
  auto ht = std::make_unique<HashTable>();
  ht->ctx = &c;
  ht->table = table;
  ht->key_type = col.type.id;
  ht->wide = key.width == 8;
  const int slot_bytes = ht->wide ? 16 : 8;
  ht->bits = PartBitsFor(n, load_factor, slot_bytes, fanout);
  const int parts = 1 << ht->bits;
  Arena arena(c);
  int* err = arena.AllocT<int>(1);
  c.Memset(err, 0, sizeof(int));
  const int grid = c.GridFor(std::max<int64_t>(n, 1), kBlock);
  if (ht->bits == 0) {
    uint64_t cap = 16;
    while (static_cast<double>(cap) * load_factor < static_cast<double>(n) + 1) cap <<= 1;
    ht->slots = c.DevAlloc(cap * slot_bytes);
    std::vector<unsigned long long> off = {0, cap};
    ht->slot_off = static_cast<unsigned long long*>(c.DevAlloc(sizeof(off[0]) * 2));
    KDB_CUDA(cudaMemcpyAsync(ht->slot_off, off.data(), sizeof(off[0]) * 2, cudaMemcpyHostToDevice, c.stream));
    c.Memset(ht->slots, 0, cap * slot_bytes);
    ht->total_slots = cap;
    c.TimedStart("hash build");
    if (n > 0) {
      if (ht->wide)
        BuildFlat<true><<<grid, kBlock, 0, c.stream>>>(key, srows, n, static_cast<ulonglong2*>(ht->slots), cap, err);
      else
        BuildFlat<false><<<grid, kBlock, 0, c.stream>>>(key, srows, n, static_cast<unsigned long long*>(ht->slots),
                                                        cap, err);
      c.kernel_launches++;
    }
    c.TimedStop();
  } else {
    unsigned* hist = arena.AllocT<unsigned>(parts);
    unsigned* cursor = arena.AllocT<unsigned>(parts);
    unsigned long long* stage_off = arena.AllocT<unsigned long long>(parts + 1);
    ht->slot_off = static_cast<unsigned long long*>(c.DevAlloc(sizeof(unsigned long long) * (parts + 1)));
    c.Memset(hist, 0, sizeof(unsigned) * parts);
    c.TimedStart("hash partition");
    PartHistogram<<<grid, kBlock, sizeof(unsigned) * parts, c.stream>>>(key, srows, n, ht->bits, hist);
    PartOffsets<<<1, 1024, 0, c.stream>>>(hist, parts, load_factor, stage_off, ht->slot_off, cursor);
    c.kernel_launches += 2;
    c.TimedStop();
    unsigned long long totals[2];
    KDB_CUDA(cudaMemcpyAsync(&totals[0], stage_off + parts, 8, cudaMemcpyDeviceToHost, c.stream));
    KDB_CUDA(cudaMemcpyAsync(&totals[1], ht->slot_off + parts, 8, cudaMemcpyDeviceToHost, c.stream));
    KDB_CUDA(cudaStreamSynchronize(c.stream));
    ht->total_slots = static_cast<int64_t>(totals[1]);
    ht->slots = c.DevAlloc(totals[1] * slot_bytes);
    // sub-tables too large for shared memory are built in place in HBM
    c.Memset(ht->slots, 0, totals[1] * slot_bytes);
    void* staged = arena.Alloc(std::max<unsigned long long>(totals[0], 2) * slot_bytes);
    c.TimedStart("hash scatter");
    if (ht->wide)
      PartScatter<true><<<grid, kBlock, 0, c.stream>>>(key, srows, n, ht->bits, stage_off, cursor,
                                                      static_cast<ulonglong2*>(staged));
    else
      PartScatter<false><<<grid, kBlock, 0, c.stream>>>(key, srows, n, ht->bits, stage_off, cursor,
                                                       static_cast<unsigned long long*>(staged));
    c.kernel_launches++;
    c.TimedStop();
    c.TimedStart("hash build");
    const size_t smem = 2 * kProbeTile * slot_bytes + kSmemTableMax;
    const int pgrid = std::min(parts, c.num_sms * 1);
    if (ht->wide) {
      KDB_CUDA(cudaFuncSetAttribute(BuildParts<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
      BuildParts<true><<<pgrid, kPartBlock, smem, c.stream>>>(static_cast<const ulonglong2*>(staged), stage_off, hist,
                                                          ht->slot_off, parts, static_cast<ulonglong2*>(ht->slots), err);
    } else {
      KDB_CUDA(cudaFuncSetAttribute(BuildParts<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
      BuildParts<false><<<pgrid, kPartBlock, smem, c.stream>>>(static_cast<const unsigned long long*>(staged), stage_off,
                                                           hist, ht->slot_off, parts,
                                                           static_cast<unsigned long long*>(ht->slots), err);
    }
    c.kernel_launches++;
    c.TimedStop();
  }
  KDB_CUDA(cudaGetLastError());
  CheckErr(c, err, "hash build");
  ht->bytes = static_cast<size_t>(ht->total_slots) * slot_bytes;
  return ht;
}

std::unique_ptr<Pairs> HashProbe(Context& c, const HashTable& ht, const std::string& table,
                                 const std::string& key_column, const SelVec* sel, bool ordered) {
  const DevColumn& col = c.Column(table, key_column);
  const KeyCol key = KeyOf(col);
  if ((key.width == 8) != ht.wide)
    throw Error(KDB_ERR_INVALID, "probe key width differs from the build key's (BIGINT against a narrower key)");
  const int64_t n = SelCount(c, table, sel);
  const int32_t* srows = sel ? sel->rows : nullptr;
  const int parts = 1 << ht.bits;
  const int slot_bytes = ht.wide ? 16 : 8;
  Arena arena(c);
  int* err = arena.AllocT<int>(1);
  unsigned long long* counter = arena.AllocT<unsigned long long>(1);
  const int grid = c.GridFor(std::max<int64_t>(n, 1), kBlock);
  // staged probe side (partitioned tables only)
  unsigned* hist = nullptr;
  unsigned long long* stage_off = nullptr;
  void* staged = nullptr;
  if (ht.bits > 0 && n > 0) {
    hist = arena.AllocT<unsigned>(parts);
    unsigned* cursor = arena.AllocT<unsigned>(parts);
    stage_off = arena.AllocT<unsigned long long>(parts + 1);
    staged = arena.Alloc((static_cast<size_t>(n) + parts + 2) * slot_bytes);
    c.Memset(hist, 0, sizeof(unsigned) * parts);
    c.TimedStart("probe partition");
    PartHistogram<<<grid, kBlock, sizeof(unsigned) * parts, c.stream>>>(key, srows, n, ht.bits, hist);
    PartOffsets<<<1, 1024, 0, c.stream>>>(hist, parts, 0.5, stage_off, nullptr, cursor);
    if (ht.wide)
      PartScatter<true><<<grid, kBlock, 0, c.stream>>>(key, srows, n, ht.bits, stage_off, cursor,
                                                      static_cast<ulonglong2*>(staged));
    else
      PartScatter<false><<<grid, kBlock, 0, c.stream>>>(key, srows, n, ht.bits, stage_off, cursor,
                                                       static_cast<unsigned long long*>(staged));
    c.kernel_launches += 3;
    c.TimedStop();
  }
  // matches: a first guess of one pair per probe row, the exact count after
  // an overflowing attempt
  unsigned long long cap = static_cast<unsigned long long>(std::max<int64_t>(n, 1024));
  auto pr = std::make_unique<Pairs>();
  pr->ctx = &c;
  for (int attempt = 0; attempt < 2; attempt++) {
    unsigned long long* out = static_cast<unsigned long long*>(arena.Alloc(cap * sizeof(unsigned long long)));
    c.Memset(err, 0, sizeof(int));
    c.Memset(counter, 0, sizeof(unsigned long long));
    c.TimedStart("hash probe");
    if (n > 0) {
      if (ht.bits == 0) {
        const uint64_t tcap = static_cast<uint64_t>(ht.total_slots);
        if (ht.wide)
          ProbeFlat<true><<<grid, kBlock, 0, c.stream>>>(key, srows, n, static_cast<const ulonglong2*>(ht.slots), tcap,
                                                         out, cap, counter);
        else
          ProbeFlat<false><<<grid, kBlock, 0, c.stream>>>(key, srows, n,
                                                          static_cast<const unsigned long long*>(ht.slots), tcap, out,
                                                          cap, counter);
      } else {
        const size_t smem = 2 * kProbeTile * slot_bytes + 2 * kTableBuf;
        const int pgrid = std::min(parts, c.num_sms);
        if (!ht.wide && !c.OptStr("KDB_PROBE_PARTS_TILED")) {
          const size_t wsmem = 2 * (kTableBuf + kTupCap * sizeof(unsigned long long));
          // KDB_TMA_PIECE: bytes per bulk copy (a partition's table and
          // tuples go as several copies in flight together)
          const char* pe = c.OptStr("KDB_TMA_PIECE");
          const uint32_t piece = pe ? static_cast<uint32_t>(std::max(16, std::atoi(pe)) & ~15) : 4096u;
          KDB_CUDA(cudaFuncSetAttribute(ProbePartsW, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(wsmem)));
          ProbePartsW<<<pgrid, kPartBlock, wsmem, c.stream>>>(static_cast<const unsigned long long*>(staged), stage_off,
                                                             hist, static_cast<const unsigned long long*>(ht.slots),
                                                             ht.slot_off, parts, out, cap, counter, err,
                                                             piece);
        } else if (ht.wide) {
          KDB_CUDA(cudaFuncSetAttribute(ProbeParts<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(smem)));
          ProbeParts<true><<<pgrid, kPartBlock, smem, c.stream>>>(static_cast<const ulonglong2*>(staged), stage_off, hist,
                                                              static_cast<const ulonglong2*>(ht.slots), ht.slot_off,
                                                              parts, out, cap, counter, err);
        } else {
          KDB_CUDA(cudaFuncSetAttribute(ProbeParts<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(smem)));
          ProbeParts<false><<<pgrid, kPartBlock, smem, c.stream>>>(
              static_cast<const unsigned long long*>(staged), stage_off, hist,
              static_cast<const unsigned long long*>(ht.slots), ht.slot_off, parts, out, cap, counter, err);
        }
      }
      c.kernel_launches++;
    }
    c.TimedStop();
    KDB_CUDA(cudaGetLastError());
    unsigned long long total = 0;
    c.D2H(&total, counter, sizeof(total));
    CheckErr(c, err, "hash probe");
    if (total <= cap) {
      pr->n = static_cast<int64_t>(total);
      if (ordered && total > 1) {
        // (probe row, build row) ascending: the reference's order, where a
        // probe row meets its bucket's rows in the order they were inserted
        uint32_t* dummy = arena.AllocT<uint32_t>(total);
        c.RadixSortPairs(reinterpret_cast<uint64_t*>(out), dummy, static_cast<int64_t>(total), arena, 64);
      }
      pr->probe = static_cast<int32_t*>(c.DevAlloc(sizeof(int32_t) * std::max<unsigned long long>(total, 1)));
      pr->build = static_cast<int32_t*>(c.DevAlloc(sizeof(int32_t) * std::max<unsigned long long>(total, 1)));
      if (total > 0) {
        SplitPairs<<<c.GridFor(static_cast<int64_t>(total), kBlock), kBlock, 0, c.stream>>>(
            out, static_cast<int64_t>(total), pr->probe, pr->build);
        c.kernel_launches++;
      }
      KDB_CUDA(cudaStreamSynchronize(c.stream));
      return pr;
    }
    cap = total;
  }
  throw Error(KDB_ERR_CAPACITY, "probe output did not converge");
}

Pairs::~Pairs() {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (probe) cudaFree(probe);
  if (build) cudaFree(build);
}


// ---------------------------------------------------------------------------
// Group-by aggregation (kernel c): runtime::AggregateHashTable with the proxy
// aggregators' results (compile/proxy/aggregate_hash_table.cc:187-333,
// compile/proxy/aggregator.cc:28-296).
//
// Global state: a table of slots {hash32 << 32 | group id + 1} over dense
// per-group arrays (key values and NULL flags, one state word and one
// non-NULL count per aggregate, the group's first stream position).  A
// group id is handed out once by the thread that claims the slot; it
// publishes the keys, then the slot, and threads meeting a claimed slot of
// the same hash wait (bounded) for that publication before comparing keys.
//
// Pre-aggregation: every CTA keeps the aggregate states of the groups its
// rows hit in a shared-memory table keyed by group id (shared-memory
// atomics), and adds them to the global states once, when its rows are
// done; a row whose group finds no room there updates the global state
// directly.  With skewed keys the hot groups' updates therefore stay inside
// the SM instead of serialising on global FP64 atomics.
// ---------------------------------------------------------------------------
namespace {

constexpr int kMaxAggKeys = 4;
constexpr int kMaxAggs = 8;
constexpr int kLocalGroups = 512;   // shared-memory pre-aggregation entries per CTA
constexpr int kLocalProbes = 16;
constexpr uint32_t kLocked = 0xffffffffu;  // slot claimed, group not yet published
constexpr uint32_t kDead = 0xfffffffeu;    // slot claimed when the group arrays were full

struct AggCols {
  const void* kd[kMaxAggKeys];
  const int8_t* kn[kMaxAggKeys];
  int kw[kMaxAggKeys];
  int nkeys;
  const void* md[kMaxAggs];  // nullptr: COUNT(*)
  const int8_t* mn[kMaxAggs];
  int mw[kMaxAggs];
  int mreal[kMaxAggs];
  int op[kMaxAggs];  // plan::AggType
  int naggs;
};

struct AggDev {
  unsigned long long* slots;
  unsigned long long cap;  // power of two
  int64_t* keys;           // [nkeys][G]
  int8_t* knull;           // [nkeys][G]
  unsigned long long* val;  // [naggs][G]
  unsigned long long* cnt;  // [naggs][G]
  unsigned long long* first;  // [G]: stream position << 8 | first row's measure-NULL bits
  unsigned long long* ngroups;
  int64_t G;  // group capacity
  int* err;
};

__device__ __forceinline__ uint64_t Mix64(uint64_t x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ULL;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebULL;
  x ^= x >> 31;
  return x;
}

__device__ __forceinline__ int64_t LoadInt(const void* d, int w, int64_t r) {
  switch (w) {
    case 1: return static_cast<const int8_t*>(d)[r];
    case 2: return static_cast<const int16_t*>(d)[r];
    case 4: return static_cast<const int32_t*>(d)[r];
    default: return static_cast<const int64_t*>(d)[r];
  }
}

// order-preserving encodings for MIN / MAX through unsigned atomics
__device__ __forceinline__ unsigned long long OrdI(int64_t v) {
  return static_cast<unsigned long long>(v) ^ (1ULL << 63);
}
__device__ __forceinline__ unsigned long long OrdF(double d) {
  unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(d));
  return (b >> 63) ? ~b : (b | (1ULL << 63));
}
__host__ __device__ inline double UnOrdF(unsigned long long k) {
  unsigned long long b = (k >> 63) ? (k & ~(1ULL << 63)) : ~k;
  double d;
  memcpy(&d, &b, 8);
  return d;
}

// Finds or inserts the group of key (kv, kn); returns its id, -1 when the
// table or the group arrays are full or a wait gave up (error word set).
__device__ int64_t FindGroup(const AggDev& a, int nkeys, const int64_t* kv, const bool* kn, uint32_t h32) {
  uint64_t i = (static_cast<uint64_t>(h32) * 0x9e3779b97f4a7c15ULL >> 20) & (a.cap - 1);
  for (uint64_t step = 0; step < a.cap; step++) {
    unsigned long long s = *reinterpret_cast<volatile unsigned long long*>(&a.slots[i]);
    if (s == 0) {
      const unsigned long long lock = (static_cast<unsigned long long>(h32) << 32) | kLocked;
      s = atomicCAS(&a.slots[i], 0ULL, lock);
      if (s == 0) {
        const unsigned long long g = atomicAdd(a.ngroups, 1ULL);
        if (static_cast<int64_t>(g) >= a.G) {
          // no group id left: the slot is marked so that its waiters stop
          atomicExch(&a.slots[i], (static_cast<unsigned long long>(h32) << 32) | kDead);
          atomicOr(a.err, kErrFull);
          return -1;
        }
        for (int k = 0; k < nkeys; k++) {
          a.keys[k * a.G + g] = kv[k];
          a.knull[k * a.G + g] = kn[k] ? 1 : 0;
        }
        __threadfence();
        atomicExch(&a.slots[i], (static_cast<unsigned long long>(h32) << 32) | (g + 1));
        return static_cast<int64_t>(g);
      }
    }
    if (static_cast<uint32_t>(s >> 32) == h32) {
      uint32_t it = 0;
      while (static_cast<uint32_t>(s) == kLocked && it++ < kWaitLimit)
        s = *reinterpret_cast<volatile unsigned long long*>(&a.slots[i]);
      if (static_cast<uint32_t>(s) == kLocked) {
        atomicOr(a.err, kErrWait);
        return -1;
      }
      if (static_cast<uint32_t>(s) == kDead) {
        atomicOr(a.err, kErrFull);
        return -1;
      }
      __threadfence();
      const int64_t g = static_cast<int64_t>(s & 0xffffffffULL) - 1;
      bool eq = true;
      for (int k = 0; k < nkeys && eq; k++) {
        const bool gn = *reinterpret_cast<volatile int8_t*>(&a.knull[k * a.G + g]) != 0;
        const int64_t gv = *reinterpret_cast<volatile int64_t*>(&a.keys[k * a.G + g]);
        eq = gn == kn[k] && (gn || gv == kv[k]);
      }
      if (eq) return g;
    }
    i = (i + 1) & (a.cap - 1);
  }
  atomicOr(a.err, kErrFull);
  return -1;
}

// One aggregate's update with one non-NULL input value (the state word's
// meaning follows the aggregate: f64 or i64 sum, ordered MIN/MAX key).
__device__ __forceinline__ void UpdateState(unsigned long long* v, int op, bool real, double f, int64_t i) {
  switch (op) {
    case static_cast<int>(plan::AggType::SUM):
    case static_cast<int>(plan::AggType::AVG):
      if (real) atomicAdd(reinterpret_cast<double*>(v), f);
      else if (op == static_cast<int>(plan::AggType::AVG)) atomicAdd(reinterpret_cast<double*>(v), static_cast<double>(i));
      else atomicAdd(v, static_cast<unsigned long long>(i));
      break;
    case static_cast<int>(plan::AggType::MIN): atomicMin(v, real ? OrdF(f) : OrdI(i)); break;
    case static_cast<int>(plan::AggType::MAX): atomicMax(v, real ? OrdF(f) : OrdI(i)); break;
    default: break;
  }
}

// Merges a partial state (pre-aggregated) into another state word.
__device__ __forceinline__ void MergeState(unsigned long long* v, int op, bool real, unsigned long long part) {
  switch (op) {
    case static_cast<int>(plan::AggType::SUM):
    case static_cast<int>(plan::AggType::AVG):
      if (real || op == static_cast<int>(plan::AggType::AVG))
        atomicAdd(reinterpret_cast<double*>(v), __longlong_as_double(static_cast<long long>(part)));
      else atomicAdd(v, part);
      break;
    case static_cast<int>(plan::AggType::MIN): atomicMin(v, part); break;
    case static_cast<int>(plan::AggType::MAX): atomicMax(v, part); break;
    default: break;
  }
}

__host__ __device__ inline unsigned long long StateInit(int op) {
  return op == static_cast<int>(plan::AggType::MIN) ? ~0ULL : 0ULL;
}

__global__ void AggInitStates(AggDev a, AggCols c) {
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < a.G;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    for (int k = 0; k < c.naggs; k++) {
      a.val[k * a.G + g] = StateInit(c.op[k]);
      a.cnt[k * a.G + g] = 0;
    }
    a.first[g] = ~0ULL;
  }
}

__global__ void __launch_bounds__(kBlock) AggUpdate(AggDev a, AggCols c, const int32_t* __restrict__ sel,
                                                    int64_t n, unsigned long long pos_base, int use_local) {
  // shared memory (dynamic, sized for the table's aggregates):
  // lfirst[L] u64, lval[naggs][L] u64, lcnt[naggs][L] u32, lg[L] i32
  extern __shared__ __align__(16) unsigned char agg_smem[];
  unsigned long long* lfirst = reinterpret_cast<unsigned long long*>(agg_smem);
  unsigned long long* lval = lfirst + kLocalGroups;
  unsigned* lcnt = reinterpret_cast<unsigned*>(lval + c.naggs * kLocalGroups);
  int32_t* lg = reinterpret_cast<int32_t*>(lcnt + c.naggs * kLocalGroups);
  for (int i = threadIdx.x; use_local && i < kLocalGroups; i += blockDim.x) {
    lg[i] = -1;
    lfirst[i] = ~0ULL;
    for (int k = 0; k < c.naggs; k++) {
      lval[k * kLocalGroups + i] = StateInit(c.op[k]);
      lcnt[k * kLocalGroups + i] = 0;
    }
  }
  __syncthreads();
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = RowAt(sel, i);
    int64_t kv[kMaxAggKeys];
    bool kn[kMaxAggKeys];
    uint64_t h = 0x243f6a8885a308d3ULL;
    for (int k = 0; k < c.nkeys; k++) {
      kn[k] = c.kn[k] != nullptr && c.kn[k][r] != 0;
      kv[k] = kn[k] ? 0 : LoadInt(c.kd[k], c.kw[k], r);
      h = Mix64(h ^ (kn[k] ? 0x5bd1e9955bd1e995ULL : static_cast<uint64_t>(kv[k])) + k);
    }
    const int64_t g = FindGroup(a, c.nkeys, kv, kn, static_cast<uint32_t>(h >> 32) | 1u);
    if (g < 0) continue;
    // the measures, and the first row's NULL flags (COUNT counts the
    // group's first row whether or not it is NULL, aggregator.cc:285-287)
    unsigned long long nullbits = 0;
    double fv[kMaxAggs];
    int64_t iv[kMaxAggs];
    for (int k = 0; k < c.naggs; k++) {
      const bool isnull = c.md[k] != nullptr && c.mn[k] != nullptr && c.mn[k][r] != 0;
      nullbits |= static_cast<unsigned long long>(isnull) << k;
      fv[k] = 0;
      iv[k] = 0;
      if (c.md[k] && !isnull) {
        if (c.mreal[k]) fv[k] = static_cast<const double*>(c.md[k])[r];
        else iv[k] = LoadInt(c.md[k], c.mw[k], r);
      }
    }
    const unsigned long long first = ((pos_base + static_cast<unsigned long long>(r)) << 8) | nullbits;
    // a shared-memory entry for the group, else the global state
    int slot = -1;
    if (use_local) {
      uint32_t j = static_cast<uint32_t>(Mix64(static_cast<uint64_t>(g)) >> 40) & (kLocalGroups - 1);
      for (int t = 0; t < kLocalProbes; t++) {
        int cur = lg[j];
        if (cur == -1) cur = atomicCAS(&lg[j], -1, static_cast<int>(g));
        if (cur == -1 || cur == g) {
          slot = static_cast<int>(j);
          break;
        }
        j = (j + 1) & (kLocalGroups - 1);
      }
    }
    if (slot >= 0) {
      atomicMin(&lfirst[slot], first);
      for (int k = 0; k < c.naggs; k++) {
        if ((nullbits >> k) & 1) continue;
        UpdateState(&lval[k * kLocalGroups + slot], c.op[k], c.mreal[k], fv[k], iv[k]);
        atomicAdd(&lcnt[k * kLocalGroups + slot], 1u);
      }
    } else {
      atomicMin(&a.first[g], first);
      for (int k = 0; k < c.naggs; k++) {
        if ((nullbits >> k) & 1) continue;
        UpdateState(&a.val[k * a.G + g], c.op[k], c.mreal[k], fv[k], iv[k]);
        atomicAdd(&a.cnt[k * a.G + g], 1ULL);
      }
    }
  }
  if (!use_local) return;
  __syncthreads();
  for (int j = threadIdx.x; j < kLocalGroups; j += blockDim.x) {
    const int g = lg[j];
    if (g < 0) continue;
    atomicMin(&a.first[g], lfirst[j]);
    for (int k = 0; k < c.naggs; k++) {
      const unsigned lc = lcnt[k * kLocalGroups + j];
      if (lc == 0) continue;
      MergeState(&a.val[k * a.G + g], c.op[k], c.mreal[k], lval[k * kLocalGroups + j]);
      atomicAdd(&a.cnt[k * a.G + g], static_cast<unsigned long long>(lc));
    }
  }
}

}  // namespace

static AggCols ColsOf(Context& c, const AggTable& t) {
  const auto& keys = t.keys;
  const auto& aggs = t.aggs;
  const auto& table = t.table;
  AggCols cols{};
  cols.nkeys = static_cast<int>(keys.size());
  for (int k = 0; k < cols.nkeys; k++) {
    const DevColumn& col = c.Column(table, keys[k]);
    cols.kd[k] = col.data;
    cols.kn[k] = col.nulls;
    cols.kw[k] = KeyWidth(col.type.id);
  }
  cols.naggs = static_cast<int>(aggs.size());
  for (int k = 0; k < cols.naggs; k++) {
    cols.op[k] = aggs[k].op;
    if (aggs[k].column.empty()) continue;
    const DevColumn& col = c.Column(table, aggs[k].column);
    cols.md[k] = col.data;
    cols.mn[k] = col.nulls;
    cols.mw[k] = plan::TypeWidth(col.type.id);
    cols.mreal[k] = col.type.id == plan::TypeId::REAL;
  }
  return cols;
}

AggTable::~AggTable() {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  for (void* p : bufs) cudaFree(p);
}

std::unique_ptr<AggTable> AggCreate(Context& c, const std::string& table, const std::vector<std::string>& keys,
                                    const std::vector<AggSpec>& aggs, int64_t max_groups) {
  if (c.dry) throw Error(KDB_ERR_UNSUPPORTED, "operators need a device context");
  if (keys.empty() || keys.size() > kMaxAggKeys) throw Error(KDB_ERR_INVALID, "1 to 4 group keys");
  if (aggs.empty() || aggs.size() > kMaxAggs) throw Error(KDB_ERR_INVALID, "1 to 8 aggregates");
  auto t = std::make_unique<AggTable>();
  t->ctx = &c;
  t->table = table;
  t->keys = keys;
  t->aggs = aggs;
  auto it = c.tables.find(table);
  if (it == c.tables.end()) throw Error(KDB_ERR_INVALID, "unknown table " + table);
  const int64_t rows = std::max<int64_t>(it->second.rows, 0);
  for (const auto& k : keys) {
    const DevColumn& col = c.Column(table, k);
    if (!KeyWidth(col.type.id)) throw Error(KDB_ERR_UNSUPPORTED, "group keys must be integer, date, enum or boolean columns");
    t->key_types.push_back(col.type);
  }
  for (const auto& a : aggs) {
    if (a.op < 0 || a.op > static_cast<int>(plan::AggType::COUNT)) throw Error(KDB_ERR_INVALID, "bad aggregate");
    if (a.column.empty()) {
      if (a.op != static_cast<int>(plan::AggType::COUNT))
        throw Error(KDB_ERR_INVALID, "only COUNT may omit its column");
      t->agg_types.push_back(plan::Type{plan::TypeId::INT, 0});
      continue;
    }
    const DevColumn& col = c.Column(table, a.column);
    if (col.type.id == plan::TypeId::TEXT) throw Error(KDB_ERR_UNSUPPORTED, "TEXT measures go through query plans");
    if (col.type.id == plan::TypeId::BOOLEAN && a.op != static_cast<int>(plan::AggType::COUNT))
      throw Error(KDB_ERR_UNSUPPORTED, "BOOLEAN measures only under COUNT");
    if (col.type.id == plan::TypeId::ENUM &&
        (a.op == static_cast<int>(plan::AggType::MIN) || a.op == static_cast<int>(plan::AggType::MAX)))
      throw Error(KDB_ERR_UNSUPPORTED, "ENUM MIN/MAX go through query plans");
    t->agg_types.push_back(col.type);
  }
  t->G = std::max<int64_t>(1, max_groups > 0 ? std::min(max_groups, std::max<int64_t>(rows, 1)) : std::max<int64_t>(rows, 1));
  uint64_t cap = 16;
  while (cap < static_cast<uint64_t>(t->G) * 2) cap <<= 1;
  t->cap = cap;
  auto alloc = [&](size_t bytes) {
    void* p = c.DevAlloc(std::max<size_t>(bytes, 16));
    t->bufs.push_back(p);
    return p;
  };
  const int64_t G = t->G;
  const size_t nk = keys.size(), na = aggs.size();
  t->slots = static_cast<unsigned long long*>(alloc(cap * 8));
  t->keyv = static_cast<int64_t*>(alloc(nk * G * 8));
  t->knull = static_cast<int8_t*>(alloc(nk * G));
  t->val = static_cast<unsigned long long*>(alloc(na * G * 8));
  t->cnt = static_cast<unsigned long long*>(alloc(na * G * 8));
  t->first = static_cast<unsigned long long*>(alloc(G * 8));
  t->ngroups = static_cast<unsigned long long*>(alloc(8));
  t->err = static_cast<int*>(alloc(16));
  c.Memset(t->slots, 0, cap * 8);
  c.Memset(t->ngroups, 0, 8);
  c.Memset(t->err, 0, 16);
  AggDev a{t->slots, cap, t->keyv, t->knull, t->val, t->cnt, t->first, t->ngroups, G, t->err};
  AggCols cols = ColsOf(c, *t);
  AggInitStates<<<c.GridFor(G, kBlock), kBlock, 0, c.stream>>>(a, cols);
  c.kernel_launches++;
  KDB_CUDA(cudaGetLastError());
  return t;
}

void AggUpdateRows(Context& c, AggTable& t, const SelVec* sel, bool pre_aggregate) {
  const int64_t n = SelCount(c, t.table, sel);
  AggDev a{t.slots, t.cap, t.keyv, t.knull, t.val, t.cnt, t.first, t.ngroups, t.G, t.err};
  AggCols cols = ColsOf(c, t);
  // positions of later updates follow the earlier ones' (the reference's
  // insertion order across morsels)
  const unsigned long long pos_base = static_cast<unsigned long long>(t.updates) << 34;
  if (t.updates >= (1 << 21)) throw Error(KDB_ERR_CAPACITY, "too many updates of one aggregate table");
  t.updates++;
  if (n > 0) {
    c.TimedStart("agg update");
    const size_t smem = pre_aggregate ? kLocalGroups * (8 + 4 + cols.naggs * (8 + 4)) : 0;
    if (smem > 48 * 1024)
      KDB_CUDA(cudaFuncSetAttribute(AggUpdate, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    AggUpdate<<<c.GridFor(n, kBlock), kBlock, smem, c.stream>>>(a, cols, sel ? sel->rows : nullptr, n, pos_base,
                                                               pre_aggregate ? 1 : 0);
    c.kernel_launches++;
    c.TimedStop();
  }
  KDB_CUDA(cudaGetLastError());
  CheckErr(c, t.err, "aggregate update");
}

HostResult AggFinalize(Context& c, AggTable& t) {
  unsigned long long ng = 0;
  c.D2H(&ng, t.ngroups, 8);
  CheckErr(c, t.err, "aggregate finalize");
  const int64_t G = t.G, n = static_cast<int64_t>(std::min<unsigned long long>(ng, G));
  const size_t nk = t.keys.size(), na = t.aggs.size();
  std::vector<int64_t> keyv(nk * n);
  std::vector<int8_t> knull(nk * n);
  std::vector<unsigned long long> val(na * n), cnt(na * n), first(n);
  for (size_t k = 0; k < nk; k++) {
    KDB_CUDA(cudaMemcpyAsync(keyv.data() + k * n, t.keyv + k * G, 8 * n, cudaMemcpyDeviceToHost, c.stream));
    KDB_CUDA(cudaMemcpyAsync(knull.data() + k * n, t.knull + k * G, n, cudaMemcpyDeviceToHost, c.stream));
  }
  for (size_t k = 0; k < na; k++) {
    KDB_CUDA(cudaMemcpyAsync(val.data() + k * n, t.val + k * G, 8 * n, cudaMemcpyDeviceToHost, c.stream));
    KDB_CUDA(cudaMemcpyAsync(cnt.data() + k * n, t.cnt + k * G, 8 * n, cudaMemcpyDeviceToHost, c.stream));
  }
  KDB_CUDA(cudaMemcpyAsync(first.data(), t.first, 8 * n, cudaMemcpyDeviceToHost, c.stream));
  KDB_CUDA(cudaStreamSynchronize(c.stream));
  // groups in first-insertion order (the reference's ForEach order over its
  // payload blocks, aggregate_hash_table.cc:245-291)
  std::vector<int64_t> order(n);
  for (int64_t g = 0; g < n; g++) order[g] = g;
  std::sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return (first[x] >> 8) < (first[y] >> 8); });
  HostResult r;
  r.rows = n;
  for (size_t k = 0; k < nk; k++) {
    HostColumn hc;
    hc.name = t.keys[k];
    hc.type = t.key_types[k];
    hc.i.resize(n);
    hc.null.resize(n);
    for (int64_t j = 0; j < n; j++) {
      hc.i[j] = keyv[k * n + order[j]];
      hc.null[j] = knull[k * n + order[j]];
    }
    r.cols.push_back(std::move(hc));
  }
  for (size_t k = 0; k < na; k++) {
    const int op = t.aggs[k].op;
    const plan::Type in = t.agg_types[k];
    const bool real = in.id == plan::TypeId::REAL;
    HostColumn hc;
    hc.name = "agg" + std::to_string(k);
    if (op == static_cast<int>(plan::AggType::COUNT)) hc.type = plan::Type{plan::TypeId::BIGINT, 0};
    else if (op == static_cast<int>(plan::AggType::AVG)) hc.type = plan::Type{plan::TypeId::REAL, 0};
    else hc.type = in;
    const bool out_real = hc.type.id == plan::TypeId::REAL;
    if (out_real) hc.f.resize(n);
    else hc.i.resize(n);
    hc.null.assign(n, 0);
    for (int64_t j = 0; j < n; j++) {
      const int64_t g = order[j];
      const unsigned long long v = val[k * n + g], nn = cnt[k * n + g];
      if (op == static_cast<int>(plan::AggType::COUNT)) {
        // COUNT(*) counts rows; COUNT(col) counts non-NULL values plus the
        // group's first row when that one was NULL
        const bool first_null = (first[g] >> k) & 1;
        hc.i[j] = static_cast<int64_t>(nn) + (t.aggs[k].column.empty() ? 0 : (first_null ? 1 : 0));
        continue;
      }
      if (nn == 0) {
        hc.null[j] = 1;
        if (out_real) hc.f[j] = 0;
        else hc.i[j] = 0;
        continue;
      }
      double d;
      switch (op) {
        case static_cast<int>(plan::AggType::AVG):
          std::memcpy(&d, &v, 8);
          hc.f[j] = d / static_cast<double>(nn);
          break;
        case static_cast<int>(plan::AggType::SUM):
          if (real) {
            std::memcpy(&d, &v, 8);
            hc.f[j] = d;
          } else {
            // typed wrap-around at the column's width, as the reference's
            // sequential adds in that type
            int64_t s = static_cast<int64_t>(v);
            switch (plan::TypeWidth(in.id)) {
              case 2: s = static_cast<int16_t>(s); break;
              case 4: s = static_cast<int32_t>(s); break;
              default: break;
            }
            hc.i[j] = s;
          }
          break;
        default:  // MIN / MAX
          if (real) hc.f[j] = UnOrdF(v);
          else hc.i[j] = static_cast<int64_t>(v ^ (1ULL << 63));
          break;
      }
    }
    r.cols.push_back(std::move(hc));
  }
  return r;
}


namespace {
__global__ void GatherTilesKernel(const int32_t* __restrict__ scratch, const uint64_t* __restrict__ off,
                                  int64_t ntiles, int32_t* __restrict__ out) {
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint64_t o = off[t], cnt = off[t + 1] - o;
    for (uint64_t i = threadIdx.x; i < cnt; i += blockDim.x) out[o + i] = scratch[t * 1024 + i];
  }
}
}  // namespace

void GatherTiles(Context& c, const int32_t* scratch, const uint64_t* off, int64_t ntiles, int32_t* out) {
  if (ntiles <= 0) return;
  const int grid = static_cast<int>(std::min<int64_t>(ntiles, c.num_sms * 8));
  c.TimedStart("scan select gather");
  GatherTilesKernel<<<grid, 256, 0, c.stream>>>(scratch, off, ntiles, out);
  c.kernel_launches++;
  c.TimedStop();
  KDB_CUDA(cudaGetLastError());
}


// ---------------------------------------------------------------------------
// Column index (kdb_index_*): key -> ascending row ids, the posting lists of
// runtime::MemoryColumnIndex / runtime::ColumnIndex (memory_column_index.cc:
// 17-121, column_index.cc:67-144).  Device layout: distinct keys in
// ascending order, run starts (keys + 1 entries) and the rows of all runs.
// A build sorts (key, row) pairs stably by key on the device; the reference's
// .kdbindex files are read into the same layout.  The distinct keys and run
// starts are mirrored on the host for lookups by key.
// ---------------------------------------------------------------------------
namespace {

// Row ids of the rows with a non-NULL key, in row order: each 1024-row tile
// compacts its rows in order (per-thread counts of 4 rows, warp shuffle scan,
// block scan of the warp totals) into its own scratch region.
__global__ void CompactNonNull(const int8_t* __restrict__ nulls, int64_t n, int32_t* __restrict__ scratch,
                               uint64_t* __restrict__ counts) {
  __shared__ unsigned wsum[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t tile = blockIdx.x; tile * 1024 < n; tile += gridDim.x) {
    const int64_t base = tile * 1024 + threadIdx.x * 4;
    bool f[4];
    unsigned mine = 0;
    for (int u = 0; u < 4; u++) {
      f[u] = base + u < n && nulls[base + u] == 0;
      mine += f[u];
    }
    unsigned incl = mine;
    for (int d = 1; d < 32; d <<= 1) {
      unsigned y = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    unsigned before = 0, total = 0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); w++) {
      const unsigned x = wsum[w];
      if (w < warp) before += x;
      total += x;
    }
    unsigned at = before + incl - mine;
    for (int u = 0; u < 4; u++)
      if (f[u]) scratch[tile * 1024 + at++] = static_cast<int32_t>(base + u);
    if (threadIdx.x == 0) counts[tile] = total;
    __syncthreads();
  }
}

// (ordered key, row) of the listed rows (all rows when `list` is null)
__global__ void IndexPairs(KeyCol key, const int32_t* __restrict__ list, int64_t m,
                           unsigned long long* __restrict__ keys, uint32_t* __restrict__ rows) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < m;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = list ? list[i] : i;
    keys[i] = static_cast<unsigned long long>(LoadKey(key, r)) ^ (1ULL << 63);
    rows[i] = static_cast<uint32_t>(r);
  }
}

// head flags per 1024-item tile: counts[t] = heads in tile t
__global__ void RunHeadCounts(const unsigned long long* __restrict__ keys, int64_t n, uint64_t* __restrict__ counts) {
  __shared__ unsigned total;
  for (int64_t t = blockIdx.x; t * 1024 < n; t += gridDim.x) {
    if (threadIdx.x == 0) total = 0;
    __syncthreads();
    unsigned mine = 0;
    for (int64_t i = t * 1024 + threadIdx.x; i < ((t + 1) * 1024 < n ? (t + 1) * 1024 : n); i += blockDim.x)
      mine += (i == 0 || keys[i] != keys[i - 1]);
    atomicAdd(&total, mine);
    __syncthreads();
    if (threadIdx.x == 0) counts[t] = total;
    __syncthreads();
  }
}

// writes the distinct keys and run starts of tile t at its offset (heads in
// ascending order: one thread per tile walks its heads)
__global__ void RunHeadWrite(const unsigned long long* __restrict__ keys, int64_t n, const uint64_t* __restrict__ off,
                             int64_t* __restrict__ dkeys, int64_t* __restrict__ starts) {
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t * 1024 < n;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint64_t o = off[t];
    for (int64_t i = t * 1024; i < ((t + 1) * 1024 < n ? (t + 1) * 1024 : n); i++)
      if (i == 0 || keys[i] != keys[i - 1]) {
        dkeys[o] = static_cast<int64_t>(keys[i] ^ (1ULL << 63));
        starts[o] = i;
        o++;
      }
  }
}

}  // namespace

ColumnIndex::~ColumnIndex() {
  if (!ctx || ctx->dry) return;
  cudaSetDevice(ctx->device);
  if (rows) cudaFree(rows);
  if (dkeys) cudaFree(dkeys);
  if (starts) cudaFree(starts);
}

int64_t ColumnIndex::Get(int64_t key, int32_t* out, int64_t cap) const {
  auto it = std::lower_bound(hkeys.begin(), hkeys.end(), key);
  if (it == hkeys.end() || *it != key) return 0;
  const size_t k = static_cast<size_t>(it - hkeys.begin());
  const int64_t b = hstarts[k], e = hstarts[k + 1];
  if (out && cap > 0) {
    const int64_t m = std::min(cap, e - b);
    if (!rows) std::memcpy(out, hrows.data() + b, sizeof(int32_t) * m);
    else KDB_CUDA(cudaMemcpy(out, rows + b, sizeof(int32_t) * m, cudaMemcpyDeviceToHost));
  }
  return e - b;
}

std::unique_ptr<ColumnIndex> IndexBuild(Context& c, const std::string& table, const std::string& column) {
  if (c.dry) throw Error(KDB_ERR_UNSUPPORTED, "operators need a device context");
  const DevColumn& col = c.Column(table, column);
  const KeyCol key = KeyOf(col);
  const int64_t n = col.n;
  if (n >= (int64_t(1) << 31)) throw Error(KDB_ERR_CAPACITY, "indexes hold row ids below 2^31");
  auto idx = std::make_unique<ColumnIndex>();
  idx->ctx = &c;
  idx->type = col.type;
  Arena arena(c);
  c.TimedStart("index build");
  // the rows with a non-NULL key, in row order (NULL keys are not indexed)
  const int32_t* list = nullptr;
  int64_t m = n;
  if (col.nulls && n > 0) {
    const int64_t nt = (n + 1023) / 1024;
    int32_t* scratch = arena.AllocT<int32_t>(nt * 1024);
    uint64_t* cnt = arena.AllocT<uint64_t>(nt + 1);
    CompactNonNull<<<static_cast<int>(std::min<int64_t>(nt, c.num_sms * 8)), 256, 0, c.stream>>>(col.nulls, n,
                                                                                                  scratch, cnt);
    c.kernel_launches++;
    c.ScanU64(cnt, nt, "index non-null");
    uint64_t mm = 0;
    c.D2H(&mm, cnt + nt, 8);
    m = static_cast<int64_t>(mm);
    int32_t* l = arena.AllocT<int32_t>(std::max<int64_t>(m, 1));
    GatherTiles(c, scratch, cnt, nt, l);
    list = l;
  }
  unsigned long long* keys = arena.AllocT<unsigned long long>(std::max<int64_t>(m, 1));
  uint32_t* rows = arena.AllocT<uint32_t>(std::max<int64_t>(m, 1));
  if (m > 0) {
    IndexPairs<<<c.GridFor(m, kBlock), kBlock, 0, c.stream>>>(key, list, m, keys, rows);
    c.kernel_launches++;
  }
  // rows are in ascending order; a stable sort by key keeps them so within
  // every key (the posting lists' insertion order)
  c.RadixSortPairs(reinterpret_cast<uint64_t*>(keys), rows, m, arena, 64);
  const int64_t ntiles = (m + 1023) / 1024;
  uint64_t* counts = arena.AllocT<uint64_t>(ntiles + 1);
  if (ntiles > 0) {
    RunHeadCounts<<<static_cast<int>(std::min<int64_t>(ntiles, c.num_sms * 8)), 256, 0, c.stream>>>(keys, m,
                                                                                                      counts);
    c.kernel_launches++;
  }
  c.ScanU64(counts, ntiles, "index runs");
  uint64_t nk = 0;
  c.D2H(&nk, counts + ntiles, 8);
  idx->n = m;
  idx->nkeys = static_cast<int64_t>(nk);
  idx->rows = static_cast<int32_t*>(c.DevAlloc(sizeof(int32_t) * std::max<int64_t>(m, 1)));
  idx->dkeys = static_cast<int64_t*>(c.DevAlloc(sizeof(int64_t) * std::max<uint64_t>(nk, 1)));
  idx->starts = static_cast<int64_t*>(c.DevAlloc(sizeof(int64_t) * (nk + 1)));
  if (m > 0)
    KDB_CUDA(cudaMemcpyAsync(idx->rows, rows, sizeof(int32_t) * m, cudaMemcpyDeviceToDevice, c.stream));
  if (ntiles > 0) {
    RunHeadWrite<<<c.GridFor(ntiles, 128), 128, 0, c.stream>>>(keys, m, counts, idx->dkeys, idx->starts);
    c.kernel_launches++;
  }
  KDB_CUDA(cudaMemcpyAsync(idx->starts + nk, &idx->n, 8, cudaMemcpyHostToDevice, c.stream));
  c.TimedStop();
  idx->hkeys.resize(nk);
  idx->hstarts.resize(nk + 1);
  if (nk) c.D2H(idx->hkeys.data(), idx->dkeys, 8 * nk);
  c.D2H(idx->hstarts.data(), idx->starts, 8 * (nk + 1));
  KDB_CUDA(cudaGetLastError());
  return idx;
}

std::unique_ptr<ColumnIndex> IndexFromPostings(Context& c, plan::Type type,
                                               std::vector<std::pair<int64_t, std::vector<int32_t>>> postings) {
  std::sort(postings.begin(), postings.end(),
            [](const auto& a, const auto& b) { return a.first < b.first; });
  auto idx = std::make_unique<ColumnIndex>();
  idx->ctx = &c;
  idx->type = type;
  std::vector<int32_t> rows;
  idx->hkeys.reserve(postings.size());
  idx->hstarts.push_back(0);
  for (size_t k = 0; k < postings.size(); k++) {
    if (k && postings[k].first == postings[k - 1].first) throw Error(KDB_ERR_INVALID, "index repeats a key");
    idx->hkeys.push_back(postings[k].first);
    rows.insert(rows.end(), postings[k].second.begin(), postings[k].second.end());
    idx->hstarts.push_back(static_cast<int64_t>(rows.size()));
  }
  idx->n = static_cast<int64_t>(rows.size());
  idx->nkeys = static_cast<int64_t>(idx->hkeys.size());
  if (c.dry) {  // compile-only context: the posting lists stay on the host
    idx->hrows = std::move(rows);
    return idx;
  }
  idx->rows = static_cast<int32_t*>(c.DevAlloc(sizeof(int32_t) * std::max<size_t>(rows.size(), 1)));
  idx->dkeys = static_cast<int64_t*>(c.DevAlloc(sizeof(int64_t) * std::max<size_t>(idx->hkeys.size(), 1)));
  idx->starts = static_cast<int64_t*>(c.DevAlloc(sizeof(int64_t) * idx->hstarts.size()));
  if (!rows.empty())
    KDB_CUDA(cudaMemcpy(idx->rows, rows.data(), sizeof(int32_t) * rows.size(), cudaMemcpyHostToDevice));
  if (!idx->hkeys.empty())
    KDB_CUDA(cudaMemcpy(idx->dkeys, idx->hkeys.data(), 8 * idx->hkeys.size(), cudaMemcpyHostToDevice));
  KDB_CUDA(cudaMemcpy(idx->starts, idx->hstarts.data(), 8 * idx->hstarts.size(), cudaMemcpyHostToDevice));
  return idx;
}

}  // namespace ops
}  // namespace kdb
