// Device runtime for generated pipeline kernels (sm_100a).
//
// Every pipeline kernel the code generator emits is compiled by NVRTC with
// this header prepended; it holds the hand-written device pieces the pipelines
// call: value types, SQL null-aware helpers, string predicates
// (runtime/string.cc:14-77), Julian-day date split (runtime/date.cc:29-44),
// 64-bit hashing, warp-aggregated slot allocation for materialisation, the
// open-addressing join / group tables and their atomic aggregate updates.
// It must stay free of standard-library includes (NVRTC has none).
#pragma once

typedef signed char int8_t;
typedef short int16_t;
typedef int int32_t;
typedef long long int64_t;
typedef unsigned char uint8_t;
typedef unsigned short uint16_t;
typedef unsigned int uint32_t;
typedef unsigned long long uint64_t;

#define KDB_DEV __device__ __forceinline__

// Error codes written to the per-launch error word (host maps them to
// KDB_ERR_*).
#define KDB_DEV_ERR_CAPACITY 1
#define KDB_DEV_ERR_TIMEOUT 2
#define KDB_DEV_ERR_UNSUPPORTED 3

// Bounded spin: every device-side wait gives up after this many polls and
// reports KDB_DEV_ERR_TIMEOUT instead of hanging the GPU.
#define KDB_SPIN_LIMIT (1 << 20)

struct KArgs {
  uint64_t w[384];
};
// A kernel's parameter block holds only the words it uses (rounded up): the
// launch copies sizeof(parameter) bytes, and a 3 KB block costs launch time.
template <int N>
struct KArgsN {
  uint64_t w[N];
};

// A TEXT value: pointer into device column data (or a kernel literal) + length.
struct kdb_str {
  const char* p;
  int32_t len;
};

KDB_DEV kdb_str kdb_mkstr(const char* p, int32_t len) {
  kdb_str s;
  s.p = p;
  s.len = len;
  return s;
}

// TEXT column storage: int64 offsets[n+1] + bytes.
KDB_DEV kdb_str kdb_text_at(const int64_t* off, const char* chars, int64_t r) {
  int64_t b = off[r];
  return kdb_mkstr(chars + b, (int32_t)(off[r + 1] - b));
}

// ---- string predicates (std::string_view semantics, unsigned bytes) --------
KDB_DEV int kdb_str_cmp(kdb_str a, kdb_str b) {
  int32_t n = a.len < b.len ? a.len : b.len;
  for (int32_t i = 0; i < n; i++) {
    unsigned char x = (unsigned char)a.p[i], y = (unsigned char)b.p[i];
    if (x != y) return x < y ? -1 : 1;
  }
  return a.len == b.len ? 0 : (a.len < b.len ? -1 : 1);
}
KDB_DEV bool kdb_str_eq(kdb_str a, kdb_str b) {
  if (a.len != b.len) return false;
  for (int32_t i = 0; i < a.len; i++)
    if (a.p[i] != b.p[i]) return false;
  return true;
}
KDB_DEV bool kdb_str_starts_with(kdb_str a, kdb_str b) {
  if (b.len > a.len) return false;
  for (int32_t i = 0; i < b.len; i++)
    if (a.p[i] != b.p[i]) return false;
  return true;
}
KDB_DEV bool kdb_str_ends_with(kdb_str a, kdb_str b) {
  if (b.len > a.len) return false;
  int32_t o = a.len - b.len;
  for (int32_t i = 0; i < b.len; i++)
    if (a.p[o + i] != b.p[i]) return false;
  return true;
}
// Substring search (string_view::find != npos).  Checks the first byte
// before comparing the rest; the LIKE '%tok%' predicates it serves use
// short needles.
// Full match of a LIKE pattern as a bit-parallel NFA: state i = the first i
// pattern tokens matched (at most 63 tokens).  tr[c] has bit i when token i
// consumes byte c (a literal c, or '_' for any byte but '\n'); star has the
// bits of the '%' tokens, which consume any run of bytes but '\n' and may
// also match nothing.
KDB_DEV uint64_t kdb_like_close(uint64_t d, uint64_t star) {
  for (int k = 0; k < 64; k++) {
    const uint64_t nd = d | ((d & star) << 1);
    if (nd == d) break;
    d = nd;
  }
  return d;
}
KDB_DEV bool kdb_like(kdb_str s, const unsigned long long* tr, unsigned long long star, int n) {
  uint64_t d = kdb_like_close(1ULL, star);
  for (int32_t i = 0; i < s.len && d; i++) {
    const unsigned char c = (unsigned char)s.p[i];
    uint64_t nd = (d & tr[c]) << 1;
    if (c != '\n') nd |= d & star;
    d = kdb_like_close(nd, star);
  }
  return (d >> n) & 1ULL;
}

KDB_DEV bool kdb_str_contains(kdb_str a, kdb_str b) {
  if (b.len == 0) return true;
  if (b.len > a.len) return false;
  char f = b.p[0];
  for (int32_t i = 0; i + b.len <= a.len; i++) {
    if (a.p[i] != f) continue;
    int32_t j = 1;
    while (j < b.len && a.p[i + j] == b.p[j]) j++;
    if (j == b.len) return true;
  }
  return false;
}

// Enum dictionary on the device: key k -> chars[off[k] .. off[k+1]).
KDB_DEV kdb_str kdb_enum_str(const int64_t* off, const char* chars, int32_t k) {
  return kdb_text_at(off, chars, k);
}

// ---- dates (runtime/date.cc:29-50) -----------------------------------------
KDB_DEV int32_t kdb_extract_year(int32_t jd) {
  uint32_t julian = (uint32_t)jd;
  julian += 32044;
  uint32_t quad = julian / 146097;
  uint32_t extra = (julian - quad * 146097) * 4 + 3;
  julian += 60 + quad * 3 + extra / 146097;
  quad = julian / 1461;
  julian -= quad * 1461;
  int32_t y = (int32_t)(julian * 4 / 1461);
  y += (int32_t)(quad * 4);
  return y - 4800;
}

// ---- 4-row vector loads ------------------------------------------------------
// A scan thread loads 4 consecutive rows of each column with 128-bit (or
// narrower, for 1-2 byte types) streaming loads: every column byte is read
// exactly once, so evict-first (__ldcs) keeps them from displacing the hash
// tables in L2.  `base` is a multiple of 4 and the columns are 256-byte
// aligned, so every vector access is naturally aligned.
KDB_DEV void kdb_ld4(const int32_t* p, int64_t base, int32_t* o) {
  int4 v = __ldcs(reinterpret_cast<const int4*>(p + base));
  o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
KDB_DEV void kdb_ld4(const double* p, int64_t base, double* o) {
  double2 a = __ldcs(reinterpret_cast<const double2*>(p + base));
  double2 b = __ldcs(reinterpret_cast<const double2*>(p + base + 2));
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
KDB_DEV void kdb_ld4(const int64_t* p, int64_t base, int64_t* o) {
  longlong2 a = __ldcs(reinterpret_cast<const longlong2*>(p + base));
  longlong2 b = __ldcs(reinterpret_cast<const longlong2*>(p + base + 2));
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
KDB_DEV void kdb_ld4(const int16_t* p, int64_t base, int16_t* o) {
  short4 v = __ldcs(reinterpret_cast<const short4*>(p + base));
  o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
KDB_DEV void kdb_ld4(const int8_t* p, int64_t base, int8_t* o) {
  char4 v = __ldcs(reinterpret_cast<const char4*>(p + base));
  o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}

// Four consecutive values from a shared-memory stage (`i` a multiple of 4,
// the column's stage region 16-byte aligned).
KDB_DEV void kdb_lds4(const int32_t* p, int i, int32_t* o) {
  int4 v = *reinterpret_cast<const int4*>(p + i);
  o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
KDB_DEV void kdb_lds4(const double* p, int i, double* o) {
  double2 a = *reinterpret_cast<const double2*>(p + i);
  double2 b = *reinterpret_cast<const double2*>(p + i + 2);
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
KDB_DEV void kdb_lds4(const int64_t* p, int i, int64_t* o) {
  longlong2 a = *reinterpret_cast<const longlong2*>(p + i);
  longlong2 b = *reinterpret_cast<const longlong2*>(p + i + 2);
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
KDB_DEV void kdb_lds4(const int16_t* p, int i, int16_t* o) {
  short4 v = *reinterpret_cast<const short4*>(p + i);
  o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
KDB_DEV void kdb_lds4(const int8_t* p, int i, int8_t* o) {
  char4 v = *reinterpret_cast<const char4*>(p + i);
  o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}

// ---- partial-word combining (finalize kernels) ---------------------------------
// Word kinds: 0 = FP64 sum (bits of a double), 1 = 64-bit integer sum,
// 2 = unsigned minimum, 3 = unsigned maximum.
KDB_DEV uint64_t kdb_word_identity(int kind) { return kind == 2 ? ~0ULL : 0ULL; }
KDB_DEV uint64_t kdb_word_combine(int kind, uint64_t a, uint64_t b) {
  switch (kind) {
    case 0: return (uint64_t)__double_as_longlong(__dadd_rn(__longlong_as_double((long long)a),
                                                           __longlong_as_double((long long)b)));
    case 1: return a + b;
    case 2: return b < a ? b : a;
    default: return b > a ? b : a;
  }
}

// ---- TMA bulk copies into shared-memory stages -------------------------------
// One mbarrier per stage (arrival count 1): the issuing thread announces the
// stage's total bytes, then starts one 1-D bulk copy per column; the phase
// completes when every byte has landed.  Waits are bounded.
KDB_DEV uint32_t kdb_smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
KDB_DEV void kdb_bar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(kdb_smem_addr(bar)) : "memory");
}
// orders this thread's generic shared-memory accesses (and barrier inits)
// before its later bulk copies
KDB_DEV void kdb_fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
KDB_DEV void kdb_bar_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(kdb_smem_addr(bar)), "r"(bytes)
               : "memory");
}
// dst, src and bytes are multiples of 16
KDB_DEV void kdb_bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   kdb_smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(kdb_smem_addr(bar))
               : "memory");
}
KDB_DEV bool kdb_bar_wait(uint64_t* bar, uint32_t parity) {
  for (int it = 0; it < KDB_SPIN_LIMIT; it++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(kdb_smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// Every thread waits; the outcome is block-uniform.  A wait that gave up
// records KDB_DEV_ERR_TIMEOUT.
KDB_DEV bool kdb_bar_wait_all(uint64_t* bar, uint32_t parity, int* err) {
  const bool ok = kdb_bar_wait(bar, parity);
  if (!__syncthreads_or(!ok)) return true;
  if (threadIdx.x == 0) atomicCAS(err, 0, KDB_DEV_ERR_TIMEOUT);
  return false;
}

// ---- hashing ----------------------------------------------------------------
KDB_DEV uint64_t kdb_mix64(uint64_t x) {
  // splitmix64 finaliser
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ULL;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebULL;
  x ^= x >> 31;
  return x;
}
KDB_DEV uint64_t kdb_hash_combine(uint64_t h, uint64_t v) {
  return kdb_mix64(h ^ (v + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2)));
}
// Join keys hash to 32 bits with murmur3's 32-bit finaliser; a 64-bit value
// is folded first (low + high * golden ratio), so equal values of any
// integer width hash alike.  The low bits of the hash index the table.
KDB_DEV uint32_t kdb_fmix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x85ebca6bu;
  x ^= x >> 13;
  x *= 0xc2b2ae35u;
  x ^= x >> 16;
  return x;
}
KDB_DEV uint32_t kdb_hash64to32(uint64_t v) {
  return kdb_fmix32((uint32_t)v + (uint32_t)(v >> 32) * 0x9e3779b9u);
}
KDB_DEV uint32_t kdb_hash_combine32(uint32_t h, uint32_t v) {
  return kdb_fmix32(h ^ (v + 0x9e3779b9u + (h << 6) + (h >> 2)));
}
KDB_DEV uint64_t kdb_hash_str(kdb_str s) {
  uint64_t h = 0xcbf29ce484222325ULL;  // FNV-1a
  for (int32_t i = 0; i < s.len; i++) {
    h ^= (unsigned char)s.p[i];
    h *= 0x100000001b3ULL;
  }
  return kdb_mix64(h ^ (uint64_t)s.len);
}
KDB_DEV uint64_t kdb_dbits(double d) {
  // -0.0 and 0.0 are Equal (evaluate.cc Equal on REAL) so hash them alike
  if (d == 0.0) d = 0.0;
  return (uint64_t)__double_as_longlong(d);
}

// Order-preserving double <-> uint64 (for atomicMin/Max and radix keys).
KDB_DEV uint64_t kdb_dord(double d) {
  uint64_t b = (uint64_t)__double_as_longlong(d);
  return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}
KDB_DEV double kdb_dord_inv(uint64_t k) {
  uint64_t b = (k & 0x8000000000000000ULL) ? (k & 0x7fffffffffffffffULL) : ~k;
  return __longlong_as_double((long long)b);
}

// ---- warp-aggregated slot allocation --------------------------------------
// One atomicAdd per warp: the active lanes that want a slot get consecutive
// indices.  Called from divergent code: uses the active mask.
KDB_DEV uint64_t kdb_alloc_slot(unsigned long long* counter) {
  unsigned mask = __activemask();
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  return base + __popc(mask & ((1u << lane) - 1));
}

// The same for a block-local counter in shared memory.
KDB_DEV uint32_t kdb_alloc_block_slot(unsigned* counter) {
  unsigned mask = __activemask();
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  unsigned base = 0;
  if (lane == leader) base = atomicAdd(counter, (unsigned)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  return base + __popc(mask & ((1u << lane) - 1));
}

KDB_DEV void kdb_set_error(int* err, int code) { atomicCAS(err, 0, code); }

// ---- atomics for aggregate state -------------------------------------------
KDB_DEV void kdb_atomic_min_u64(uint64_t* p, uint64_t v) {
  atomicMin((unsigned long long*)p, (unsigned long long)v);
}
KDB_DEV void kdb_atomic_max_u64(uint64_t* p, uint64_t v) {
  atomicMax((unsigned long long*)p, (unsigned long long)v);
}
KDB_DEV void kdb_atomic_min_i64(int64_t* p, int64_t v) { atomicMin((long long*)p, (long long)v); }
KDB_DEV void kdb_atomic_max_i64(int64_t* p, int64_t v) { atomicMax((long long*)p, (long long)v); }
KDB_DEV void kdb_atomic_add_i64(int64_t* p, int64_t v) {
  atomicAdd((unsigned long long*)p, (unsigned long long)v);
}

// TEXT MIN/MAX: the state is a 64-bit handle (48-bit device pointer | 16-bit
// length) replaced by CAS while the new string compares better.  Strings
// longer than 65535 bytes are rejected by the caller.
KDB_DEV uint64_t kdb_str_handle(kdb_str s) {
  return (((uint64_t)s.p) & 0xFFFFFFFFFFFFULL) | ((uint64_t)(uint16_t)s.len << 48);
}
KDB_DEV kdb_str kdb_str_from_handle(uint64_t h) {
  uint64_t ptr = h & 0xFFFFFFFFFFFFULL;
  // restore canonical sign extension of the 48-bit address
  if (ptr & 0x800000000000ULL) ptr |= 0xFFFF000000000000ULL;
  return kdb_mkstr((const char*)ptr, (int32_t)(h >> 48));
}
KDB_DEV void kdb_atomic_str_minmax(uint64_t* p, kdb_str v, bool is_min) {
  uint64_t nv = kdb_str_handle(v);
  uint64_t cur = *(volatile uint64_t*)p;
  for (int it = 0; it < KDB_SPIN_LIMIT; it++) {
    if (cur != 0) {
      int c = kdb_str_cmp(v, kdb_str_from_handle(cur));
      if (is_min ? (c >= 0) : (c <= 0)) return;
    }
    uint64_t prev = atomicCAS((unsigned long long*)p, cur, nv);
    if (prev == cur) return;
    cur = prev;
  }
}

// ---- open-addressing join table ---------------------------------------------
// Entry = (hash32 << 32) | (row + 1); 0 = empty.  Duplicate keys are separate
// entries (a probe walks the run until an empty slot).  Capacity is a power
// of two at least twice the build rows, so the table never fills.
// Join filter: one bit per 32-bit hash, placed by the hash's multiplicative
// remix (top bits), independent of the table index (its low bits).
KDB_DEV uint32_t kdb_bloom_bit(uint32_t h, int log2_bits) { return (h * 0x9e3779b1u) >> (32 - log2_bits); }
KDB_DEV void kdb_bloom_set(uint32_t* bits, uint32_t h, int log2_bits) {
  const uint32_t b = kdb_bloom_bit(h, log2_bits);
  atomicOr(&bits[b >> 5], 1u << (b & 31));
}
KDB_DEV bool kdb_bloom_test(const uint32_t* __restrict__ bits, uint32_t h, int log2_bits) {
  const uint32_t b = kdb_bloom_bit(h, log2_bits);
  return (__ldg(&bits[b >> 5]) >> (b & 31)) & 1u;
}

// Same, storing the (32-bit) key in the slot's high word instead of the hash.
// Returns whether the walk passed a slot holding the same key: of two rows
// with equal keys (same hash, same walk; slots are only ever filled) the one
// inserted second always passes the first one's slot, so a table with a
// duplicate key reports it at least once.
KDB_DEV bool kdb_join_insert_keyed(uint64_t* slots, uint64_t mask, uint32_t h, uint32_t key, uint32_t row) {
  uint64_t e = ((uint64_t)key << 32) | (uint64_t)(row + 1);
  const uint32_t m = (uint32_t)mask;
  uint32_t i = h & m;
  bool dup = false;
  for (uint32_t k = 0; k <= m; k++) {
    const unsigned long long old = atomicCAS((unsigned long long*)&slots[i], 0ULL, (unsigned long long)e);
    if (old == 0ULL) return dup;
    dup |= (uint32_t)(old >> 32) == key;
    i = (i + 1) & m;
  }
  return dup;
}

KDB_DEV void kdb_join_insert(uint64_t* slots, uint64_t mask, uint32_t h, uint32_t row) {
  uint64_t e = ((uint64_t)h << 32) | (uint64_t)(row + 1);
  const uint32_t m = (uint32_t)mask;  // tables hold at most 2^32 slots
  uint32_t i = h & m;
  for (uint32_t k = 0; k <= m; k++) {
    if (atomicCAS((unsigned long long*)&slots[i], 0ULL, (unsigned long long)e) == 0ULL) return;
    i = (i + 1) & m;
  }
}

// ---- group tables ------------------------------------------------------------
// Packed keys: the whole group key fits in 63 bits; the slot word holds
// key | 1<<63 and is claimed by a single CAS (no wait on other threads).
// Overflow detection: tables are sized at most half full from the expected
// group count, where a probe run averages about two slots; a run longer than
// KDB_MAX_PROBE slots therefore means the estimate was wrong, and the lookup
// reports KDB_DEV_ERR_CAPACITY (the host regrows the table and reruns).  No
// shared counter is touched on the hot path.
#define KDB_MAX_PROBE 256

KDB_DEV int64_t kdb_group_find_packed(uint64_t* slots, uint64_t mask, uint64_t key, int* err) {
  uint64_t i = kdb_mix64(key) & mask;
  for (uint64_t k = 0; k <= mask && k < KDB_MAX_PROBE; k++) {
    uint64_t s = *(volatile uint64_t*)&slots[i];
    if (s == key) return (int64_t)i;
    if (s == 0) {
      uint64_t prev = atomicCAS((unsigned long long*)&slots[i], 0ULL, (unsigned long long)key);
      if (prev == 0 || prev == key) return (int64_t)i;
    }
    i = (i + 1) & mask;
  }
  kdb_set_error(err, KDB_DEV_ERR_CAPACITY);
  return -1;
}

// General keys: the slot word is 0 (empty), 1 (being initialised) or the
// key hash (bit 63 set).  The claiming thread writes the key columns, fences
// and publishes the hash; others wait (bounded) while they see 1, then
// compare keys with `eq` (which must read key columns with __ldcg).
template <typename EQ, typename INIT>
KDB_DEV int64_t kdb_group_find(uint64_t* slots, uint64_t mask, uint64_t h, EQ eq, INIT init, int* err) {
  uint64_t i = h & mask;
  for (uint64_t k = 0; k <= mask && k < KDB_MAX_PROBE; k++) {
    uint64_t s = *(volatile uint64_t*)&slots[i];
    if (s == 0) {
      uint64_t prev = atomicCAS((unsigned long long*)&slots[i], 0ULL, 1ULL);
      if (prev == 0) {
        init(i);
        __threadfence();
        atomicExch((unsigned long long*)&slots[i], (unsigned long long)h);
        return (int64_t)i;
      }
      s = prev;
    }
    if (s == 1) {
      // the claiming thread may be a lane of this warp: back off so the
      // scheduler runs it (independent thread scheduling), bounded
      int it = 0;
      while ((s = *(volatile uint64_t*)&slots[i]) == 1 && it < KDB_SPIN_LIMIT) {
        __nanosleep(64);
        it++;
      }
      if (s == 1) {
        kdb_set_error(err, KDB_DEV_ERR_TIMEOUT);
        return -1;
      }
    }
    if (s == h && eq(i)) return (int64_t)i;
    i = (i + 1) & mask;
  }
  kdb_set_error(err, KDB_DEV_ERR_CAPACITY);
  return -1;
}

// ---- block reductions (ungrouped aggregates) ---------------------------------
struct KdbAddF64 {
  KDB_DEV double operator()(double a, double b) const { return a + b; }
};
struct KdbAddI64 {
  KDB_DEV int64_t operator()(int64_t a, int64_t b) const {
    return (int64_t)((uint64_t)a + (uint64_t)b);
  }
};
struct KdbMinU64 {
  KDB_DEV uint64_t operator()(uint64_t a, uint64_t b) const { return a < b ? a : b; }
};
struct KdbMaxU64 {
  KDB_DEV uint64_t operator()(uint64_t a, uint64_t b) const { return a > b ? a : b; }
};
struct KdbMinI64 {
  KDB_DEV int64_t operator()(int64_t a, int64_t b) const { return a < b ? a : b; }
};
struct KdbMaxI64 {
  KDB_DEV int64_t operator()(int64_t a, int64_t b) const { return a > b ? a : b; }
};
struct KdbOrI32 {
  KDB_DEV int32_t operator()(int32_t a, int32_t b) const { return a | b; }
};

// Reduces one value per thread over the block; the result is valid in
// thread 0.  `scratch` holds at least 32 T.  All threads must call it.
template <typename T, typename OP>
KDB_DEV T kdb_block_reduce(T v, OP op, T* scratch) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_down_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  if (warp == 0) {
    // every lane of warp 0 takes part in each full-mask shuffle; lanes past
    // the warp count only feed values that are never combined
    T x = lane < nw ? scratch[lane] : scratch[0];
    for (int o = 16; o > 0; o >>= 1) {
      T y = __shfl_down_sync(0xffffffffu, x, o);
      if (lane + o < nw) x = op(x, y);
    }
    v = x;
  }
  return v;
}

// Order-by tie key: position of stream index i in the reference's top-down
// merge sort (runtime/vector.cc:89-103), whose merge emits the right run first
// on ties.  Bit d (from the top) is 0 when i falls in the right half at depth
// d, so sorting equal rows by this key reproduces the reference's tie order.
KDB_DEV uint64_t kdb_tie_path(uint64_t i, uint64_t n) {
  uint64_t l = 0, r = n - 1, key = 0;
  int depth = 0;
  while (l < r && depth < 64) {
    uint64_t m = l + (r - l) / 2;
    if (i > m) {
      l = m + 1;
    } else {
      key |= 1ULL << (63 - depth);
      r = m;
    }
    depth++;
  }
  return key;
}

// Big-endian 8-byte chunk c of a string, zero padded (ORDER BY on TEXT).
KDB_DEV uint64_t kdb_str_chunk(kdb_str s, int c) {
  uint64_t k = 0;
  for (int b = 0; b < 8; b++) {
    int idx = c * 8 + b;
    uint64_t byte = idx < s.len ? (uint64_t)(unsigned char)s.p[idx] : 0ULL;
    k = (k << 8) | byte;
  }
  return k;
}
