// Batched form: many queries of one scan-select -> hash-join -> group-by
// template, of uneven sizes, executed together as one CUDA graph of fused
// kernels.
//
//   SELECT d.<key>, SUM(f.<price> * (1 - f.<disc>))
//   FROM dim d JOIN fact f ON f.<fk> = d.<key>
//   WHERE d.<date> < date_lt AND d.<seg> = seg
//   GROUP BY d.<key>
//
// (the plan HashJoin(ScanSelect(dim), Scan(fact)) -> GroupByAggregate of
// hash_join_translator.cc:34-139 / group_by_aggregate_translator.cc:36-111,
// with per-query predicate constants).  Plain execution pays a launch
// sequence, host synchronisations and code-generation per query; here every
// phase of all queries is one launch:
//   1. build  -- filter each query's dimension rows and insert the survivors
//      into that query's join table (CAS on (key, row) slots);
//   2. probe  -- over the fact rows: probe, and add the measure into the
//      matched build row's accumulator (the dimension key is the table's
//      primary key, so the build row is the group; duplicate build keys are
//      detected and reported);
//   3. output -- compact each query's touched build rows into its result.
// Each CTA owns a fixed chunk of one query's rows (block x 16), and chunks
// are numbered query after query, so the CTAs resident at any moment work on
// a few queries and their join tables and accumulators stay in L2.
// Capacities are sized when the batch is configured, so no phase needs a
// read-back and the whole batch is captured once into a CUDA graph and
// replayed.  Tunables (chosen by kdb_batch_tune): block size, join-table load
// factor, and radix fan-out P -- with P > 1 each query's join table is split
// into P sub-tables by the top bits of the key hash, so a probe's working set
// is one sub-table (for build sides larger than L2).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "capi_internal.h"

namespace kdb {
namespace {

constexpr int kRowsPerThread = 16;  // rows of one chunk per thread
constexpr int kProbeUnroll = 4;     // independent probes in flight per thread

struct QueryDesc {
  // dimension side
  const int32_t* d_key;
  const int32_t* d_date;
  const int32_t* d_seg;
  int64_t nd;
  int32_t date_lt;
  int32_t seg;
  // fact side
  const int32_t* f_fk;
  const double* f_price;
  const double* f_disc;
  int64_t nf;
  // join table: P sub-tables of `sub_cap` slots each, slots[slot_base ...]
  int64_t slot_base;
  uint32_t sub_cap;
  uint32_t pad;
  // per-build-row accumulators acc[acc_base + row]
  int64_t acc_base;
  // result region out[out_base ...] (capacity nd)
  int64_t out_base;
  // CTA ranges of the three phases (one chunk of rows per CTA)
  int32_t build_block0, build_blocks;
  int32_t probe_block0, probe_blocks;
  int32_t out_block0, out_blocks;
};

// Per build row: the running sum and the complement of the first fact row
// that reached it (0 = untouched; atomicMax of ~row keeps the smallest row).
struct Acc {
  double sum;
  unsigned long long first_inv;
};
static_assert(sizeof(Acc) == 16, "Acc layout");

// 64-bit mix of the key: the top bits choose the sub-table, the low 32 bits
// the home slot inside it, so the two are independent.
__device__ __forceinline__ uint64_t KeyHash(int32_t k) {
  uint64_t x = static_cast<uint64_t>(static_cast<uint32_t>(k)) * 0x9E3779B97F4A7C15ULL;
  x ^= x >> 31;
  x *= 0xBF58476D1CE4E5B9ULL;
  x ^= x >> 29;
  return x;
}

__device__ __forceinline__ uint32_t SubTable(uint64_t h, int fanout_bits) {
  return fanout_bits ? static_cast<uint32_t>(h >> (64 - fanout_bits)) : 0u;
}

__device__ __forceinline__ uint32_t HomeSlot(uint64_t h, uint32_t cap) {
  return static_cast<uint32_t>((static_cast<uint64_t>(static_cast<uint32_t>(h)) * cap) >> 32);
}

// block -> query by binary search over the queries' first blocks
template <int kPhase>
__device__ __forceinline__ int FindQuery(const QueryDesc* qs, int nq, int block) {
  int lo = 0, hi = nq - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    int b0 = kPhase == 0 ? qs[mid].build_block0 : kPhase == 1 ? qs[mid].probe_block0 : qs[mid].out_block0;
    if (b0 <= block) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Rows [r0, r1) of this CTA's chunk.
template <int kPhase>
__device__ __forceinline__ const QueryDesc& Chunk(const QueryDesc* qs, int nq, int64_t& r0, int64_t& r1) {
  __shared__ int sq;
  if (threadIdx.x == 0) sq = FindQuery<kPhase>(qs, nq, blockIdx.x);
  __syncthreads();
  const QueryDesc& q = qs[sq];
  const int b0 = kPhase == 0 ? q.build_block0 : kPhase == 1 ? q.probe_block0 : q.out_block0;
  const int64_t chunk = static_cast<int64_t>(blockDim.x) * kRowsPerThread;
  const int64_t n = kPhase == 1 ? q.nf : q.nd;
  r0 = (blockIdx.x - b0) * chunk;
  r1 = r0 + chunk < n ? r0 + chunk : n;
  return q;
}

// Rows of every dimension table per (query, sub-table): sizes the
// sub-tables so that none can overflow whatever the predicates select.
__global__ void BatchPartCount(const QueryDesc* __restrict__ qs, int nq, int fanout_bits,
                               unsigned* __restrict__ counts) {
  extern __shared__ unsigned hist[];
  const int parts = 1 << fanout_bits;
  for (int i = threadIdx.x; i < parts; i += blockDim.x) hist[i] = 0;
  int64_t r0, r1;
  const QueryDesc& q = Chunk<0>(qs, nq, r0, r1);
  const int qi = static_cast<int>(&q - qs);
  for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x)
    atomicAdd(&hist[SubTable(KeyHash(__ldcs(q.d_key + r)), fanout_bits)], 1u);
  __syncthreads();
  for (int i = threadIdx.x; i < parts; i += blockDim.x)
    if (hist[i]) atomicAdd(&counts[static_cast<int64_t>(qi) * parts + i], hist[i]);
}

// slot = (key << 32) | (row + 1); 0 = empty
__global__ void BatchBuild(const QueryDesc* __restrict__ qs, int nq, unsigned long long* __restrict__ slots,
                           int fanout_bits, int* __restrict__ err) {
  int64_t r0, r1;
  const QueryDesc& q = Chunk<0>(qs, nq, r0, r1);
  for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    if (!(__ldcs(q.d_date + r) < q.date_lt)) continue;
    if (!(__ldcs(q.d_seg + r) == q.seg)) continue;
    const int32_t k = __ldcs(q.d_key + r);
    const uint64_t h = KeyHash(k);
    unsigned long long* sub = slots + q.slot_base + static_cast<int64_t>(SubTable(h, fanout_bits)) * q.sub_cap;
    uint32_t i = HomeSlot(h, q.sub_cap);
    const unsigned long long e =
        (static_cast<unsigned long long>(static_cast<uint32_t>(k)) << 32) | static_cast<unsigned long long>(r + 1);
    bool placed = false;
    for (uint32_t n = 0; n < q.sub_cap; n++) {
      const unsigned long long prev = atomicCAS(sub + i, 0ULL, e);
      if (prev == 0) {
        placed = true;
        break;
      }
      if (static_cast<uint32_t>(prev >> 32) == static_cast<uint32_t>(k))
        atomicCAS(err, 0, 3);  // duplicate dimension key: not a primary key
      if (++i == q.sub_cap) i = 0;
    }
    if (!placed) atomicCAS(err, 0, 4);
  }
}

// sum and first fact row per build row; kProbeUnroll rows per thread are
// loaded and hashed together so their table reads overlap.
// eager: the measures of the unrolled rows load with their keys, so their
// HBM latency overlaps the probes (otherwise only matching rows load them)
__global__ void BatchProbe(const QueryDesc* __restrict__ qs, int nq, const unsigned long long* __restrict__ slots,
                           int fanout_bits, Acc* __restrict__ acc, int eager) {
  int64_t r0, r1;
  const QueryDesc& q = Chunk<1>(qs, nq, r0, r1);
  const int64_t step = blockDim.x;
  for (int64_t base = r0 + threadIdx.x; base < r1; base += kProbeUnroll * step) {
    int32_t k[kProbeUnroll];
    double mp[kProbeUnroll], md[kProbeUnroll];
    uint32_t pos[kProbeUnroll];
    const unsigned long long* sub[kProbeUnroll];
    unsigned long long e[kProbeUnroll];
#pragma unroll
    for (int j = 0; j < kProbeUnroll; j++) {
      const int64_t r = base + j * step;
      k[j] = r < r1 ? __ldcs(q.f_fk + r) : 0;
      mp[j] = eager && r < r1 ? __ldcs(q.f_price + r) : 0.0;
      md[j] = eager && r < r1 ? __ldcs(q.f_disc + r) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < kProbeUnroll; j++) {
      const uint64_t h = KeyHash(k[j]);
      sub[j] = slots + q.slot_base + static_cast<int64_t>(SubTable(h, fanout_bits)) * q.sub_cap;
      pos[j] = HomeSlot(h, q.sub_cap);
      e[j] = base + j * step < r1 ? sub[j][pos[j]] : 0ULL;
    }
#pragma unroll
    for (int j = 0; j < kProbeUnroll; j++) {
      const int64_t r = base + j * step;
      if (r >= r1) continue;
      unsigned long long s = e[j];
      uint32_t i = pos[j];
      for (uint32_t n = 0; s != 0 && n < q.sub_cap; n++) {
        if (static_cast<uint32_t>(s >> 32) == static_cast<uint32_t>(k[j])) {
          Acc* a = acc + q.acc_base + (static_cast<int64_t>(static_cast<uint32_t>(s)) - 1);
          // plain per-row IEEE arithmetic, like the reference's generated code
          const double pr = eager ? mp[j] : __ldcs(q.f_price + r), di = eager ? md[j] : __ldcs(q.f_disc + r);
          const double v = __dmul_rn(pr, __dsub_rn(1.0, di));
          atomicAdd(&a->sum, v);
          // the first fact row only moves down: skip the atomic once an
          // earlier row is already recorded (a stale read costs one atomic)
          const unsigned long long fi = ~static_cast<unsigned long long>(r);
          if (__ldcg(&a->first_inv) < fi) atomicMax(&a->first_inv, fi);
          break;  // keys are unique on the build side
        }
        if (++i == q.sub_cap) i = 0;
        s = sub[j][i];
      }
    }
  }
}

// per query: build rows with a match -> (key, sum, first fact row); one
// counter atomic per warp
__global__ void BatchOutput(const QueryDesc* __restrict__ qs, int nq, const Acc* __restrict__ acc,
                            int32_t* __restrict__ out_key, double* __restrict__ out_sum,
                            unsigned long long* __restrict__ out_first, unsigned long long* __restrict__ out_count) {
  int64_t r0, r1;
  const QueryDesc& q = Chunk<2>(qs, nq, r0, r1);
  const int qi = static_cast<int>(&q - qs);
  const unsigned lane = threadIdx.x & 31;
  for (int64_t rb = r0; rb < r1; rb += blockDim.x) {  // uniform trip count per warp
    const int64_t r = rb + threadIdx.x;
    Acc a{0.0, 0ULL};
    if (r < r1) a = acc[q.acc_base + r];
    const bool hit = a.first_inv != 0;
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (m == 0) continue;
    unsigned long long o0 = 0;
    if (lane == 0) o0 = atomicAdd(out_count + qi, static_cast<unsigned long long>(__popc(m)));
    o0 = __shfl_sync(0xffffffffu, o0, 0);
    if (hit) {
      const int64_t o = q.out_base + static_cast<int64_t>(o0) + __popc(m & ((1u << lane) - 1));
      out_key[o] = q.d_key[r];
      out_sum[o] = a.sum;
      out_first[o] = ~a.first_inv;
    }
  }
}

}  // namespace

struct BatchConfig {
  int block = 256;
  double load_factor = 0.5;
  int fanout = 1;
};

// One batch: query descriptors, device buffers, the captured graph.
class Batch {
 public:
  Batch(Context& ctx, std::vector<QueryDesc> qs) : ctx_(ctx), host_qs_(std::move(qs)) {}
  ~Batch() { Release(); }

  void Configure(const BatchConfig& cfg) {
    Release();
    cfg_ = cfg;
    int fbits = 0;
    while ((1 << fbits) < cfg.fanout) fbits++;
    fanout_bits_ = fbits;
    const int parts = 1 << fbits;
    const int nq = static_cast<int>(host_qs_.size());
    const int64_t chunk = static_cast<int64_t>(cfg.block) * kRowsPerThread;
    int64_t bb = 0, pb = 0, ob = 0;
    for (auto& q : host_qs_) {
      if (q.nd >= static_cast<int64_t>(UINT32_MAX))
        throw Error(KDB_ERR_CAPACITY, "batch dimension table too large");
      auto blocks = [&](int64_t rows) { return std::max<int64_t>(1, (rows + chunk - 1) / chunk); };
      q.build_block0 = static_cast<int32_t>(bb);
      q.build_blocks = static_cast<int32_t>(blocks(q.nd));
      bb += q.build_blocks;
      q.probe_block0 = static_cast<int32_t>(pb);
      q.probe_blocks = static_cast<int32_t>(blocks(q.nf));
      pb += q.probe_blocks;
      q.out_block0 = static_cast<int32_t>(ob);
      q.out_blocks = static_cast<int32_t>(blocks(q.nd));
      ob += q.out_blocks;
      if (bb > INT_MAX || pb > INT_MAX) throw Error(KDB_ERR_CAPACITY, "batch too large");
    }
    build_grid_ = static_cast<int>(bb);
    probe_grid_ = static_cast<int>(pb);
    out_grid_ = static_cast<int>(ob);
    KDB_CUDA(cudaMalloc(&d_qs_, sizeof(QueryDesc) * nq));
    KDB_CUDA(cudaMemcpy(d_qs_, host_qs_.data(), sizeof(QueryDesc) * nq, cudaMemcpyHostToDevice));
    // largest sub-table population per query (all dimension rows, so it
    // bounds what any predicate lets through)
    std::vector<unsigned> most(nq);
    if (fbits > 0) {
      unsigned* counts = nullptr;
      const size_t nc = static_cast<size_t>(nq) * parts;
      KDB_CUDA(cudaMalloc(&counts, sizeof(unsigned) * nc));
      KDB_CUDA(cudaMemsetAsync(counts, 0, sizeof(unsigned) * nc, ctx_.stream));
      BatchPartCount<<<build_grid_, cfg.block, sizeof(unsigned) * parts, ctx_.stream>>>(d_qs_, nq, fbits, counts);
      KDB_CUDA(cudaGetLastError());
      std::vector<unsigned> h(nc);
      KDB_CUDA(cudaMemcpyAsync(h.data(), counts, sizeof(unsigned) * nc, cudaMemcpyDeviceToHost, ctx_.stream));
      KDB_CUDA(cudaStreamSynchronize(ctx_.stream));
      cudaFree(counts);
      for (int q = 0; q < nq; q++)
        most[q] = *std::max_element(h.begin() + static_cast<int64_t>(q) * parts,
                                    h.begin() + static_cast<int64_t>(q + 1) * parts);
    } else {
      for (int q = 0; q < nq; q++) most[q] = static_cast<unsigned>(host_qs_[q].nd);
    }
    int64_t slot_total = 0, acc_total = 0;
    for (int qi = 0; qi < nq; qi++) {
      auto& q = host_qs_[qi];
      // capacity above the most rows a sub-table can receive: probes always
      // end at an empty slot
      const double want = std::ceil(static_cast<double>(most[qi]) / cfg.load_factor) + 1;
      q.sub_cap = static_cast<uint32_t>(std::max(8.0, want));
      q.slot_base = slot_total;
      slot_total += static_cast<int64_t>(q.sub_cap) * parts;
      q.acc_base = acc_total;
      q.out_base = acc_total;
      acc_total += std::max<int64_t>(q.nd, 1);
    }
    slot_total_ = slot_total;
    acc_total_ = acc_total;
    KDB_CUDA(cudaMemcpy(d_qs_, host_qs_.data(), sizeof(QueryDesc) * nq, cudaMemcpyHostToDevice));
    KDB_CUDA(cudaMalloc(&slots_, sizeof(unsigned long long) * std::max<int64_t>(slot_total, 1)));
    KDB_CUDA(cudaMalloc(&acc_, sizeof(Acc) * acc_total));
    KDB_CUDA(cudaMalloc(&out_key_, sizeof(int32_t) * acc_total));
    KDB_CUDA(cudaMalloc(&out_sum_, sizeof(double) * acc_total));
    KDB_CUDA(cudaMalloc(&out_first_, sizeof(unsigned long long) * acc_total));
    KDB_CUDA(cudaMalloc(&out_count_, sizeof(unsigned long long) * nq));
    KDB_CUDA(cudaMalloc(&err_, sizeof(int)));
    Capture();
  }

  // Replays the batch (all phases of all queries).
  void Run() {
    KDB_CUDA(cudaGraphLaunch(exec_, ctx_.stream));
    ctx_.kernel_launches += 3;
  }

  float RunTimed(int reps) {
    cudaEvent_t a, b;
    KDB_CUDA(cudaEventCreate(&a));
    KDB_CUDA(cudaEventCreate(&b));
    Run();
    KDB_CUDA(cudaEventRecord(a, ctx_.stream));
    for (int i = 0; i < reps; i++) Run();
    KDB_CUDA(cudaEventRecord(b, ctx_.stream));
    KDB_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    KDB_CUDA(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms / reps;
  }

  int CheckError() {
    int e = 0;
    KDB_CUDA(cudaMemcpyAsync(&e, err_, sizeof(int), cudaMemcpyDeviceToHost, ctx_.stream));
    KDB_CUDA(cudaStreamSynchronize(ctx_.stream));
    return e;
  }

  // Result of query q: groups in first-match order of the fact stream.
  void Result(int q, std::vector<int32_t>& keys, std::vector<double>& sums) {
    unsigned long long n = 0;
    KDB_CUDA(cudaMemcpyAsync(&n, out_count_ + q, sizeof(n), cudaMemcpyDeviceToHost, ctx_.stream));
    KDB_CUDA(cudaStreamSynchronize(ctx_.stream));
    const QueryDesc& d = host_qs_[q];
    std::vector<int32_t> k(n);
    std::vector<double> s(n);
    std::vector<unsigned long long> f(n);
    if (n) {
      KDB_CUDA(cudaMemcpyAsync(k.data(), out_key_ + d.out_base, 4 * n, cudaMemcpyDeviceToHost, ctx_.stream));
      KDB_CUDA(cudaMemcpyAsync(s.data(), out_sum_ + d.out_base, 8 * n, cudaMemcpyDeviceToHost, ctx_.stream));
      KDB_CUDA(cudaMemcpyAsync(f.data(), out_first_ + d.out_base, 8 * n, cudaMemcpyDeviceToHost, ctx_.stream));
      KDB_CUDA(cudaStreamSynchronize(ctx_.stream));
    }
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return f[a] < f[b]; });
    keys.resize(n);
    sums.resize(n);
    for (size_t i = 0; i < n; i++) {
      keys[i] = k[order[i]];
      sums[i] = s[order[i]];
    }
  }

  const BatchConfig& config() const { return cfg_; }
  int64_t total_rows() const {
    int64_t t = 0;
    for (const auto& q : host_qs_) t += q.nd + q.nf;
    return t;
  }
  int64_t total_bytes() const {
    int64_t t = 0;
    for (const auto& q : host_qs_) t += q.nd * 12 + q.nf * 20;
    return t;
  }
  int num_queries() const { return static_cast<int>(host_qs_.size()); }

 private:
  void Capture() {
    const int nq = static_cast<int>(host_qs_.size());
    cudaStream_t s = ctx_.stream;
    KDB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(slots_, 0, sizeof(unsigned long long) * std::max<int64_t>(slot_total_, 1), s);
    cudaMemsetAsync(acc_, 0, sizeof(Acc) * acc_total_, s);
    cudaMemsetAsync(out_count_, 0, sizeof(unsigned long long) * nq, s);
    cudaMemsetAsync(err_, 0, sizeof(int), s);
    BatchBuild<<<build_grid_, cfg_.block, 0, s>>>(d_qs_, nq, slots_, fanout_bits_, err_);
    BatchProbe<<<probe_grid_, cfg_.block, 0, s>>>(d_qs_, nq, slots_, fanout_bits_, acc_,
                                                   ctx_.OptStr("KDB_BATCH_LAZY_MEASURES") ? 0 : 1);
    BatchOutput<<<out_grid_, cfg_.block, 0, s>>>(d_qs_, nq, acc_, out_key_, out_sum_, out_first_, out_count_);
    cudaGraph_t g;
    KDB_CUDA(cudaStreamEndCapture(s, &g));
    KDB_CUDA(cudaGraphInstantiate(&exec_, g, 0));
    cudaGraphDestroy(g);
  }

  void Release() {
    if (exec_) cudaGraphExecDestroy(exec_);
    exec_ = nullptr;
    for (void* p : {static_cast<void*>(d_qs_), static_cast<void*>(slots_), static_cast<void*>(acc_),
                    static_cast<void*>(out_key_), static_cast<void*>(out_sum_), static_cast<void*>(out_first_),
                    static_cast<void*>(out_count_), static_cast<void*>(err_)})
      if (p) cudaFree(p);
    d_qs_ = nullptr;
    slots_ = nullptr;
    acc_ = nullptr;
    out_first_ = out_count_ = nullptr;
    out_key_ = nullptr;
    out_sum_ = nullptr;
    err_ = nullptr;
  }

  Context& ctx_;
  std::vector<QueryDesc> host_qs_;
  BatchConfig cfg_;
  int fanout_bits_ = 0;
  int build_grid_ = 0, probe_grid_ = 0, out_grid_ = 0;
  int64_t slot_total_ = 0, acc_total_ = 0;
  QueryDesc* d_qs_ = nullptr;
  unsigned long long* slots_ = nullptr;
  Acc* acc_ = nullptr;
  int32_t* out_key_ = nullptr;
  double* out_sum_ = nullptr;
  unsigned long long* out_first_ = nullptr;
  unsigned long long* out_count_ = nullptr;
  int* err_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
};

}  // namespace kdb

struct kdb_batch {
  kdb_ctx* owner;
  std::unique_ptr<kdb::Batch> b;
};

namespace {

template <typename F>
int BGuard(kdb_ctx* ctx, F&& f) {
  try {
    f();
    return KDB_OK;
  } catch (const kdb::Error& e) {
    kdb_ctx_set_error(ctx, e.what());
    return e.code;
  } catch (const std::exception& e) {
    kdb_ctx_set_error(ctx, e.what());
    return KDB_ERR_INVALID;
  }
}

}  // namespace

extern "C" {

int kdb_batch_create(kdb_ctx* ctx, const kdb_batch_query* queries, int32_t n, kdb_batch** out) {
  if (!ctx || !queries || n <= 0 || !out) return KDB_ERR_INVALID;
  *out = nullptr;
  return BGuard(ctx, [&] {
    kdb::Context& c = *kdb_ctx_context(ctx);
    if (c.dry) throw kdb::Error(KDB_ERR_UNSUPPORTED, "batches need a GPU context");
    std::vector<kdb::QueryDesc> qs(n);
    for (int i = 0; i < n; i++) {
      const kdb_batch_query& q = queries[i];
      const auto& key = c.Column(q.dim_table, q.dim_key);
      const auto& date = c.Column(q.dim_table, q.dim_date);
      const auto& seg = c.Column(q.dim_table, q.dim_seg);
      const auto& fk = c.Column(q.fact_table, q.fact_fk);
      const auto& price = c.Column(q.fact_table, q.fact_price);
      const auto& disc = c.Column(q.fact_table, q.fact_disc);
      auto i32 = [](const kdb::DevColumn& col) {
        return col.type.id == kdb::plan::TypeId::INT || col.type.id == kdb::plan::TypeId::DATE ||
               col.type.id == kdb::plan::TypeId::ENUM;
      };
      if (!i32(key) || !i32(date) || !i32(seg) || !i32(fk) || price.type.id != kdb::plan::TypeId::REAL ||
          disc.type.id != kdb::plan::TypeId::REAL)
        throw kdb::Error(KDB_ERR_INVALID, "batch template columns have the wrong types");
      if (key.nulls || date.nulls || seg.nulls || fk.nulls || price.nulls || disc.nulls)
        throw kdb::Error(KDB_ERR_UNSUPPORTED, "batch template columns must not be nullable");
      kdb::QueryDesc d{};
      d.d_key = static_cast<const int32_t*>(key.data);
      d.d_date = static_cast<const int32_t*>(date.data);
      d.d_seg = static_cast<const int32_t*>(seg.data);
      d.nd = key.n;
      d.date_lt = q.date_lt;
      d.seg = q.seg;
      d.f_fk = static_cast<const int32_t*>(fk.data);
      d.f_price = static_cast<const double*>(price.data);
      d.f_disc = static_cast<const double*>(disc.data);
      d.nf = fk.n;
      qs[i] = d;
    }
    auto b = std::make_unique<kdb_batch>();
    b->owner = ctx;
    b->b = std::make_unique<kdb::Batch>(c, std::move(qs));
    b->b->Configure(kdb::BatchConfig{});
    *out = b.release();
  });
}

int kdb_batch_configure(kdb_batch* b, int32_t block, double load_factor, int32_t fanout) {
  if (!b) return KDB_ERR_INVALID;
  return BGuard(b->owner, [&] {
    if ((block != 128 && block != 256 && block != 512) || load_factor <= 0.05 || load_factor > 0.95 ||
        fanout < 1 || fanout > 4096 || (fanout & (fanout - 1)))
      throw kdb::Error(KDB_ERR_INVALID, "bad batch configuration");
    b->b->Configure(kdb::BatchConfig{block, load_factor, fanout});
  });
}

int kdb_batch_tune(kdb_batch* b, int32_t reps, char* report, int64_t cap) {
  if (!b) return KDB_ERR_INVALID;
  return BGuard(b->owner, [&] {
    std::ostringstream o;
    o << "[";
    kdb::BatchConfig best;
    float best_ms = 1e30f;
    bool first = true;
    for (int block : {128, 256, 512})
      for (double lf : {0.5, 0.7, 0.9})
        for (int fan : {1, 64, 256, 1024}) {
          b->b->Configure(kdb::BatchConfig{block, lf, fan});
          float ms = b->b->RunTimed(std::max(1, reps));
          o << (first ? "" : ",") << "{\"block\":" << block << ",\"load_factor\":" << lf << ",\"fanout\":" << fan
            << ",\"ms\":" << ms << "}";
          first = false;
          if (ms < best_ms) {
            best_ms = ms;
            best = kdb::BatchConfig{block, lf, fan};
          }
        }
    o << "]";
    b->b->Configure(best);
    std::string s = o.str();
    if (report && cap > 0) {
      int64_t n = std::min<int64_t>(cap - 1, s.size());
      std::memcpy(report, s.data(), n);
      report[n] = 0;
    }
  });
}

int kdb_batch_run(kdb_batch* b) {
  if (!b) return KDB_ERR_INVALID;
  return BGuard(b->owner, [&] {
    b->b->Run();
    KDB_CUDA(cudaStreamSynchronize(kdb_ctx_context(b->owner)->stream));
    int e = b->b->CheckError();
    if (e == 3) throw kdb::Error(KDB_ERR_UNSUPPORTED, "batch dimension key is not unique");
    if (e == 4) throw kdb::Error(KDB_ERR_CAPACITY, "batch join table overflow");
  });
}

double kdb_batch_run_timed(kdb_batch* b, int32_t reps) {
  if (!b) return -1;
  double ms = -1;
  int rc = BGuard(b->owner, [&] { ms = b->b->RunTimed(std::max(1, reps)); });
  return rc == KDB_OK ? ms : -1;
}

int64_t kdb_batch_result(kdb_batch* b, int32_t q, int32_t* keys, double* sums, int64_t cap) {
  if (!b || q < 0 || q >= b->b->num_queries()) return KDB_ERR_INVALID;
  int64_t n = -1;
  int rc = BGuard(b->owner, [&] {
    std::vector<int32_t> k;
    std::vector<double> s;
    b->b->Result(q, k, s);
    n = static_cast<int64_t>(k.size());
    for (int64_t i = 0; i < std::min<int64_t>(n, cap); i++) {
      if (keys) keys[i] = k[i];
      if (sums) sums[i] = s[i];
    }
  });
  return rc == KDB_OK ? n : rc;
}

int kdb_batch_config(kdb_batch* b, int32_t* block, double* load_factor, int32_t* fanout) {
  if (!b) return KDB_ERR_INVALID;
  const auto& c = b->b->config();
  if (block) *block = c.block;
  if (load_factor) *load_factor = c.load_factor;
  if (fanout) *fanout = c.fanout;
  return KDB_OK;
}

void kdb_batch_free(kdb_batch* b) { delete b; }

}  // extern "C"
