// Host-side engine: device-resident tables, compiled-pipeline cache, and the
// plan executor that turns plan::Operator trees into device pipelines.
//
// Replaces, for the hot path, the reference's compile + execution layers
// (compile/query_translator.cc:16-34, execution/executable_query.cc:199-255)
// and the runtime structures its generated code calls per tuple
// (runtime/column_data, hash_table, aggregate_hash_table, vector).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "host_result.h"
#include "plan.h"

namespace kdb {

// Error with a KDB_ERR_* code.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void CudaCheck(cudaError_t e, const char* what);
#define KDB_CUDA(x) ::kdb::CudaCheck((x), #x)

// A TEXT value in a materialised buffer (same layout as device kdb_str).
struct DevStr {
  const char* p;
  int32_t len;
  int32_t pad;
};
static_assert(sizeof(DevStr) == 16, "DevStr layout");

// One HBM-resident base-table column (runtime::ColumnData equivalent).
struct DevColumn {
  plan::Type type;
  int64_t n = 0;
  void* data = nullptr;      // fixed width values
  int64_t* toff = nullptr;   // TEXT: offsets[n+1]
  char* tchars = nullptr;    // TEXT: bytes
  int8_t* nulls = nullptr;   // optional NULL flags
  size_t bytes = 0;
  int32_t max_text_len = 0;
};

struct DevTable {
  std::map<std::string, DevColumn> cols;
  int64_t rows = -1;
};

// Enum dictionary mirrored on the device; `rank[k]` is key k's position in
// string order, so ORDER BY / MIN / MAX / < on enums compare ranks
// (compile/proxy/aggregator.cc:163-171, evaluate.cc:203-250).
struct DevEnum {
  std::vector<std::string> values;
  int64_t* d_off = nullptr;
  char* d_chars = nullptr;
  int32_t* d_rank = nullptr;
  std::vector<int32_t> rank;
};

// A materialised intermediate: columnar, device resident.  TEXT columns
// hold DevStr (pointers into base columns or kernel literals).
struct MatCol {
  plan::Type type;
  bool nullable = false;
  void* data = nullptr;
  int8_t* nulls = nullptr;
};

struct MatBuffer {
  std::vector<MatCol> cols;
  uint64_t* pos = nullptr;   // stream position of each row (reference emission order key)
  bool pos_is_index = false;  // pos[r] == r: rows are already in stream order
  int64_t rows = 0;
  int64_t cap = 0;
};

// A compiled pipeline program (one CUDA module from NVRTC).
struct Program {
  CUmodule module = nullptr;
  std::map<std::string, CUfunction> fns;
  std::string log;
};

// Compiled pipelines shared by a context and its serving slots.
struct ProgramCache {
  std::mutex mu;
  std::unordered_map<std::string, std::unique_ptr<Program>> programs;
  // functions whose source starts with kGridDependencyWait (see Launch)
  std::unordered_set<CUfunction> waits;
};

// First statement of every generated kernel: wait until the grid launched
// before it in the stream has completed and its writes are visible (a no-op
// unless the kernel was launched as a programmatic dependent), then let the
// next kernel's CTAs be scheduled as this grid's CTAs finish.
constexpr const char* kGridDependencyWait =
    "  asm volatile(\"griddepcontrol.wait;\" ::: \"memory\");\n"
    "  asm volatile(\"griddepcontrol.launch_dependents;\" ::: \"memory\");\n";

// Host mirror of the device KArgs struct (passed by value).
struct KArgs {
  uint64_t w[384];
};

class Context;

// Host blocks that downloaded results own (pinned unless compile-only).  A
// block comes back to the pool when its last owner lets go; the pool keeps
// a few for the next results and frees the rest.
class HostBlockPool : public std::enable_shared_from_this<HostBlockPool> {
 public:
  explicit HostBlockPool(bool pinned) : pinned_(pinned) {}
  ~HostBlockPool();
  std::shared_ptr<char> Acquire(size_t bytes);

 private:
  static constexpr size_t kKeep = 8;  // free blocks kept for reuse
  void Release(char* p, size_t bytes);
  void FreeBlock(char* p) const;
  bool pinned_;
  std::mutex mu_;
  std::vector<std::pair<size_t, char*>> free_;
};
class JoinPrior;

// Segments gathered into one buffer for a single device-to-host copy.
constexpr int kMaxPackSegs = 32;
struct PackSeg {
  const char* src;
  uint64_t bytes;
  uint64_t off;
};
struct PackSegs {
  PackSeg seg[kMaxPackSegs];
  int n = 0;
};

// The device work of one query execution, kept to be replayed as a CUDA
// graph when the same plan runs again over unchanged tables.
struct Recorder {
  std::vector<std::function<void(cudaStream_t)>> ops;
  // per op: the kernel's role ("" for memsets), for profiled replays
  std::vector<std::string> tags;
  int64_t launches = 0;
  bool replayable = true;
};

// Stream-ordered device allocations owned by one query execution.
class Arena {
 public:
  explicit Arena(Context& ctx) : ctx_(ctx) {}
  ~Arena();
  void* Alloc(size_t bytes);
  template <typename T>
  T* AllocT(size_t count) {
    return static_cast<T*>(Alloc(count * sizeof(T) + 16));
  }
  size_t bytes() const { return bytes_; }
  // While set, allocations are made by `to` (an owner that outlives this
  // query, such as a serving build-cache entry) instead.
  void RedirectTo(Arena* to) { redirect_ = to; }

 private:
  Context& ctx_;
  std::vector<void*> ptrs_;
  size_t bytes_ = 0;
  Arena* redirect_ = nullptr;
};

// Build-side state a serving loop keeps on the device across requests
// (defined with the executor): a Skinner join child's filtered rows and its
// join-column indexes, keyed by what the child reads and filters.
struct BuildCache;
std::shared_ptr<BuildCache> MakeBuildCache(size_t max_bytes);
// hits, misses, cached bytes and entries so far
void BuildCacheStats(BuildCache& c, int64_t* hits, int64_t* misses, int64_t* bytes, int64_t* entries);

class Context {
 public:
  // device < 0: compile-only context (no GPU needed): every pipeline is
  // generated and compiled by NVRTC, nothing is allocated, copied or run,
  // and device reads return zeros.
  explicit Context(int device);
  // A serving slot: its own stream, sharing `parent`'s resident tables, enum
  // dictionaries and compiled pipelines (the parent must outlive it and must
  // not change its tables while slots run).
  explicit Context(Context& parent);
  ~Context();

  int device = 0;
  bool dry = false;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  std::map<std::string, DevTable> tables;
  std::map<int32_t, DevEnum> enums;
  std::string last_error;
  int64_t kernel_launches = 0;
  double last_device_ms = 0;
  // Skinner join: work budget per episode (tuples examined) and UCT seed
  // (runtime/skinner_join_executor.cc:20-22 budget_per_episode / join_seed)
  int64_t skinner_budget = 1 << 20;
  uint32_t skinner_seed = 0;
  int64_t last_skinner_episodes = 0;
  int64_t last_skinner_work = 0;  // tuples examined by all episodes
  int64_t last_skinner_batches = 0;  // launches of episode batches
  // Join-order policy: 0 = UCT as the reference, 1 = UCT seeded by the
  // learned prior (falls back to 0 without a model or above 8 tables),
  // 2 = uniformly random connected orders (training-data collection).
  int skinner_policy = 0;
  JoinPrior* join_prior = nullptr;
  // Serving slots: children and indexes of Skinner joins reused across
  // requests (null: every query builds its own, like the reference).
  std::shared_ptr<BuildCache> build_cache;
  // (features, reward) of every (prefix, next table) step of every episode
  // of the last Skinner join, when logging is on
  bool skinner_log = false;
  std::vector<float> skinner_features;
  std::vector<float> skinner_rewards;

  // Code-generation switches and tuning values, named KDB_* (for example
  // KDB_NO_VECTOR_SCAN, KDB_DENSE_BLOCK=128): set with kdb_ctx_set_option;
  // a context starts from the KDB_* environment variables present when it
  // is created.  Changing one drops the prepared recordings (they were
  // generated under the old values).
  std::map<std::string, std::string> options;
  const char* OptStr(const char* name) const {
    auto it = options.find(name);
    return it == options.end() ? nullptr : it->second.c_str();
  }

  // device error word shared by all launches of a query
  int* d_err = nullptr;

  // Recording (prepared-query replay): while `rec` is set, every launch and
  // memset of the query is also kept; a host-to-device copy or a Skinner
  // join makes the query not replayable.  `catalog_version` changes with
  // every table or enum change and invalidates prepared queries.
  Recorder* rec = nullptr;
  uint64_t catalog_version = 0;
  void Issue(std::function<void(cudaStream_t)> op, bool is_kernel = true) {
    kernel_launches += is_kernel;
    if (dry) return;
    op(stream);
    if (rec) {
      rec->launches += is_kernel;
      rec->ops.push_back(std::move(op));
      rec->tags.push_back(is_kernel ? cur_tag_ : std::string());
    }
  }
  // a retried step drops what its failed attempt recorded
  std::pair<size_t, int64_t> RecordMark() const {
    return rec ? std::make_pair(rec->ops.size(), rec->launches) : std::make_pair(size_t(0), int64_t(0));
  }
  void RecordTruncate(const std::pair<size_t, int64_t>& mark) {
    if (rec && rec->ops.size() > mark.first) {
      rec->ops.resize(mark.first);
      rec->tags.resize(mark.first);
      rec->launches = mark.second;
    }
  }
  void NotReplayable() {
    if (rec) rec->replayable = false;
  }

  void AddColumn(const std::string& table, const std::string& column, const plan::Type& type,
                 const void* data, int64_t n, const int8_t* nulls);
  // A fixed-width column in host memory to bring into HBM.
  struct HostColumnSpec {
    std::string table, column;
    plan::Type type;
    const void* data = nullptr;
    int64_t n = 0;
    const int8_t* nulls = nullptr;
  };
  // Adds or refreshes fixed-width columns from host memory with every copy
  // split into chunks spread over the copy streams, all in flight together
  // (no synchronisation between columns); the context's stream waits for
  // all of them, so work issued on it afterwards sees the new contents.
  // The host memory must stay unchanged until that work has run (pinned
  // memory copies asynchronously; pageable memory is copied before the
  // call returns).  Returns the bytes copied.
  int64_t StreamColumns(const std::vector<HostColumnSpec>& cols);
  // Chunk size and number of copy streams used by StreamColumns.
  int64_t ingest_chunk_bytes = int64_t(64) << 20;
  int ingest_streams = 2;
  void AddTextColumn(const std::string& table, const std::string& column, const int64_t* offsets,
                     const char* chars, int64_t n, const int8_t* nulls);
  // A reference TEXT .kdb file's bytes (runtime/column_data.h:45-57:
  // StringMetadata {int32 cardinality; {int32 length; uint64 offset}[]}, then
  // the strings): the metadata is checked on the host against the file
  // size, the file goes to HBM in one copy, and the device decodes it into
  // the column's offsets and bytes (a scan of the lengths, one gather).
  void AddTextColumnFromKdb(const std::string& table, const std::string& column, const char* raw,
                            size_t size, const int8_t* nulls, int64_t null_rows);
  void DropTable(const std::string& table);
  void RegisterEnum(int32_t id, std::vector<std::string> values);
  int64_t ColumnBytes() const;

  const DevColumn& Column(const std::string& table, const std::string& column) const;
  const DevEnum& Enum(int32_t id) const;

  // NVRTC compile (cached by source text) and kernel lookup.
  CUfunction Kernel(const std::string& source, const std::string& name);
  void Launch(CUfunction f, int grid, int block, const KArgs& args, size_t smem = 0,
              const char* tag = "pipeline");
  // Per-launch CUDA-event timing (enabled by kdb_ctx_set_profiling).
  bool profile = false;
  struct LaunchTiming {
    std::string tag;
    cudaEvent_t start, stop;
  };
  std::vector<LaunchTiming> timings;
  // the role of the kernels issued between TimedStart and TimedStop
  std::string cur_tag_;
  std::vector<std::pair<std::string, float>> last_kernels;
  void BeginQueryProfile();
  void EndQueryProfile();
  // Queues a kernel that spins on the SM clock for about `us` microseconds
  // (a bounded cycle count; it touches no memory): profiled replays queue
  // their launches behind it.
  void DelayStream(double us);
  // the two events that time each query (made on first use)
  void QueryEvents(cudaEvent_t* start, cudaEvent_t* end);
  void TimedStart(const char* tag);
  void TimedStop();
  int GridFor(int64_t n, int block) const;

  // Device memory / copies that honour the compile-only mode.
  void* DevAlloc(size_t bytes);
  void DevFree(void* p);
  void Memset(void* d, int v, size_t bytes);
  void H2D(void* d, const void* h, size_t bytes);
  void D2H(void* h, const void* d, size_t bytes);  // synchronous
  // Pinned host staging buffer of at least `bytes` (reused across queries).
  void* HostStage(size_t bytes);
  // Pinned host block of at least `bytes` for a downloaded result: the
  // result keeps it until it is freed, then it returns to the context's pool
  // (no host copy of the columns, no pinned allocation per query).
  std::shared_ptr<char> AcquireHostBlock(size_t bytes);
  // Puts `count` blocks of `bytes` into the pool ahead of use (a pinned
  // allocation synchronises with the device).
  void ReserveHostBlocks(int count, size_t bytes);

  // Static kernels (kernels.cu).
  void RadixSortPairs(uint64_t* keys, uint32_t* vals, int64_t n, Arena& arena, int key_bits = 64);
  // sorts n < 2^31 16-byte items {uint64 key, uint32 tie, uint32 value} by
  // (key, tie) (block sort + merge-path passes; items equal in (key, tie)
  // come out in no particular order)
  void MergeSortItems(void* items, int64_t n, Arena& arena);
  // the same order by a sample sort (splitters, one bucketing pass, one
  // shared-memory sort per bucket); false, with the items untouched, when a
  // bucket came out too large (the caller then merge sorts)
  bool SampleSortItems(void* items, int64_t n, Arena& arena);
  // (key, tie) order by key-range buckets; false (nothing done) when a
  // bucket is too large for one CTA's shared memory
  // With `ties` (zeroed by the caller), also counts the items whose key
  // (and tie bits under `tie_mask`) another item shares.
  // With `key_range` (min and max of the items' keys, already on the
  // device), no pass computes it.
  bool RangeSortItems(void* items, int64_t n, Arena& arena, unsigned long long* ties = nullptr,
                      uint32_t tie_mask = 0, const unsigned long long* key_range = nullptr);
  // exclusive prefix sum of a[0..n) in place, the total into a[n]
  void ScanU64(uint64_t* a, int64_t n, const char* tag = "skinner scan");
  // the same over *n_ptr elements (a device word), skipped when *n_ptr > cap
  void ScanU64Bounded(uint64_t* a, const uint64_t* n_ptr, int64_t cap, const char* tag = "skinner scan");
  // gathers the segments into the device staging buffer and queues one copy
  // of `total` bytes to `host` (pinned); the caller synchronises
  void PackToHost(const PackSegs& segs, size_t total, void* host);
  // device decode of a TEXT .kdb image at d_raw (kernels.cu)
  void DecodeKdbText(const char* d_raw, int64_t n, int64_t* toff, char* tchars);
  void CheckDeviceError(const char* what);

  EnumDicts HostEnums() const;

 private:
  std::shared_ptr<ProgramCache> cache_ = std::make_shared<ProgramCache>();
  cudaEvent_t query_ev_[2] = {nullptr, nullptr};
  bool owns_catalog_ = true;
  void* stage_ = nullptr;
  size_t stage_bytes_ = 0;
  std::shared_ptr<HostBlockPool> host_blocks_;
  void* dev_stage_ = nullptr;  // device side of PackToHost
  size_t dev_stage_bytes_ = 0;
  std::vector<cudaStream_t> copy_streams_;  // StreamColumns
  std::vector<cudaEvent_t> copy_events_;
  cudaEvent_t copy_start_ = nullptr;
  void FreeColumn(DevColumn& c);
};

// A plan executed once and kept for replay: its device buffers, the CUDA
// graph of its launches, and the location of its result.
struct PreparedQuery {
  std::unique_ptr<Arena> arena;
  cudaGraphExec_t exec = nullptr;
  // the recorded launches and memsets: a replay issues them one by one
  // instead of launching the graph when that measured faster at prepare
  // time (a short query pays the graph launch's fixed latency)
  std::vector<std::function<void(cudaStream_t)>> ops;
  std::vector<std::string> tags;  // per op, as recorded
  bool direct = false;
  MatBuffer result;
  uint64_t catalog_version = 0;
  int64_t launches = 0;
  void Replay(cudaStream_t s) const;
  ~PreparedQuery();
};

// Runs a plan on the device and returns the host result.  With `prepared`,
// the first run of a plan records it, and later runs over unchanged tables
// replay the recorded graph (no code generation, one graph launch).
HostResult ExecutePlan(Context& ctx, const plan::Operator& root,
                       std::unique_ptr<PreparedQuery>* prepared = nullptr);

}  // namespace kdb
