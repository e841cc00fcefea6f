// Context: device residency of columns and enums, the NVRTC pipeline cache
// and kernel launch plumbing.
#include "engine.h"

#include <nvrtc.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>

namespace kdb {

namespace {

const char* kDeviceRuntime =
#include "device_runtime.inc"
    ;

// Driver API entry points, resolved through the runtime so the library does
// not link libcuda directly (it must load on machines without a driver).
struct Driver {
  CUresult (*ModuleLoadData)(CUmodule*, const void*) = nullptr;
  CUresult (*ModuleGetFunction)(CUfunction*, CUmodule, const char*) = nullptr;
  CUresult (*LaunchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                           unsigned, CUstream, void**, void**) = nullptr;
  CUresult (*ModuleUnload)(CUmodule) = nullptr;
  CUresult (*FuncSetAttribute)(CUfunction, CUfunction_attribute, int) = nullptr;
  CUresult (*LaunchKernelEx)(const CUlaunchConfig*, CUfunction, void**, void**) = nullptr;
  bool loaded = false;

  template <typename F>
  void Get(const char* name, F& fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    KDB_CUDA(cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q));
    if (!p || q != cudaDriverEntryPointSuccess)
      throw Error(-2, std::string("driver entry point missing: ") + name);
    fn = reinterpret_cast<F>(p);
  }
  void Load() {
    if (loaded) return;
    Get("cuModuleLoadData", ModuleLoadData);
    Get("cuModuleGetFunction", ModuleGetFunction);
    Get("cuLaunchKernel", LaunchKernel);
    Get("cuModuleUnload", ModuleUnload);
    Get("cuFuncSetAttribute", FuncSetAttribute);
    // optional: without it every kernel launches in plain stream order
    void* ex = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuLaunchKernelEx", &ex, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess && ex)
      LaunchKernelEx = reinterpret_cast<decltype(LaunchKernelEx)>(ex);
    else
      cudaGetLastError();
    loaded = true;
  }
};
Driver g_drv;

void CuCheck(CUresult r, const char* what) {
  if (r != CUDA_SUCCESS) throw Error(-2, std::string(what) + " failed (CUresult " + std::to_string(r) + ")");
}

void NvrtcCheck(nvrtcResult r, const char* what) {
  if (r != NVRTC_SUCCESS) throw Error(-3, std::string(what) + ": " + nvrtcGetErrorString(r));
}

}  // namespace

void CudaCheck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(-2, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// Arena
// ---------------------------------------------------------------------------

Arena::~Arena() {
  if (ctx_.dry) return;
  for (void* p : ptrs_) cudaFreeAsync(p, ctx_.stream);
}

void* Arena::Alloc(size_t bytes) {
  if (redirect_) return redirect_->Alloc(bytes);
  if (bytes == 0) bytes = 16;
  if (ctx_.dry) return ctx_.DevAlloc(bytes);
  void* p = nullptr;
  KDB_CUDA(cudaMallocAsync(&p, bytes, ctx_.stream));
  ptrs_.push_back(p);
  bytes_ += bytes;
  return p;
}

namespace {
uint64_t g_fake_next = 0x7f0000000000ULL;
}

void* Context::DevAlloc(size_t bytes) {
  if (dry) {
    void* p = reinterpret_cast<void*>(g_fake_next);
    g_fake_next += (bytes + 255) & ~size_t(255);
    return p;
  }
  void* p = nullptr;
  KDB_CUDA(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
  return p;
}

void Context::DevFree(void* p) {
  if (!dry && p) cudaFree(p);
}

void Context::Memset(void* d, int v, size_t bytes) {
  if (dry || !bytes) return;
  KDB_CUDA(cudaMemsetAsync(d, v, bytes, stream));
  if (rec) {
    rec->ops.push_back([d, v, bytes](cudaStream_t s) { cudaMemsetAsync(d, v, bytes, s); });
    rec->tags.emplace_back();
  }
}

void Context::H2D(void* d, const void* h, size_t bytes) {
  NotReplayable();
  if (!dry && bytes) KDB_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, stream));
}

void Context::D2H(void* h, const void* d, size_t bytes) {
  if (dry) {
    std::memset(h, 0, bytes);
    return;
  }
  if (bytes) KDB_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, stream));
  KDB_CUDA(cudaStreamSynchronize(stream));
}

void* Context::HostStage(size_t bytes) {
  if (bytes <= stage_bytes_ && stage_) return stage_;
  size_t want = std::max<size_t>(bytes, 1 << 20);
  if (dry) {
    std::free(stage_);
    stage_ = std::malloc(want);
  } else {
    if (stage_) cudaFreeHost(stage_);
    KDB_CUDA(cudaMallocHost(&stage_, want));
  }
  stage_bytes_ = want;
  return stage_;
}

HostBlockPool::~HostBlockPool() {
  for (auto& b : free_) FreeBlock(b.second);
}

void HostBlockPool::FreeBlock(char* p) const {
  if (pinned_) cudaFreeHost(p);
  else std::free(p);
}

std::shared_ptr<char> HostBlockPool::Acquire(size_t bytes) {
  char* p = nullptr;
  size_t size = 0;
  {
    std::lock_guard<std::mutex> g(mu_);
    size_t best = free_.size();
    for (size_t i = 0; i < free_.size(); i++)
      if (free_[i].first >= bytes && (best == free_.size() || free_[i].first < free_[best].first)) best = i;
    if (best < free_.size()) {
      size = free_[best].first;
      p = free_[best].second;
      free_.erase(free_.begin() + best);
    }
  }
  if (!p) {
    size = size_t(1) << 20;
    while (size < bytes) size <<= 1;
    if (pinned_) {
      void* h = nullptr;
      // mapped: small results are written into the block by a kernel
      KDB_CUDA(cudaHostAlloc(&h, size, cudaHostAllocMapped));
      p = static_cast<char*>(h);
    } else {
      p = static_cast<char*>(std::malloc(size));
      if (!p) throw Error(-3, "host allocation failed");
    }
  }
  std::weak_ptr<HostBlockPool> pool = shared_from_this();
  const bool pinned = pinned_;
  return std::shared_ptr<char>(p, [pool, size, pinned](char* q) {
    if (auto live = pool.lock()) live->Release(q, size);
    else if (pinned) cudaFreeHost(q);
    else std::free(q);
  });
}

void HostBlockPool::Release(char* p, size_t bytes) {
  {
    std::lock_guard<std::mutex> g(mu_);
    if (free_.size() < kKeep) {
      free_.emplace_back(bytes, p);
      return;
    }
  }
  FreeBlock(p);
}

std::shared_ptr<char> Context::AcquireHostBlock(size_t bytes) {
  if (!host_blocks_) host_blocks_ = std::make_shared<HostBlockPool>(!dry);
  return host_blocks_->Acquire(bytes);
}

void Context::ReserveHostBlocks(int count, size_t bytes) {
  std::vector<std::shared_ptr<char>> held;
  for (int i = 0; i < count; i++) held.push_back(AcquireHostBlock(bytes));
}

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------

extern "C" char** environ;

namespace {
// the KDB_* environment variables, as a context's initial options
std::map<std::string, std::string> OptionsFromEnvironment() {
  std::map<std::string, std::string> o;
  for (char** e = environ; e && *e; e++) {
    const char* kv = *e;
    if (std::strncmp(kv, "KDB_", 4) != 0) continue;
    const char* eq = std::strchr(kv, '=');
    if (eq) o.emplace(std::string(kv, eq - kv), std::string(eq + 1));
  }
  return o;
}
}  // namespace

Context::Context(int dev) : device(dev) {
  options = OptionsFromEnvironment();
  if (dev < 0) {
    dry = true;
    d_err = static_cast<int*>(DevAlloc(16));
    return;
  }
  KDB_CUDA(cudaSetDevice(dev));
  KDB_CUDA(cudaFree(nullptr));
  KDB_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
  KDB_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  // keep freed stream-ordered memory in the pool between queries
  cudaMemPool_t pool;
  KDB_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
  uint64_t threshold = UINT64_MAX;
  KDB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
  KDB_CUDA(cudaMalloc(&d_err, sizeof(int) * 4));
  KDB_CUDA(cudaMemset(d_err, 0, sizeof(int) * 4));
  g_drv.Load();
}

Context::Context(Context& parent)
    : device(parent.device), dry(parent.dry), num_sms(parent.num_sms), tables(parent.tables),
      enums(parent.enums), skinner_budget(parent.skinner_budget), skinner_seed(parent.skinner_seed),
      skinner_policy(parent.skinner_policy), join_prior(parent.join_prior), options(parent.options),
      cache_(parent.cache_), owns_catalog_(false) {
  if (dry) {
    d_err = static_cast<int*>(DevAlloc(16));
    return;
  }
  KDB_CUDA(cudaSetDevice(device));
  KDB_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  KDB_CUDA(cudaMalloc(&d_err, sizeof(int) * 4));
  KDB_CUDA(cudaMemset(d_err, 0, sizeof(int) * 4));
}

Context::~Context() {
  if (dry) {
    std::free(stage_);
    return;
  }
  for (cudaStream_t cs : copy_streams_) cudaStreamSynchronize(cs);
  for (cudaStream_t cs : copy_streams_) cudaStreamDestroy(cs);
  for (cudaEvent_t e : copy_events_) cudaEventDestroy(e);
  if (copy_start_) cudaEventDestroy(copy_start_);
  if (stage_) cudaFreeHost(stage_);
  cudaSetDevice(device);
  for (cudaEvent_t e : query_ev_)
    if (e) cudaEventDestroy(e);
  if (dev_stage_) cudaFreeAsync(dev_stage_, stream);
  cudaStreamSynchronize(stream);
  if (owns_catalog_) {
    for (auto& [n, t] : tables)
      for (auto& [cn, c] : t.cols) FreeColumn(c);
    for (auto& [id, e] : enums) {
      cudaFree(e.d_off);
      cudaFree(e.d_chars);
      cudaFree(e.d_rank);
    }
  }
  if (cache_.use_count() == 1)
    for (auto& [k, p] : cache_->programs)
      if (p->module) g_drv.ModuleUnload(p->module);
  cudaFree(d_err);
  cudaStreamDestroy(stream);
}

void Context::FreeColumn(DevColumn& c) {
  DevFree(c.data);
  DevFree(c.toff);
  DevFree(c.tchars);
  DevFree(c.nulls);
  c = DevColumn();
}

static void CheckRows(DevTable& t, int64_t n, const std::string& name) {
  if (t.rows >= 0 && t.rows != n)
    throw Error(-1, "column " + name + " has " + std::to_string(n) + " rows, table has " +
                        std::to_string(t.rows));
  t.rows = n;
}

void Context::AddColumn(const std::string& table, const std::string& column, const plan::Type& type,
                        const void* data, int64_t n, const int8_t* nulls) {
  catalog_version++;
  if (type.id == plan::TypeId::TEXT) throw Error(-1, "TEXT columns use kdb_table_add_text_column");
  if (n < 0) throw Error(-1, "negative row count");
  DevTable& t = tables[table];
  CheckRows(t, n, column);
  auto it = t.cols.find(column);
  size_t w = plan::TypeWidth(type.id);
  if (it != t.cols.end()) {
    DevColumn& old = it->second;
    if (old.type == type && old.n == n && (old.nulls != nullptr) == (nulls != nullptr)) {
      // same shape: refresh the resident buffers in place
      H2D(old.data, data, w * n);
      if (nulls) H2D(old.nulls, nulls, n);
      if (!dry) KDB_CUDA(cudaStreamSynchronize(stream));
      return;
    }
    FreeColumn(old);
  }
  DevColumn c;
  c.type = type;
  c.n = n;
  c.bytes = w * n;
  c.data = DevAlloc(std::max<size_t>(c.bytes, 16));
  H2D(c.data, data, c.bytes);
  if (nulls) {
    c.nulls = static_cast<int8_t*>(DevAlloc(std::max<int64_t>(n, 16)));
    H2D(c.nulls, nulls, n);
    c.bytes += n;
  }
  if (!dry) KDB_CUDA(cudaStreamSynchronize(stream));
  t.cols[column] = c;
}

int64_t Context::StreamColumns(const std::vector<HostColumnSpec>& cols) {
  catalog_version++;
  struct Copy {
    void* dst;
    const char* src;
    size_t bytes;
  };
  std::vector<Copy> copies;
  for (const auto& spec : cols) {
    if (spec.type.id == plan::TypeId::TEXT) throw Error(-1, "TEXT columns use kdb_table_add_text_column");
    if (spec.n < 0 || (spec.n > 0 && !spec.data)) throw Error(-1, "bad host column " + spec.column);
    DevTable& t = tables[spec.table];
    CheckRows(t, spec.n, spec.column);
    const size_t w = plan::TypeWidth(spec.type.id);
    auto it = t.cols.find(spec.column);
    DevColumn* c = nullptr;
    if (it != t.cols.end() && it->second.type == spec.type && it->second.n == spec.n &&
        (it->second.nulls != nullptr) == (spec.nulls != nullptr)) {
      c = &it->second;  // same shape: refreshed in place
    } else {
      if (it != t.cols.end()) {
        if (!dry) KDB_CUDA(cudaStreamSynchronize(stream));
        FreeColumn(it->second);
      }
      DevColumn nc;
      nc.type = spec.type;
      nc.n = spec.n;
      nc.bytes = w * spec.n;
      nc.data = DevAlloc(std::max<size_t>(nc.bytes, 16));
      if (spec.nulls) {
        nc.nulls = static_cast<int8_t*>(DevAlloc(std::max<int64_t>(spec.n, 16)));
        nc.bytes += spec.n;
      }
      t.cols[spec.column] = nc;
      c = &t.cols[spec.column];
    }
    if (w * spec.n) copies.push_back({c->data, static_cast<const char*>(spec.data), w * spec.n});
    if (spec.nulls && spec.n) copies.push_back({c->nulls, reinterpret_cast<const char*>(spec.nulls),
                                                static_cast<size_t>(spec.n)});
  }
  int64_t total = 0;
  for (const auto& cp : copies) total += static_cast<int64_t>(cp.bytes);
  if (dry || copies.empty()) return total;
  const int ns = std::max(1, std::min(ingest_streams, 8));
  while (static_cast<int>(copy_streams_.size()) < ns) {
    cudaStream_t cs;
    cudaEvent_t ev;
    KDB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    KDB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    copy_streams_.push_back(cs);
    copy_events_.push_back(ev);
  }
  if (!copy_start_) KDB_CUDA(cudaEventCreateWithFlags(&copy_start_, cudaEventDisableTiming));
  // the copies start after the work already queued on the context's stream
  // (which may still read the columns being refreshed)
  KDB_CUDA(cudaEventRecord(copy_start_, stream));
  for (int i = 0; i < ns; i++) KDB_CUDA(cudaStreamWaitEvent(copy_streams_[i], copy_start_, 0));
  const size_t chunk = static_cast<size_t>(std::max<int64_t>(ingest_chunk_bytes, 1 << 16));
  int next = 0;
  for (const auto& cp : copies) {
    for (size_t off = 0; off < cp.bytes; off += chunk) {
      const size_t b = std::min(chunk, cp.bytes - off);
      KDB_CUDA(cudaMemcpyAsync(static_cast<char*>(cp.dst) + off, cp.src + off, b, cudaMemcpyHostToDevice,
                               copy_streams_[next]));
      next = (next + 1) % ns;
    }
  }
  for (int i = 0; i < ns; i++) {
    KDB_CUDA(cudaEventRecord(copy_events_[i], copy_streams_[i]));
    KDB_CUDA(cudaStreamWaitEvent(stream, copy_events_[i], 0));
  }
  return total;
}

void Context::AddTextColumn(const std::string& table, const std::string& column,
                            const int64_t* offsets, const char* chars, int64_t n,
                            const int8_t* nulls) {
  catalog_version++;
  if (n < 0) throw Error(-1, "negative row count");
  DevTable& t = tables[table];
  CheckRows(t, n, column);
  auto it = t.cols.find(column);
  if (it != t.cols.end()) FreeColumn(it->second);
  DevColumn c;
  c.type = plan::Type{plan::TypeId::TEXT, 0};
  c.n = n;
  int64_t nbytes = offsets[n] - offsets[0];
  std::vector<int64_t> off(offsets, offsets + n + 1);
  int64_t base = off[0];
  for (auto& o : off) o -= base;
  for (int64_t r = 0; r < n; r++)
    c.max_text_len = std::max<int32_t>(c.max_text_len, static_cast<int32_t>(off[r + 1] - off[r]));
  c.toff = static_cast<int64_t*>(DevAlloc(sizeof(int64_t) * (n + 1)));
  H2D(c.toff, off.data(), sizeof(int64_t) * (n + 1));
  c.tchars = static_cast<char*>(DevAlloc(std::max<int64_t>(nbytes, 16)));
  H2D(c.tchars, chars + base, nbytes);
  c.bytes = sizeof(int64_t) * (n + 1) + nbytes;
  if (nulls) {
    c.nulls = static_cast<int8_t*>(DevAlloc(std::max<int64_t>(n, 16)));
    H2D(c.nulls, nulls, n);
    c.bytes += n;
  }
  if (!dry) KDB_CUDA(cudaStreamSynchronize(stream));
  t.cols[column] = c;
}

void Context::AddTextColumnFromKdb(const std::string& table, const std::string& column, const char* raw,
                                   size_t size, const int8_t* nulls, int64_t null_rows) {
  if (size < 8) throw Error(-1, "short TEXT file");
  int32_t card;
  std::memcpy(&card, raw, 4);
  if (card < 0) throw Error(-1, "TEXT file with a negative cardinality");
  const uint64_t meta_end = 8 + 16 * static_cast<uint64_t>(card);
  if (meta_end > size) throw Error(-1, "TEXT file shorter than its metadata");
  if (nulls && null_rows != card) throw Error(-1, "null file length differs from column length");
  int32_t max_len = 0;
  uint64_t nbytes = 0;
  for (int32_t r = 0; r < card; r++) {
    int32_t len;
    uint64_t o;
    std::memcpy(&len, raw + 8 + 16 * static_cast<uint64_t>(r), 4);
    std::memcpy(&o, raw + 8 + 16 * static_cast<uint64_t>(r) + 8, 8);
    if (len < 0 || o < meta_end || o > size || static_cast<uint64_t>(len) > size - o)
      throw Error(-1, "corrupt TEXT file (slot " + std::to_string(r) + ")");
    max_len = std::max(max_len, len);
    nbytes += static_cast<uint64_t>(len);
  }
  catalog_version++;
  DevTable& t = tables[table];
  CheckRows(t, card, column);
  auto it = t.cols.find(column);
  if (it != t.cols.end()) {
    if (!dry) KDB_CUDA(cudaStreamSynchronize(stream));
    FreeColumn(it->second);
  }
  DevColumn c;
  c.type = plan::Type{plan::TypeId::TEXT, 0};
  c.n = card;
  c.max_text_len = max_len;
  c.toff = static_cast<int64_t*>(DevAlloc(sizeof(int64_t) * (card + 1)));
  c.tchars = static_cast<char*>(DevAlloc(std::max<uint64_t>(nbytes, 16)));
  c.bytes = sizeof(int64_t) * (card + 1) + nbytes;
  if (!dry && card > 0) {
    void* d_raw = nullptr;
    KDB_CUDA(cudaMallocAsync(&d_raw, size, stream));
    KDB_CUDA(cudaMemcpyAsync(d_raw, raw, size, cudaMemcpyHostToDevice, stream));
    DecodeKdbText(static_cast<const char*>(d_raw), card, c.toff, c.tchars);
    KDB_CUDA(cudaFreeAsync(d_raw, stream));
  } else if (!dry) {
    Memset(c.toff, 0, sizeof(int64_t));
  }
  if (nulls) {
    c.nulls = static_cast<int8_t*>(DevAlloc(std::max<int64_t>(card, 16)));
    H2D(c.nulls, nulls, card);
    c.bytes += card;
  }
  if (!dry) KDB_CUDA(cudaStreamSynchronize(stream));
  t.cols[column] = c;
}

void Context::DropTable(const std::string& table) {
  catalog_version++;
  auto it = tables.find(table);
  if (it == tables.end()) return;
  if (!dry) KDB_CUDA(cudaStreamSynchronize(stream));
  for (auto& [n, c] : it->second.cols) FreeColumn(c);
  tables.erase(it);
}

void Context::RegisterEnum(int32_t id, std::vector<std::string> values) {
  catalog_version++;
  auto it = enums.find(id);
  if (it != enums.end()) {
    if (it->second.values == values) return;
    DevFree(it->second.d_off);
    DevFree(it->second.d_chars);
    DevFree(it->second.d_rank);
    enums.erase(it);
  }
  DevEnum e;
  e.values = std::move(values);
  int32_t n = static_cast<int32_t>(e.values.size());
  std::vector<int64_t> off(n + 1, 0);
  std::string chars;
  for (int32_t k = 0; k < n; k++) {
    chars += e.values[k];
    off[k + 1] = static_cast<int64_t>(chars.size());
  }
  std::vector<int32_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int32_t a, int32_t b) { return e.values[a] < e.values[b]; });
  e.rank.assign(n, 0);
  for (int32_t r = 0; r < n; r++) e.rank[order[r]] = r;
  e.d_off = static_cast<int64_t*>(DevAlloc(sizeof(int64_t) * (n + 1)));
  H2D(e.d_off, off.data(), sizeof(int64_t) * (n + 1));
  e.d_chars = static_cast<char*>(DevAlloc(std::max<size_t>(chars.size(), 16)));
  H2D(e.d_chars, chars.data(), chars.size());
  e.d_rank = static_cast<int32_t*>(DevAlloc(sizeof(int32_t) * std::max(n, 1)));
  H2D(e.d_rank, e.rank.data(), sizeof(int32_t) * n);
  if (!dry) KDB_CUDA(cudaStreamSynchronize(stream));
  enums[id] = std::move(e);
}

int64_t Context::ColumnBytes() const {
  int64_t b = 0;
  for (auto& [n, t] : tables)
    for (auto& [cn, c] : t.cols) b += static_cast<int64_t>(c.bytes);
  return b;
}

const DevColumn& Context::Column(const std::string& table, const std::string& column) const {
  auto t = tables.find(table);
  if (t == tables.end()) throw Error(-1, "unknown relation " + table);
  auto c = t->second.cols.find(column);
  if (c == t->second.cols.end()) throw Error(-1, "unknown column " + table + "." + column);
  return c->second;
}

const DevEnum& Context::Enum(int32_t id) const {
  auto it = enums.find(id);
  if (it == enums.end()) throw Error(-1, "enum " + std::to_string(id) + " not registered");
  return it->second;
}

EnumDicts Context::HostEnums() const {
  EnumDicts d;
  for (auto& [id, e] : enums) d[id] = e.values;
  return d;
}

CUfunction Context::Kernel(const std::string& source, const std::string& name) {
  std::lock_guard<std::mutex> lock(cache_->mu);
  auto& programs_ = cache_->programs;
  auto it = programs_.find(source);
  if (it == programs_.end()) {
    auto prog = std::make_unique<Program>();
    std::string full = std::string(kDeviceRuntime) + "\n" + source;
    if (const char* dir = std::getenv("KDB_DUMP_DIR")) {
      // debugging aid: keep every generated pipeline source
      std::ofstream(std::string(dir) + "/pipeline_" + std::to_string(programs_.size()) + ".cu") << source;
    }
    nvrtcProgram p;
    NvrtcCheck(nvrtcCreateProgram(&p, full.c_str(), "kdb_pipeline.cu", 0, nullptr, nullptr),
               "nvrtcCreateProgram");
    const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "--fmad=false",
                          "-lineinfo", "-DNDEBUG"};
    nvrtcResult cr = nvrtcCompileProgram(p, 5, opts);
    size_t log_size = 0;
    nvrtcGetProgramLogSize(p, &log_size);
    std::string log(log_size, '\0');
    if (log_size) nvrtcGetProgramLog(p, &log[0]);
    if (cr != NVRTC_SUCCESS) {
      nvrtcDestroyProgram(&p);
      if (const char* dump = std::getenv("KDB_DUMP_FAILED_SOURCE")) {
        std::ofstream(dump) << full;
      }
      throw Error(-3, "NVRTC compile failed: " + log.substr(0, 4000));
    }
    size_t cubin_size = 0;
    NvrtcCheck(nvrtcGetCUBINSize(p, &cubin_size), "nvrtcGetCUBINSize");
    std::vector<char> cubin(cubin_size);
    NvrtcCheck(nvrtcGetCUBIN(p, cubin.data()), "nvrtcGetCUBIN");
    nvrtcDestroyProgram(&p);
    if (!dry) CuCheck(g_drv.ModuleLoadData(&prog->module, cubin.data()), "cuModuleLoadData");
    prog->log = log;
    it = programs_.emplace(source, std::move(prog)).first;
  }
  Program& prog = *it->second;
  if (dry) return nullptr;
  auto f = prog.fns.find(name);
  if (f == prog.fns.end()) {
    CUfunction fn;
    CuCheck(g_drv.ModuleGetFunction(&fn, prog.module, name.c_str()), "cuModuleGetFunction");
    f = prog.fns.emplace(name, fn).first;
    // a kernel whose first statement waits for the preceding grid may be
    // launched before that grid has finished (programmatic dependent launch)
    if (source.find(kGridDependencyWait) != std::string::npos) cache_->waits.insert(fn);
  }
  return f->second;
}

namespace {

// One kernel launch; `pdl`: with programmatic stream serialization, so the
// kernel's CTAs may be scheduled while the previous kernel in the stream
// drains (they wait at their first statement until it has completed and
// its memory is visible).
CUresult LaunchOne(CUfunction f, int grid, int block, size_t smem, CUstream s, void** params, bool pdl) {
  if (!pdl || !g_drv.LaunchKernelEx)
    return g_drv.LaunchKernel(f, grid, 1, 1, block, 1, 1, static_cast<unsigned>(smem), s, params, nullptr);
  CUlaunchAttribute attr;
  std::memset(&attr, 0, sizeof(attr));
  attr.id = CU_LAUNCH_ATTRIBUTE_PROGRAMMATIC_STREAM_SERIALIZATION;
  attr.value.programmaticStreamSerializationAllowed = 1;
  CUlaunchConfig cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  cfg.gridDimX = static_cast<unsigned>(grid);
  cfg.gridDimY = cfg.gridDimZ = 1;
  cfg.blockDimX = static_cast<unsigned>(block);
  cfg.blockDimY = cfg.blockDimZ = 1;
  cfg.sharedMemBytes = static_cast<unsigned>(smem);
  cfg.hStream = s;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  return g_drv.LaunchKernelEx(&cfg, f, params, nullptr);
}

}  // namespace

int Context::GridFor(int64_t n, int block) const {
  int64_t want = (n + block - 1) / block;
  int64_t cap = static_cast<int64_t>(num_sms) * (2048 / block);
  return static_cast<int>(std::max<int64_t>(1, std::min(want, cap)));
}

void Context::Launch(CUfunction f, int grid, int block, const KArgs& args, size_t smem,
                     const char* tag) {
  kernel_launches++;
  if (dry) return;
  void* params[] = {const_cast<KArgs*>(&args)};
  // static plus dynamic shared memory above 48 KB needs the opt-in, also
  // when the dynamic part alone is smaller
  if (smem > 0)
    CuCheck(g_drv.FuncSetAttribute(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES,
                                   static_cast<int>(smem)),
            "cuFuncSetAttribute");
  // profiling runs time every kernel between two events: launched one
  // after the other, without programmatic overlap
  bool pdl = false;
  if (!OptStr("KDB_NO_PDL") && !profile) {
    std::lock_guard<std::mutex> lock(cache_->mu);
    pdl = cache_->waits.count(f) != 0;
  }
  TimedStart(tag);
  CuCheck(LaunchOne(f, grid, block, smem, reinterpret_cast<CUstream>(stream), params, pdl), "cuLaunchKernel");
  TimedStop();
  if (rec) {
    rec->launches++;
    auto held = std::make_shared<KArgs>(args);
    rec->ops.push_back([f, grid, block, smem, held, pdl](cudaStream_t s) {
      void* p[] = {held.get()};
      LaunchOne(f, grid, block, smem, reinterpret_cast<CUstream>(s), p, pdl);
    });
    rec->tags.emplace_back(tag ? tag : "");
  }
}

void Context::QueryEvents(cudaEvent_t* start, cudaEvent_t* end) {
  for (cudaEvent_t& e : query_ev_)
    if (!e) KDB_CUDA(cudaEventCreate(&e));
  *start = query_ev_[0];
  *end = query_ev_[1];
}

void Context::TimedStart(const char* tag) {
  cur_tag_ = tag ? tag : "";
  if (!profile || dry) return;
  LaunchTiming t;
  t.tag = tag;
  KDB_CUDA(cudaEventCreate(&t.start));
  KDB_CUDA(cudaEventCreate(&t.stop));
  KDB_CUDA(cudaEventRecord(t.start, stream));
  timings.push_back(t);
}

void Context::TimedStop() {
  cur_tag_.clear();
  if (!profile || dry || timings.empty()) return;
  KDB_CUDA(cudaEventRecord(timings.back().stop, stream));
}

void Context::BeginQueryProfile() {
  for (auto& t : timings) {
    cudaEventDestroy(t.start);
    cudaEventDestroy(t.stop);
  }
  timings.clear();
}

void Context::EndQueryProfile() {
  last_kernels.clear();
  if (!profile || dry) return;
  KDB_CUDA(cudaStreamSynchronize(stream));
  for (auto& t : timings) {
    float ms = 0;
    KDB_CUDA(cudaEventElapsedTime(&ms, t.start, t.stop));
    last_kernels.emplace_back(t.tag, ms);
    cudaEventDestroy(t.start);
    cudaEventDestroy(t.stop);
  }
  timings.clear();
}

void Context::CheckDeviceError(const char* what) {
  if (dry) return;
  int err[4] = {0, 0, 0, 0};
  KDB_CUDA(cudaMemcpyAsync(err, d_err, sizeof(err), cudaMemcpyDeviceToHost, stream));
  KDB_CUDA(cudaStreamSynchronize(stream));
  if (err[0]) {
    KDB_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int) * 4, stream));
    if (err[0] == 1) throw Error(-4, std::string(what) + ": device table capacity exceeded");
    if (err[0] == 2) throw Error(-6, std::string(what) + ": bounded device wait gave up");
    throw Error(-5, std::string(what) + ": unsupported value on device");
  }
}

}  // namespace kdb
