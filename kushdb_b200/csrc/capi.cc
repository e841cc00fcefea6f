// extern "C" boundary (include/kdb_b200.h): no exceptions cross it.
#include <cstring>
#include <fstream>
#include <sstream>
#include <unordered_map>

#include "capi_internal.h"

struct kdb_ctx {
  // parsed plans by their JSON text, each with its prepared (recorded)
  // execution once it has run
  struct Entry {
    std::unique_ptr<kdb::plan::Operator> plan;
    std::unique_ptr<kdb::PreparedQuery> prepared;
  };
  std::unique_ptr<kdb::Context> c;
  std::string err;
  std::unordered_map<std::string, Entry> plans;
  bool prepare = true;
};

namespace {
constexpr size_t kMaxPreparedTotal = size_t(4) << 30;  // device memory held by all prepared queries
}

namespace {

template <typename F>
int Guard(kdb_ctx* ctx, F&& f) {
  if (!ctx) return KDB_ERR_INVALID;
  try {
    f();
    return KDB_OK;
  } catch (const kdb::Error& e) {
    ctx->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    ctx->err = e.what();
    return KDB_ERR_INVALID;
  }
}

std::vector<char> ReadFile(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw kdb::Error(KDB_ERR_INVALID, "cannot open " + path);
  return std::vector<char>((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
}

}  // namespace

namespace {
void RunPlan(kdb_ctx* ctx, const char* plan_json, kdb_result** out);
}  // namespace

kdb::Context* kdb_ctx_context(kdb_ctx* ctx) { return ctx->c.get(); }
void kdb_ctx_set_error(kdb_ctx* ctx, const std::string& msg) {
  if (ctx) ctx->err = msg;
}

extern "C" {

int kdb_ctx_create(int device, kdb_ctx** out) {
  if (!out) return KDB_ERR_INVALID;
  *out = nullptr;
  auto* ctx = new kdb_ctx();
  try {
    ctx->c = std::make_unique<kdb::Context>(device);
  } catch (const std::exception& e) {
    static thread_local std::string last;
    last = e.what();
    delete ctx;
    return KDB_ERR_CUDA;
  }
  *out = ctx;
  return KDB_OK;
}

int kdb_ctx_destroy(kdb_ctx* ctx) {
  delete ctx;
  return KDB_OK;
}

const char* kdb_last_error(kdb_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int64_t kdb_ctx_kernel_launches(kdb_ctx* ctx) { return ctx ? ctx->c->kernel_launches : -1; }

int64_t kdb_ctx_column_bytes(kdb_ctx* ctx) { return ctx ? ctx->c->ColumnBytes() : -1; }

void* kdb_ctx_stream(kdb_ctx* ctx) { return ctx ? static_cast<void*>(ctx->c->stream) : nullptr; }

int kdb_ctx_set_profiling(kdb_ctx* ctx, int enabled) {
  return Guard(ctx, [&] { ctx->c->profile = enabled != 0; });
}

int64_t kdb_last_query_kernels(kdb_ctx* ctx, char* buf, int64_t cap) {
  if (!ctx) return KDB_ERR_INVALID;
  std::ostringstream o;
  o << "[";
  bool firstk = true;
  for (const auto& [tag, ms] : ctx->c->last_kernels) {
    o << (firstk ? "" : ",") << "{\"tag\":\"" << tag << "\",\"ms\":" << ms << "}";
    firstk = false;
  }
  o << "]";
  std::string s = o.str();
  if (buf && cap > 0) {
    int64_t n = std::min<int64_t>(cap - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return static_cast<int64_t>(s.size()) + 1;
}

int kdb_table_add_column(kdb_ctx* ctx, const char* table, const char* column, const char* type,
                         const void* host_data, int64_t n, const int8_t* host_nulls) {
  return Guard(ctx, [&] {
    if (!table || !column || !type || (n > 0 && !host_data))
      throw kdb::Error(KDB_ERR_INVALID, "null argument");
    ctx->c->AddColumn(table, column, kdb::plan::ParseType(type), host_data, n, host_nulls);
  });
}

int kdb_table_add_text_column(kdb_ctx* ctx, const char* table, const char* column,
                              const int64_t* offsets, const char* chars, int64_t n,
                              const int8_t* host_nulls) {
  return Guard(ctx, [&] {
    if (!table || !column || !offsets) throw kdb::Error(KDB_ERR_INVALID, "null argument");
    ctx->c->AddTextColumn(table, column, offsets, chars, n, host_nulls);
  });
}

// runtime/column_data.cc:121-229 file layout.
int kdb_column_open_kdb(kdb_ctx* ctx, const char* table, const char* column, const char* type,
                        const char* path, const char* null_path) {
  return Guard(ctx, [&] {
    kdb::plan::Type t = kdb::plan::ParseType(type);
    std::vector<char> raw = ReadFile(path);
    std::vector<char> nulls;
    if (null_path && *null_path) nulls = ReadFile(null_path);
    const int8_t* np = nulls.empty() ? nullptr : reinterpret_cast<const int8_t*>(nulls.data());
    if (t.id == kdb::plan::TypeId::TEXT) {
      ctx->c->AddTextColumnFromKdb(table, column, raw.data(), raw.size(), np,
                                   static_cast<int64_t>(nulls.size()));
    } else {
      int w = kdb::plan::TypeWidth(t.id);
      if (raw.size() % w) throw kdb::Error(KDB_ERR_INVALID, "file length is not a multiple of the type's width");
      int64_t n = static_cast<int64_t>(raw.size()) / w;
      if (np && static_cast<int64_t>(nulls.size()) != n)
        throw kdb::Error(KDB_ERR_INVALID, "null file length differs from column length");
      ctx->c->AddColumn(table, column, t, raw.data(), n, np);
    }
  });
}

int kdb_table_drop(kdb_ctx* ctx, const char* table) {
  return Guard(ctx, [&] { ctx->c->DropTable(table); });
}

int64_t kdb_table_num_rows(kdb_ctx* ctx, const char* table) {
  if (!ctx) return -1;
  auto it = ctx->c->tables.find(table);
  return it == ctx->c->tables.end() ? -1 : it->second.rows;
}

int kdb_enum_register(kdb_ctx* ctx, int32_t enum_id, const int64_t* offsets, const char* chars,
                      int32_t n) {
  return Guard(ctx, [&] {
    std::vector<std::string> v;
    for (int32_t k = 0; k < n; k++) v.emplace_back(chars + offsets[k], offsets[k + 1] - offsets[k]);
    ctx->c->RegisterEnum(enum_id, std::move(v));
  });
}

// runtime/enum.cc:19-131: EnumData{u64 entry_offset; u64 mask; u64 array[]}
// then EnumEntry{u64 str_offset; u32 str_len; u32 value} indexed by key.
int kdb_enum_open_kdbenum(kdb_ctx* ctx, int32_t enum_id, const char* path) {
  return Guard(ctx, [&] {
    std::vector<char> raw = ReadFile(path);
    const uint64_t size = raw.size();
    if (size < 16) throw kdb::Error(KDB_ERR_INVALID, "short .kdbenum file");
    uint64_t entry_offset;
    std::memcpy(&entry_offset, raw.data(), 8);
    if (entry_offset < 16 || entry_offset > size) throw kdb::Error(KDB_ERR_INVALID, "corrupt .kdbenum file (header)");
    // entries are dense in key order; the first string follows the last entry
    uint64_t n = 0;
    if (entry_offset + 16 <= size) {
      uint64_t first_str;
      std::memcpy(&first_str, raw.data() + entry_offset, 8);
      if (first_str < entry_offset + 16 || first_str > size || (first_str - entry_offset) % 16)
        throw kdb::Error(KDB_ERR_INVALID, "corrupt .kdbenum file (entries)");
      n = (first_str - entry_offset) / 16;
    }
    if (n > static_cast<uint64_t>(INT32_MAX)) throw kdb::Error(KDB_ERR_INVALID, "corrupt .kdbenum file (size)");
    std::vector<std::string> values(n);
    for (uint64_t k = 0; k < n; k++) {
      const uint64_t pos = entry_offset + 16 * k;
      uint64_t so;
      uint32_t sl, v;
      std::memcpy(&so, raw.data() + pos, 8);
      std::memcpy(&sl, raw.data() + pos + 8, 4);
      std::memcpy(&v, raw.data() + pos + 12, 4);
      if (v != k || so > size || sl > size - so)
        throw kdb::Error(KDB_ERR_INVALID, "corrupt .kdbenum file (entry " + std::to_string(k) + ")");
      values[k] = std::string(raw.data() + so, sl);
    }
    ctx->c->RegisterEnum(enum_id, std::move(values));
  });
}

int kdb_query_execute(kdb_ctx* ctx, const char* plan_json, kdb_result** out) {
  if (out) *out = nullptr;
  return Guard(ctx, [&] { RunPlan(ctx, plan_json, out); });
}

int kdb_query_execute_host(kdb_ctx* ctx, const char* plan_json, const kdb_host_column* cols, int32_t ncols,
                           kdb_result** out) {
  if (out) *out = nullptr;
  return Guard(ctx, [&] {
    if (ncols < 0 || (ncols > 0 && !cols)) throw kdb::Error(KDB_ERR_INVALID, "bad column list");
    std::vector<kdb::Context::HostColumnSpec> specs;
    for (int32_t i = 0; i < ncols; i++) {
      const kdb_host_column& c = cols[i];
      if (!c.table || !c.column || !c.type) throw kdb::Error(KDB_ERR_INVALID, "null column field");
      specs.push_back({c.table, c.column, kdb::plan::ParseType(c.type), c.data, c.n, c.nulls});
    }
    ctx->c->StreamColumns(specs);
    RunPlan(ctx, plan_json, out);
  });
}

int kdb_ctx_set_ingest(kdb_ctx* ctx, int64_t chunk_bytes, int32_t streams) {
  return Guard(ctx, [&] {
    if (chunk_bytes < (1 << 16) || streams < 1 || streams > 8)
      throw kdb::Error(KDB_ERR_INVALID, "chunk of at least 64 KiB, 1 to 8 streams");
    ctx->c->ingest_chunk_bytes = chunk_bytes;
    ctx->c->ingest_streams = streams;
  });
}

}  // extern "C"

namespace {

void RunPlan(kdb_ctx* ctx, const char* plan_json, kdb_result** out) {
  {
    if (!plan_json || !out) throw kdb::Error(KDB_ERR_INVALID, "null argument");
    // parsed plans are cached by their text (a prepared statement's tree)
    auto& cache = ctx->plans;
    auto it = cache.find(plan_json);
    if (it == cache.end()) {
      if (cache.size() >= 256) cache.clear();
      kdb_ctx::Entry e;
      e.plan = kdb::plan::ParsePlan(plan_json);
      it = cache.emplace(plan_json, std::move(e)).first;
    }
    auto res = std::make_unique<kdb_result>();
    kdb_ctx::Entry& entry = it->second;
    res->r = kdb::ExecutePlan(*ctx->c, *entry.plan, ctx->prepare ? &entry.prepared : nullptr);
    if (entry.prepared) {
      // keep the device memory held by prepared queries bounded
      size_t total = 0;
      for (auto& [k, e] : cache)
        if (e.prepared) total += e.prepared->arena->bytes();
      if (total > kMaxPreparedTotal)
        for (auto& [k, e] : cache)
          if (&e != &entry) e.prepared.reset();
    }
    *out = res.release();
  }
}

}  // namespace

extern "C" {

int kdb_ctx_set_option(kdb_ctx* ctx, const char* name, const char* value) {
  return Guard(ctx, [&] {
    if (!name || std::strncmp(name, "KDB_", 4) != 0) throw kdb::Error(KDB_ERR_INVALID, "option names start with KDB_");
    if (value) ctx->c->options[name] = value;
    else ctx->c->options.erase(name);
    ctx->c->catalog_version++;  // recordings were generated under the old options
  });
}

int64_t kdb_ctx_get_option(kdb_ctx* ctx, const char* name, char* buf, int64_t cap) {
  if (!ctx || !name) return KDB_ERR_INVALID;
  const char* v = ctx->c->OptStr(name);
  if (!v) return 0;
  const int64_t n = static_cast<int64_t>(std::strlen(v));
  if (buf && cap > 0) {
    const int64_t m = std::min<int64_t>(cap - 1, n);
    std::memcpy(buf, v, m);
    buf[m] = 0;
  }
  return n + 1;
}

int kdb_ctx_set_prepared_queries(kdb_ctx* ctx, int32_t on) {
  return Guard(ctx, [&] {
    ctx->prepare = on != 0;
    if (!ctx->prepare)
      for (auto& [k, e] : ctx->plans) e.prepared.reset();
  });
}

int kdb_ctx_set_skinner(kdb_ctx* ctx, int64_t budget_per_episode, uint32_t seed) {
  return Guard(ctx, [&] {
    if (budget_per_episode < 1) throw kdb::Error(KDB_ERR_INVALID, "budget must be positive");
    ctx->c->skinner_budget = budget_per_episode;
    ctx->c->skinner_seed = seed;
  });
}

int64_t kdb_last_skinner_episodes(kdb_ctx* ctx) { return ctx ? ctx->c->last_skinner_episodes : -1; }

int64_t kdb_last_skinner_work(kdb_ctx* ctx) { return ctx ? ctx->c->last_skinner_work : -1; }

int64_t kdb_last_skinner_batches(kdb_ctx* ctx) { return ctx ? ctx->c->last_skinner_batches : -1; }

int64_t kdb_last_skinner_samples(kdb_ctx* ctx, float* features, float* rewards, int64_t cap) {
  if (!ctx) return KDB_ERR_INVALID;
  const auto& f = ctx->c->skinner_features;
  const auto& r = ctx->c->skinner_rewards;
  const int64_t n = static_cast<int64_t>(r.size());
  const int64_t k = std::min<int64_t>(n, std::max<int64_t>(cap, 0));
  const size_t width = r.empty() ? 0 : f.size() / r.size();
  if (features && k) std::memcpy(features, f.data(), sizeof(float) * width * k);
  if (rewards && k) std::memcpy(rewards, r.data(), sizeof(float) * k);
  return n;
}

int kdb_sort_pairs(kdb_ctx* ctx, uint64_t* d_keys, uint32_t* d_vals, int64_t n, int32_t key_bits) {
  return Guard(ctx, [&] {
    if (n < 0 || (n > 0 && (!d_keys || !d_vals))) throw kdb::Error(KDB_ERR_INVALID, "bad sort arguments");
    if (key_bits < 1 || key_bits > 64) throw kdb::Error(KDB_ERR_INVALID, "key_bits must be in [1, 64]");
    ctx->c->BeginQueryProfile();
    {
      kdb::Arena arena(*ctx->c);
      ctx->c->RadixSortPairs(d_keys, d_vals, n, arena, key_bits);
    }
    if (!ctx->c->dry) KDB_CUDA(cudaStreamSynchronize(ctx->c->stream));
    ctx->c->EndQueryProfile();
  });
}

double kdb_last_query_device_ms(kdb_ctx* ctx) { return ctx ? ctx->c->last_device_ms : -1; }

int64_t kdb_result_num_rows(const kdb_result* r) { return r ? r->r.rows : -1; }
int32_t kdb_result_num_cols(const kdb_result* r) { return r ? static_cast<int32_t>(r->r.cols.size()) : -1; }

int kdb_result_col_type(const kdb_result* r, int32_t col, char* buf, int32_t cap) {
  if (!r || col < 0 || col >= static_cast<int32_t>(r->r.cols.size()) || !buf) return KDB_ERR_INVALID;
  const auto& t = r->r.cols[col].type;
  std::string s = t.id == kdb::plan::TypeId::ENUM ? "ENUM:" + std::to_string(t.enum_id)
                                                  : kdb::plan::TypeName(t.id);
  std::snprintf(buf, cap, "%s", s.c_str());
  return KDB_OK;
}

int kdb_result_get_i64(const kdb_result* r, int32_t col, int64_t* out) {
  if (!r || col < 0 || col >= static_cast<int32_t>(r->r.cols.size())) return KDB_ERR_INVALID;
  return r->r.cols[col].CopyInts(r->r.rows, out) ? KDB_OK : KDB_ERR_INVALID;
}

int kdb_result_get_f64(const kdb_result* r, int32_t col, double* out) {
  if (!r || col < 0 || col >= static_cast<int32_t>(r->r.cols.size())) return KDB_ERR_INVALID;
  return r->r.cols[col].CopyReals(r->r.rows, out) ? KDB_OK : KDB_ERR_INVALID;
}

int kdb_result_get_nulls(const kdb_result* r, int32_t col, int8_t* out) {
  if (!r || col < 0 || col >= static_cast<int32_t>(r->r.cols.size())) return KDB_ERR_INVALID;
  r->r.cols[col].CopyNulls(r->r.rows, out);
  return KDB_OK;
}

int64_t kdb_result_get_text(const kdb_result* r, int32_t col, int64_t row, char* buf, int64_t cap) {
  if (!r || col < 0 || col >= static_cast<int32_t>(r->r.cols.size())) return KDB_ERR_INVALID;
  const auto& c = r->r.cols[col];
  if (row < 0 || row >= static_cast<int64_t>(c.s.size())) return KDB_ERR_INVALID;
  const std::string& s = c.s[row];
  if (buf && cap > 0) std::memcpy(buf, s.data(), std::min<int64_t>(cap, s.size()));
  return static_cast<int64_t>(s.size());
}

int64_t kdb_result_format(kdb_ctx* ctx, const kdb_result* r, char* buf, int64_t cap) {
  if (!ctx || !r) return KDB_ERR_INVALID;
  std::string s = kdb::FormatResult(r->r, ctx->c->HostEnums());
  if (buf && cap > 0) {
    int64_t n = std::min<int64_t>(cap - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return static_cast<int64_t>(s.size()) + 1;
}

void kdb_result_free(kdb_result* r) { delete r; }

}  // extern "C"
