// extern "C" layer of the per-operator entry points (operators.cu): selection
// vectors, hash build / probe, group-by aggregation, column indexes and the
// Skinner join operator on its own.  No exception crosses the boundary.
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "capi_internal.h"
#include "json.h"
#include "operators.h"

struct kdb_selvec {
  std::unique_ptr<kdb::ops::SelVec> s;
};
struct kdb_hash {
  std::unique_ptr<kdb::ops::HashTable> h;
};
struct kdb_pairs {
  std::unique_ptr<kdb::ops::Pairs> p;
};
struct kdb_agg {
  std::unique_ptr<kdb::ops::AggTable> a;
  bool pre_aggregate = true;
};
struct kdb_index {
  std::unique_ptr<kdb::ops::ColumnIndex> i;
};

namespace {

// Runs one operator call; with profiling on, its kernels' CUDA-event times
// become the context's last-query kernel list (as for a whole plan).
template <typename F>
int OpGuard(kdb_ctx* ctx, F&& f) {
  if (!ctx) return KDB_ERR_INVALID;
  try {
    kdb::Context& c = *kdb_ctx_context(ctx);
    c.BeginQueryProfile();
    f(c);
    // (a call that ran a whole plan has collected its own kernels already)
    if (!c.timings.empty()) c.EndQueryProfile();
    return KDB_OK;
  } catch (const kdb::Error& e) {
    kdb_ctx_set_error(ctx, e.what());
    return e.code;
  } catch (const std::exception& e) {
    kdb_ctx_set_error(ctx, e.what());
    return KDB_ERR_INVALID;
  }
}

std::vector<std::string> Names(const char* const* v, int32_t n) {
  std::vector<std::string> out;
  for (int32_t i = 0; i < n; i++) {
    if (!v || !v[i]) throw kdb::Error(KDB_ERR_INVALID, "null column name");
    out.emplace_back(v[i]);
  }
  return out;
}

std::vector<char> ReadAll(const char* path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw kdb::Error(KDB_ERR_INVALID, std::string("cannot open ") + path);
  return std::vector<char>((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
}

// .kdbindex (runtime/column_index.h:21-41, written by column_index.cc:150-240):
// {u64 mask; u64 array[mask + 1]} then, chained from the array, entries
// {K key (padded to 8 bytes); u64 size; u64 next; int32 values[size]} at
// byte offsets (0 ends a chain).  Every offset and size is checked against
// the file before it is read.
std::vector<std::pair<int64_t, std::vector<int32_t>>> ReadKdbIndex(const std::vector<char>& raw, int width) {
  auto u64 = [&](uint64_t off) {
    if (off > raw.size() || raw.size() - off < 8) throw kdb::Error(KDB_ERR_INVALID, "corrupt .kdbindex file");
    uint64_t v;
    std::memcpy(&v, raw.data() + off, 8);
    return v;
  };
  const uint64_t mask = u64(0);
  if (mask >= (raw.size() - 8) / 8 || ((mask + 1) & mask) != 0)
    throw kdb::Error(KDB_ERR_INVALID, "corrupt .kdbindex file (bucket array)");
  const uint64_t header = 8 + 8 * (mask + 1);
  std::vector<std::pair<int64_t, std::vector<int32_t>>> out;
  uint64_t budget = raw.size() / 24 + 1;  // entries are at least 24 bytes: bounds every chain walk
  for (uint64_t b = 0; b <= mask; b++) {
    for (uint64_t pos = u64(8 + 8 * b); pos != 0; pos = u64(pos + 16)) {
      if (pos < header || budget-- == 0) throw kdb::Error(KDB_ERR_INVALID, "corrupt .kdbindex file (chain)");
      const uint64_t size = u64(pos + 8);
      if (size > (raw.size() - std::min<uint64_t>(raw.size(), pos + 24)) / 4)
        throw kdb::Error(KDB_ERR_INVALID, "corrupt .kdbindex file (posting list)");
      int64_t key = 0;
      switch (width) {
        case 1: key = static_cast<int8_t>(raw[pos]); break;
        case 2: {
          int16_t v;
          std::memcpy(&v, raw.data() + pos, 2);
          key = v;
          break;
        }
        case 4: {
          int32_t v;
          std::memcpy(&v, raw.data() + pos, 4);
          key = v;
          break;
        }
        default: std::memcpy(&key, raw.data() + pos, 8); break;
      }
      std::vector<int32_t> rows(size);
      if (size) std::memcpy(rows.data(), raw.data() + pos + 24, 4 * size);
      out.emplace_back(key, std::move(rows));
    }
  }
  return out;
}

}  // namespace

extern "C" {

// ---- selection vectors ------------------------------------------------------
int kdb_scan_select(kdb_ctx* ctx, const char* table, const char* const* columns, int32_t ncols,
                    const char* filter_json, kdb_selvec** out) {
  if (out) *out = nullptr;
  return OpGuard(ctx, [&](kdb::Context& c) {
    if (!table || !filter_json || !out || ncols < 0) throw kdb::Error(KDB_ERR_INVALID, "null argument");
    auto cols = Names(columns, ncols);
    auto filter = kdb::plan::ParseExpr(kdb::json::Parse(filter_json));
    if (filter->type.id != kdb::plan::TypeId::BOOLEAN) throw kdb::Error(KDB_ERR_INVALID, "filter must be BOOLEAN");
    auto sv = kdb::ScanSelectRows(c, table, cols, *filter);
    *out = new kdb_selvec{std::move(sv)};
  });
}

int kdb_sort(kdb_ctx* ctx, const char* table, const char* const* key_columns, const int8_t* asc, int32_t nkeys,
             const kdb_selvec* sel, kdb_selvec** out) {
  if (out) *out = nullptr;
  return OpGuard(ctx, [&](kdb::Context& c) {
    if (!table || !key_columns || !asc || !out || nkeys <= 0) throw kdb::Error(KDB_ERR_INVALID, "null argument");
    std::vector<bool> dir;
    for (int32_t k = 0; k < nkeys; k++) dir.push_back(asc[k] != 0);
    auto sv = kdb::ops::SortRows(c, table, Names(key_columns, nkeys), dir, sel ? sel->s.get() : nullptr);
    *out = new kdb_selvec{std::move(sv)};
  });
}

int64_t kdb_selvec_size(const kdb_selvec* s) { return s ? s->s->n : -1; }

const int32_t* kdb_selvec_device_rows(const kdb_selvec* s) { return s ? s->s->rows : nullptr; }

int64_t kdb_selvec_get(const kdb_selvec* s, int32_t* rows, int64_t cap) {
  if (!s) return KDB_ERR_INVALID;
  const int64_t m = std::min<int64_t>(cap, s->s->n);
  if (rows && m > 0) {
    cudaSetDevice(s->s->ctx->device);
    if (cudaStreamSynchronize(s->s->ctx->stream) != cudaSuccess ||
        cudaMemcpy(rows, s->s->rows, sizeof(int32_t) * m, cudaMemcpyDeviceToHost) != cudaSuccess)
      return KDB_ERR_CUDA;
  }
  return s->s->n;
}

void kdb_selvec_free(kdb_selvec* s) { delete s; }

// ---- hash join ----------------------------------------------------------------
int kdb_hash_build(kdb_ctx* ctx, const char* table, const char* key_column, const kdb_selvec* sel,
                   double load_factor, int32_t fanout, kdb_hash** out) {
  if (out) *out = nullptr;
  return OpGuard(ctx, [&](kdb::Context& c) {
    if (!table || !key_column || !out || fanout < 0) throw kdb::Error(KDB_ERR_INVALID, "bad argument");
    auto h = kdb::ops::HashBuild(c, table, key_column, sel ? sel->s.get() : nullptr, load_factor, fanout);
    *out = new kdb_hash{std::move(h)};
  });
}

int kdb_hash_info(const kdb_hash* h, int32_t* fanout, int64_t* slots, int64_t* bytes) {
  if (!h) return KDB_ERR_INVALID;
  if (fanout) *fanout = 1 << h->h->bits;
  if (slots) *slots = h->h->total_slots;
  if (bytes) *bytes = static_cast<int64_t>(h->h->bytes);
  return KDB_OK;
}

int kdb_hash_probe(kdb_ctx* ctx, const kdb_hash* h, const char* table, const char* key_column,
                   const kdb_selvec* sel, int32_t ordered, kdb_pairs** out) {
  if (out) *out = nullptr;
  return OpGuard(ctx, [&](kdb::Context& c) {
    if (!h || !table || !key_column || !out) throw kdb::Error(KDB_ERR_INVALID, "null argument");
    if (h->h->ctx != &c) throw kdb::Error(KDB_ERR_INVALID, "hash table belongs to another context");
    auto p = kdb::ops::HashProbe(c, *h->h, table, key_column, sel ? sel->s.get() : nullptr, ordered != 0);
    *out = new kdb_pairs{std::move(p)};
  });
}

void kdb_hash_free(kdb_hash* h) { delete h; }

int64_t kdb_pairs_size(const kdb_pairs* p) { return p ? p->p->n : -1; }

int64_t kdb_pairs_get(const kdb_pairs* p, int32_t* probe_rows, int32_t* build_rows, int64_t cap) {
  if (!p) return KDB_ERR_INVALID;
  const int64_t m = std::min<int64_t>(cap, p->p->n);
  if (m > 0) {
    cudaSetDevice(p->p->ctx->device);
    if (probe_rows && cudaMemcpy(probe_rows, p->p->probe, 4 * m, cudaMemcpyDeviceToHost) != cudaSuccess)
      return KDB_ERR_CUDA;
    if (build_rows && cudaMemcpy(build_rows, p->p->build, 4 * m, cudaMemcpyDeviceToHost) != cudaSuccess)
      return KDB_ERR_CUDA;
  }
  return p->p->n;
}

void kdb_pairs_free(kdb_pairs* p) { delete p; }

// ---- group-by aggregation --------------------------------------------------------
int kdb_agg_create(kdb_ctx* ctx, const char* table, const char* const* key_columns, int32_t nkeys,
                   const kdb_agg_spec* aggs, int32_t naggs, int64_t max_groups, kdb_agg** out) {
  if (out) *out = nullptr;
  return OpGuard(ctx, [&](kdb::Context& c) {
    if (!table || !out || !aggs || naggs < 0 || nkeys < 0) throw kdb::Error(KDB_ERR_INVALID, "bad argument");
    std::vector<kdb::ops::AggSpec> specs;
    for (int32_t k = 0; k < naggs; k++) specs.push_back({aggs[k].agg, aggs[k].column ? aggs[k].column : ""});
    auto a = kdb::ops::AggCreate(c, table, Names(key_columns, nkeys), specs, max_groups);
    *out = new kdb_agg{std::move(a)};
  });
}

int kdb_agg_set_pre_aggregation(kdb_agg* a, int32_t on) {
  if (!a) return KDB_ERR_INVALID;
  a->pre_aggregate = on != 0;
  return KDB_OK;
}

int kdb_agg_update(kdb_ctx* ctx, kdb_agg* a, const kdb_selvec* sel) {
  return OpGuard(ctx, [&](kdb::Context& c) {
    if (!a) throw kdb::Error(KDB_ERR_INVALID, "null argument");
    kdb::ops::AggUpdateRows(c, *a->a, sel ? sel->s.get() : nullptr, a->pre_aggregate);
  });
}

int kdb_agg_finalize(kdb_ctx* ctx, kdb_agg* a, kdb_result** out) {
  if (out) *out = nullptr;
  return OpGuard(ctx, [&](kdb::Context& c) {
    if (!a || !out) throw kdb::Error(KDB_ERR_INVALID, "null argument");
    auto r = std::make_unique<kdb_result>();
    r->r = kdb::ops::AggFinalize(c, *a->a);
    *out = r.release();
  });
}

void kdb_agg_free(kdb_agg* a) { delete a; }

// ---- column indexes ------------------------------------------------------------------
int kdb_index_build(kdb_ctx* ctx, const char* table, const char* column, kdb_index** out) {
  if (out) *out = nullptr;
  return OpGuard(ctx, [&](kdb::Context& c) {
    if (!table || !column || !out) throw kdb::Error(KDB_ERR_INVALID, "null argument");
    *out = new kdb_index{kdb::ops::IndexBuild(c, table, column)};
  });
}

int kdb_index_open_kdbindex(kdb_ctx* ctx, const char* path, const char* type, kdb_index** out) {
  if (out) *out = nullptr;
  return OpGuard(ctx, [&](kdb::Context& c) {
    if (!path || !type || !out) throw kdb::Error(KDB_ERR_INVALID, "null argument");
    const kdb::plan::Type t = kdb::plan::ParseType(type);
    int w = 0;
    switch (t.id) {
      case kdb::plan::TypeId::BOOLEAN: w = 1; break;
      case kdb::plan::TypeId::SMALLINT: w = 2; break;
      case kdb::plan::TypeId::INT:
      case kdb::plan::TypeId::DATE:
      case kdb::plan::TypeId::ENUM: w = 4; break;
      case kdb::plan::TypeId::BIGINT: w = 8; break;
      default: throw kdb::Error(KDB_ERR_UNSUPPORTED, "indexes over integer, date, enum or boolean keys");
    }
    *out = new kdb_index{kdb::ops::IndexFromPostings(c, t, ReadKdbIndex(ReadAll(path), w))};
  });
}

int64_t kdb_index_num_keys(const kdb_index* i) { return i ? i->i->nkeys : -1; }
int64_t kdb_index_num_rows(const kdb_index* i) { return i ? i->i->n : -1; }

int64_t kdb_index_get(const kdb_index* i, int64_t key, int32_t* rows, int64_t cap) {
  if (!i) return KDB_ERR_INVALID;
  try {
    if (!i->i->ctx->dry) cudaSetDevice(i->i->ctx->device);
    return i->i->Get(key, rows, cap);
  } catch (const std::exception&) {
    return KDB_ERR_CUDA;
  }
}

int64_t kdb_index_keys(const kdb_index* i, int64_t* keys, int64_t cap) {
  if (!i) return KDB_ERR_INVALID;
  const int64_t m = std::min<int64_t>(cap, i->i->nkeys);
  if (keys && m > 0) std::memcpy(keys, i->i->hkeys.data(), 8 * m);
  return i->i->nkeys;
}

void kdb_index_free(kdb_index* i) { delete i; }

// ---- Skinner join on its own -------------------------------------------------------
int kdb_skinner_execute(kdb_ctx* ctx, const char* skinner_json, int32_t policy, int64_t budget_per_episode,
                        uint32_t seed, kdb_result** out) {
  if (out) *out = nullptr;
  return OpGuard(ctx, [&](kdb::Context& c) {
    if (!skinner_json || !out) throw kdb::Error(KDB_ERR_INVALID, "null argument");
    if (policy < 0 || policy > 2 || budget_per_episode <= 0) throw kdb::Error(KDB_ERR_INVALID, "bad policy or budget");
    auto op = kdb::plan::ParseOperator(kdb::json::Parse(skinner_json));
    if (op->kind != kdb::plan::OpKind::SKINNER_JOIN) throw kdb::Error(KDB_ERR_INVALID, "not a SKINNER_JOIN operator");
    for (const auto& ch : op->children)
      if (ch->kind != kdb::plan::OpKind::SCAN && ch->kind != kdb::plan::OpKind::SCAN_SELECT)
        throw kdb::Error(KDB_ERR_UNSUPPORTED, "the operator's children must be scans (run other trees as plans)");
    // the options apply to this call only
    const int64_t old_budget = c.skinner_budget;
    const uint32_t old_seed = c.skinner_seed;
    const int old_policy = c.skinner_policy;
    c.skinner_budget = budget_per_episode;
    c.skinner_seed = seed;
    c.skinner_policy = policy;
    auto restore = [&] {
      c.skinner_budget = old_budget;
      c.skinner_seed = old_seed;
      c.skinner_policy = old_policy;
    };
    auto r = std::make_unique<kdb_result>();
    try {
      r->r = kdb::ExecutePlan(c, *op, nullptr);
    } catch (...) {
      restore();
      throw;
    }
    restore();
    *out = r.release();
  });
}

}  // extern "C"
