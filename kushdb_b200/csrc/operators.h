// Host-side objects of the per-operator entry points (operators.cu): device
// selection vectors, hash tables, probe results, aggregate tables and column
// indexes.  Each belongs to one Context and must be freed before it.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "engine.h"

namespace kdb {
namespace ops {

// Ascending row ids of one table's rows that passed a scan-select.
struct SelVec {
  Context* ctx = nullptr;
  std::string table;
  int32_t* rows = nullptr;  // device, n entries
  int64_t n = 0;
  ~SelVec();
};

// A device join table over one integer key column (runtime::HashTable).
// bits == 0: one open-addressing table; bits > 0: 2^bits sub-tables chosen by
// the key hash's top bits (radix partitioned).
struct HashTable {
  Context* ctx = nullptr;
  std::string table;
  plan::TypeId key_type = plan::TypeId::INT;
  bool wide = false;  // 64-bit keys: 16-byte slots
  int bits = 0;
  void* slots = nullptr;
  unsigned long long* slot_off = nullptr;  // device, 2^bits + 1 sub-table offsets (slots)
  int64_t total_slots = 0;
  size_t bytes = 0;
  ~HashTable();
};

// (probe row, build row) pairs of a probe, as two device arrays.
struct Pairs {
  Context* ctx = nullptr;
  int32_t* probe = nullptr;
  int32_t* build = nullptr;
  int64_t n = 0;
  ~Pairs();
};

std::unique_ptr<HashTable> HashBuild(Context& c, const std::string& table, const std::string& key_column,
                                     const SelVec* sel, double load_factor, int32_t fanout);
std::unique_ptr<Pairs> HashProbe(Context& c, const HashTable& ht, const std::string& table,
                                 const std::string& key_column, const SelVec* sel, bool ordered);
// Sub-table bits the automatic fan-out chooses for n rows (host rule).
int PartBitsFor(int64_t n, double load_factor, int slot_bytes, int32_t fanout);

// Rows of `table` (all, or those of `sel`) in ORDER BY order of the key
// columns (asc[k] per key; a NULL sorts after every value ascending and
// before descending, as proxy::LessThan used both ways; ties keep the
// input order, as runtime::Vector's merge sort does).  Keys: integer, date,
// boolean, enum (string order) and real columns.
std::unique_ptr<SelVec> SortRows(Context& c, const std::string& table, const std::vector<std::string>& keys,
                                 const std::vector<bool>& asc, const SelVec* sel);

// One aggregate of a group-by: op is a plan::AggType (SUM, MIN, MAX, AVG,
// COUNT); an empty column under COUNT counts rows.
struct AggSpec {
  int op = 0;
  std::string column;
};

// A device group-by table over one table's integer key columns
// (runtime::AggregateHashTable); see operators.cu for the layout.
struct AggTable {
  Context* ctx = nullptr;
  std::string table;
  std::vector<std::string> keys;
  std::vector<AggSpec> aggs;
  std::vector<plan::Type> key_types, agg_types;
  int64_t G = 0;        // group capacity
  uint64_t cap = 0;     // slots
  int64_t updates = 0;  // update calls so far
  unsigned long long* slots = nullptr;
  int64_t* keyv = nullptr;
  int8_t* knull = nullptr;
  unsigned long long* val = nullptr;
  unsigned long long* cnt = nullptr;
  unsigned long long* first = nullptr;
  unsigned long long* ngroups = nullptr;
  int* err = nullptr;
  std::vector<void*> bufs;
  ~AggTable();
};

std::unique_ptr<AggTable> AggCreate(Context& c, const std::string& table, const std::vector<std::string>& keys,
                                    const std::vector<AggSpec>& aggs, int64_t max_groups);
void AggUpdateRows(Context& c, AggTable& t, const SelVec* sel, bool pre_aggregate);
HostResult AggFinalize(Context& c, AggTable& t);

// Posting lists of one column: key -> ascending row ids (MemoryColumnIndex /
// ColumnIndex).  NULL keys are not indexed.
struct ColumnIndex {
  Context* ctx = nullptr;
  plan::Type type;
  int64_t n = 0;      // rows indexed
  int64_t nkeys = 0;  // distinct keys
  int32_t* rows = nullptr;   // device, n
  int64_t* dkeys = nullptr;  // device, nkeys ascending
  int64_t* starts = nullptr;  // device, nkeys + 1
  std::vector<int64_t> hkeys, hstarts;  // host mirrors
  std::vector<int32_t> hrows;           // the rows, in a compile-only context
  // rows of `key` (at most cap copied to out); returns how many there are
  int64_t Get(int64_t key, int32_t* out, int64_t cap) const;
  ~ColumnIndex();
};
std::unique_ptr<ColumnIndex> IndexBuild(Context& c, const std::string& table, const std::string& column);
std::unique_ptr<ColumnIndex> IndexFromPostings(Context& c, plan::Type type,
                                               std::vector<std::pair<int64_t, std::vector<int32_t>>> postings);

// Copies each 1024-row tile's compacted row ids (scratch[t * 1024 ..], count
// from the exclusive offsets off[t] .. off[t + 1]) to out[off[t] ..].
void GatherTiles(Context& c, const int32_t* scratch, const uint64_t* off, int64_t ntiles, int32_t* out);

}  // namespace ops

// Compiles `filter` (a boolean expression over `columns` of `table`, bound
// by position) into a scan-select kernel; returns the qualifying rows.
std::unique_ptr<ops::SelVec> ScanSelectRows(Context& ctx, const std::string& table,
                                            const std::vector<std::string>& columns, const plan::Expr& filter);

}  // namespace kdb
