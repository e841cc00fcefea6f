// Compiled CPU baseline loops -- TEST / BENCHMARK INFRASTRUCTURE ONLY.
//
// Hand-restated versions of the scalar loops the reference's translators
// generate for the three benchmark plans, with the runtime structures those
// loops call restated alongside:
//   * runtime::AggregateHashTable + proxy UpdateOrInsert / Hash / Salt
//     (runtime/aggregate_hash_table.cc:9-135,
//      compile/proxy/aggregate_hash_table.cc:187-337): 64-bit entries
//      {salt16, block_offset16, block_idx32}, payloads in 4 KiB blocks,
//      linear probing, doubling when size > capacity / 1.5;
//   * runtime::HashTable (runtime/hash_table.cc:13-67): unordered_map from a
//     HashCombine'd int32 hash to a vector of packed build tuples;
//   * runtime::Vector::Sort (runtime/vector.cc:45-110) for ORDER BY.
// Aggregators follow compile/proxy/aggregator.cc (SUM sequential, AVG as a
// cumulative moving average, COUNT int64).  The plain entry points run one
// thread, like the reference's executor (execution/executable_query.cc:
// 229-244); the `_mt` variants split the rows over `threads` host threads,
// each running the same loop into its own table, and merge the partial
// tables (for a CPU arm that uses every host core).  Used as the timed CPU
// arm of the benchmark, never by the product.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

constexpr int kBlockSize = 1 << 12;
constexpr double kLoadFactor = 1.5;

// runtime::AggregateHashTable (restated)
struct AggTable {
  uint32_t size = 0, capacity = 1024;
  uint64_t mask = 1023;
  std::vector<uint64_t> entries = std::vector<uint64_t>(1024, 0);
  std::vector<uint8_t*> blocks{nullptr, new uint8_t[kBlockSize]};
  uint16_t last_offset = 0;
  uint16_t payload_size;
  explicit AggTable(uint16_t ps) : payload_size(ps) {}
  ~AggTable() {
    for (auto* b : blocks) delete[] b;
  }
  static uint64_t Entry(uint16_t salt, uint16_t off, uint32_t idx) {
    return (uint64_t(salt) << 48) | (uint64_t(off) << 32) | idx;
  }
  void Resize() {
    uint32_t cap = capacity * 2;
    uint64_t m = cap - 1;
    std::vector<uint64_t> e(cap, 0);
    for (uint32_t b = 1; b < blocks.size(); b++) {
      uint32_t end = b == blocks.size() - 1 ? last_offset : kBlockSize;
      for (uint32_t off = 0; off + payload_size <= end; off += payload_size) {
        uint64_t h;
        std::memcpy(&h, blocks[b] + off, 8);
        uint64_t i = h & m;
        while ((e[i] & 0xFFFFFFFFu) > 0) i = (i + 1) & m;
        e[i] = Entry(uint16_t(h >> 48), uint16_t(off), b);
      }
    }
    entries.swap(e);
    capacity = cap;
    mask = m;
  }
  uint8_t* Insert(uint64_t& entry, uint64_t hash, uint16_t salt) {
    size++;
    if (last_offset + payload_size > kBlockSize) {
      blocks.push_back(new uint8_t[kBlockSize]);
      last_offset = 0;
    }
    uint32_t b = uint32_t(blocks.size() - 1);
    uint16_t off = last_offset;
    last_offset = uint16_t(last_offset + payload_size);
    entry = Entry(salt, off, b);
    return blocks[b] + off;
  }
  template <typename F>
  void ForEach(F f) {
    for (uint32_t b = 1; b < blocks.size(); b++) {
      uint32_t end = b == blocks.size() - 1 ? last_offset : kBlockSize;
      for (uint32_t off = 0; off + payload_size <= end; off += payload_size) f(blocks[b] + off);
    }
  }
};

// proxy AggregateHashTable::Hash (compile/proxy/aggregate_hash_table.cc:313-333)
inline uint64_t MixKey(uint64_t hash, int64_t k) {
  const uint64_t magic = 0xc6a4a7935bd1e995ULL;
  uint64_t kh = uint64_t(k) * magic;
  kh ^= uint64_t(int64_t(kh) >> 47);
  kh *= magic;
  hash ^= kh;
  hash *= magic;
  hash += 0xe6546b64ULL;
  return hash;
}

struct Q1Payload {  // {hash, key0, key1, 4 sums, 3 x (cma, count), count}
  uint64_t hash;
  int32_t rf, ls;
  double sum_qty, sum_price, sum_disc_price, sum_charge;
  double avg_qty, cnt_qty, avg_price, cnt_price, avg_disc, cnt_disc;
  int64_t count;
};

// merge sort of runtime/vector.cc:45-110 over row indices
template <typename C>
void MergeSort(std::vector<int32_t>& v, C comp, int l, int r, std::vector<int32_t>& tmp) {
  if (l >= r) return;
  int m = l + (r - l) / 2;
  MergeSort(v, comp, l, m, tmp);
  MergeSort(v, comp, m + 1, r, tmp);
  int i = l, j = m + 1, k = 0;
  tmp.resize(r - l + 1);
  while (i <= m && j <= r) tmp[k++] = comp(v[i], v[j]) ? v[i++] : v[j++];
  while (i <= m) tmp[k++] = v[i++];
  while (j <= r) tmp[k++] = v[j++];
  std::memcpy(&v[l], tmp.data(), sizeof(int32_t) * (r - l + 1));
}

double Now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}


struct Q1Part {  // one thread's share of the Q1 group-by
  AggTable ht{sizeof(Q1Payload)};
};

void Q1Range(const int32_t* date, const int32_t* rf, const int32_t* ls, const double* qty, const double* price,
             const double* disc, const double* tax, int64_t b, int64_t e, int32_t date_leq, AggTable& ht) {
  for (int64_t i = b; i < e; i++) {
    if (!(date[i] <= date_leq)) continue;
    int32_t k0 = rf[i], k1 = ls[i];
    double q = qty[i], p = price[i], d = disc[i], tx = tax[i];
    if (ht.size == ht.capacity || double(ht.size) > double(ht.capacity) / kLoadFactor) ht.Resize();
    uint64_t h = MixKey(MixKey(0, k0), k1);
    uint16_t salt = uint16_t(h >> 48);
    uint64_t idx = h & ht.mask;
    while (true) {
      uint64_t& en = ht.entries[idx];
      uint32_t bidx = uint32_t(en);
      if (bidx == 0) {
        auto* pl = reinterpret_cast<Q1Payload*>(ht.Insert(en, h, salt));
        pl->hash = h;
        pl->rf = k0;
        pl->ls = k1;
        pl->sum_qty = q;
        pl->sum_price = p;
        pl->sum_disc_price = p * (1.0 - d);
        pl->sum_charge = p * (1.0 - d) * (1.0 + tx);
        pl->avg_qty = q;
        pl->cnt_qty = 1;
        pl->avg_price = p;
        pl->cnt_price = 1;
        pl->avg_disc = d;
        pl->cnt_disc = 1;
        pl->count = 1;
        break;
      }
      if (uint16_t(en >> 48) == salt) {
        auto* pl = reinterpret_cast<Q1Payload*>(ht.blocks[bidx] + uint16_t(en >> 32));
        if (pl->rf == k0 && pl->ls == k1) {
          pl->sum_qty = pl->sum_qty + q;
          pl->sum_price = pl->sum_price + p;
          pl->sum_disc_price = pl->sum_disc_price + p * (1.0 - d);
          pl->sum_charge = pl->sum_charge + p * (1.0 - d) * (1.0 + tx);
          pl->cnt_qty += 1;
          pl->avg_qty = pl->avg_qty + (q - pl->avg_qty) / pl->cnt_qty;
          pl->cnt_price += 1;
          pl->avg_price = pl->avg_price + (p - pl->avg_price) / pl->cnt_price;
          pl->cnt_disc += 1;
          pl->avg_disc = pl->avg_disc + (d - pl->avg_disc) / pl->cnt_disc;
          pl->count += 1;
          break;
        }
      }
      idx = (idx + 1) & ht.mask;
    }
  }
}

// Q1 output: merge the thread tables' groups (sums add, averages weighted
// by their counts), ORDER BY the two enum keys' string ranks.
void Q1Output(std::vector<Q1Part>& parts, const int32_t* rank_rf, const int32_t* rank_ls, double* out,
              int32_t max_groups, int32_t* ngroups) {
  std::vector<Q1Payload> rows;
  for (auto& part : parts)
    part.ht.ForEach([&](uint8_t* pp) {
      const Q1Payload& pl = *reinterpret_cast<Q1Payload*>(pp);
      for (auto& r : rows)
        if (r.rf == pl.rf && r.ls == pl.ls) {
          r.sum_qty += pl.sum_qty;
          r.sum_price += pl.sum_price;
          r.sum_disc_price += pl.sum_disc_price;
          r.sum_charge += pl.sum_charge;
          r.avg_qty = (r.avg_qty * r.cnt_qty + pl.avg_qty * pl.cnt_qty) / (r.cnt_qty + pl.cnt_qty);
          r.avg_price = (r.avg_price * r.cnt_price + pl.avg_price * pl.cnt_price) / (r.cnt_price + pl.cnt_price);
          r.avg_disc = (r.avg_disc * r.cnt_disc + pl.avg_disc * pl.cnt_disc) / (r.cnt_disc + pl.cnt_disc);
          r.cnt_qty += pl.cnt_qty;
          r.cnt_price += pl.cnt_price;
          r.cnt_disc += pl.cnt_disc;
          r.count += pl.count;
          return;
        }
      rows.push_back(pl);
    });
  std::vector<int32_t> order(rows.size()), tmp;
  for (size_t i = 0; i < rows.size(); i++) order[i] = int32_t(i);
  auto comp = [&](int32_t a, int32_t b) {
    if (rank_rf[rows[a].rf] < rank_rf[rows[b].rf]) return true;
    if (rank_rf[rows[b].rf] < rank_rf[rows[a].rf]) return false;
    if (rank_ls[rows[a].ls] < rank_ls[rows[b].ls]) return true;
    if (rank_ls[rows[b].ls] < rank_ls[rows[a].ls]) return false;
    return false;
  };
  if (!order.empty()) MergeSort(order, comp, 0, int(order.size()) - 1, tmp);
  int32_t g = 0;
  for (int32_t o : order) {
    if (g >= max_groups) break;
    const Q1Payload& pl = rows[o];
    double* r = out + 10 * g;
    r[0] = pl.rf;
    r[1] = pl.ls;
    r[2] = pl.sum_qty;
    r[3] = pl.sum_price;
    r[4] = pl.sum_disc_price;
    r[5] = pl.sum_charge;
    r[6] = pl.avg_qty;
    r[7] = pl.avg_price;
    r[8] = pl.avg_disc;
    r[9] = double(pl.count);
    g++;
  }
  *ngroups = int32_t(rows.size());
}

// runtime::HashTable: map<int32 hash, vector<packed tuple>>
using JoinTable = std::unordered_map<int32_t, std::vector<int32_t>>;

inline int32_t KeyHash(int32_t key) {
  int32_t h = 0;
  int64_t v = int64_t(uint32_t(key));  // INT hash = zext (value/int.cc:347-349)
  h ^= int32_t(v + 0x9e3779b9 + (int64_t(h) << 6) + (h >> 2));  // HashCombine
  return h;
}

struct Q3Payload {
  uint64_t hash;
  int32_t key;
  int32_t pad;
  double sum;
};

void Q3ProbeRange(const JoinTable& ht, const int32_t* okey, const double* oprice, const double* odisc, int64_t b,
                  int64_t e, AggTable& agg) {
  for (int64_t i = b; i < e; i++) {
    int32_t k = okey[i];
    auto it = ht.find(KeyHash(k));
    if (it == ht.end()) continue;
    for (int32_t bk : it->second) {
      if (bk != k) continue;
      double r = oprice[i] * (1.0 - odisc[i]);
      if (agg.size == agg.capacity || double(agg.size) > double(agg.capacity) / kLoadFactor) agg.Resize();
      uint64_t hh = MixKey(0, bk);
      uint16_t salt = uint16_t(hh >> 48);
      uint64_t idx = hh & agg.mask;
      while (true) {
        uint64_t& en = agg.entries[idx];
        uint32_t bidx = uint32_t(en);
        if (bidx == 0) {
          auto* pl = reinterpret_cast<Q3Payload*>(agg.Insert(en, hh, salt));
          pl->hash = hh;
          pl->key = bk;
          pl->sum = r;
          break;
        }
        if (uint16_t(en >> 48) == salt) {
          auto* pl = reinterpret_cast<Q3Payload*>(agg.blocks[bidx] + uint16_t(en >> 32));
          if (pl->key == bk) {
            pl->sum = pl->sum + r;
            break;
          }
        }
        idx = (idx + 1) & agg.mask;
      }
    }
  }
}

// ORDER BY sum DESC over the groups of all thread tables (merged by key)
void Q3Output(std::vector<AggTable*>& parts, int32_t top, int32_t* out_keys, double* out_sums, int32_t* ngroups) {
  std::vector<Q3Payload> rows;
  if (parts.size() == 1) {
    parts[0]->ForEach([&](uint8_t* p) { rows.push_back(*reinterpret_cast<Q3Payload*>(p)); });
  } else {
    std::unordered_map<int32_t, size_t> at;
    for (auto* part : parts)
      part->ForEach([&](uint8_t* p) {
        const Q3Payload& pl = *reinterpret_cast<Q3Payload*>(p);
        auto it = at.find(pl.key);
        if (it == at.end()) {
          at.emplace(pl.key, rows.size());
          rows.push_back(pl);
        } else {
          rows[it->second].sum += pl.sum;
        }
      });
  }
  std::vector<int32_t> order(rows.size()), tmp;
  for (size_t i = 0; i < rows.size(); i++) order[i] = int32_t(i);
  auto comp = [&](int32_t a, int32_t b) {
    if (rows[a].sum < rows[b].sum) return false;  // DESC
    if (rows[b].sum < rows[a].sum) return true;
    return false;
  };
  if (!order.empty()) MergeSort(order, comp, 0, int(order.size()) - 1, tmp);
  for (int32_t g = 0; g < top && g < int32_t(order.size()); g++) {
    out_keys[g] = rows[order[g]].key;
    out_sums[g] = rows[order[g]].sum;
  }
  *ngroups = int32_t(rows.size());
}

template <typename F>
void ParallelRanges(int threads, int64_t n, F f) {
  threads = std::max(1, threads);
  std::vector<std::thread> ts;
  for (int t = 0; t < threads; t++) {
    const int64_t b = n * t / threads, e = n * (t + 1) / threads;
    ts.emplace_back([&f, t, b, e] { f(t, b, e); });
  }
  for (auto& th : ts) th.join();
}

}  // namespace

extern "C" {

// ScanSelect(date < date_lt AND disc >= lo AND disc <= hi) -> Aggregate
// SUM(price*disc), COUNT(*).  Returns seconds; sum/count via out params.
double kdbo_baseline_scan_agg(const int32_t* date, const double* disc, const double* price,
                              int64_t n, int32_t date_lt, double lo, double hi, double* sum,
                              int64_t* count, int8_t* empty) {
  double t0 = Now();
  bool first = true;
  double s = 0;
  int64_t c = 0;
  for (int64_t i = 0; i < n; i++) {
    if (!(date[i] < date_lt)) continue;
    double d = disc[i];
    if (!(d >= lo)) continue;
    if (!(d <= hi)) continue;
    double v = price[i] * d;
    if (first) {
      s = v;
      c = 1;
      first = false;
    } else {
      s = s + v;
      c++;
    }
  }
  double t1 = Now();
  *sum = s;
  *count = c;
  *empty = first ? 1 : 0;
  return t1 - t0;
}

double kdbo_baseline_scan_agg_mt(const int32_t* date, const double* disc, const double* price, int64_t n,
                                 int32_t date_lt, double lo, double hi, double* sum, int64_t* count,
                                 int8_t* empty, int32_t threads) {
  double t0 = Now();
  const int T = std::max(1, int(threads));
  std::vector<double> ps(T, 0.0);
  std::vector<int64_t> pc(T, 0);
  std::vector<int8_t> pe(T, 1);
  ParallelRanges(T, n, [&](int t, int64_t b, int64_t e) {
    kdbo_baseline_scan_agg(date + b, disc + b, price + b, e - b, date_lt, lo, hi, &ps[t], &pc[t], &pe[t]);
  });
  double s = 0;
  int64_t c = 0;
  bool any = false;
  for (int t = 0; t < T; t++)
    if (!pe[t]) {
      s = any ? s + ps[t] : ps[t];
      c += pc[t];
      any = true;
    }
  double t1 = Now();
  *sum = s;
  *count = c;
  *empty = any ? 0 : 1;
  return t1 - t0;
}

// Q1 shape: ScanSelect(date <= date_leq) -> GroupBy(rf, ls) with
// SUM(qty), SUM(price), SUM(price*(1-disc)), SUM(price*(1-disc)*(1+tax)),
// AVG(qty), AVG(price), AVG(disc), COUNT(*) -> ORDER BY rf, ls (enum keys
// order by their strings; `rank_*` give each key's string rank).
// Writes up to max_groups rows of 10 doubles (rf, ls, 4 sums, 3 avgs,
// count) in output order; returns seconds.
double kdbo_baseline_group_by(const int32_t* date, const int32_t* rf, const int32_t* ls,
                              const double* qty, const double* price, const double* disc,
                              const double* tax, int64_t n, int32_t date_leq,
                              const int32_t* rank_rf, const int32_t* rank_ls, double* out,
                              int32_t max_groups, int32_t* ngroups) {
  double t0 = Now();
  std::vector<Q1Part> parts(1);
  Q1Range(date, rf, ls, qty, price, disc, tax, 0, n, date_leq, parts[0].ht);
  Q1Output(parts, rank_rf, rank_ls, out, max_groups, ngroups);
  return Now() - t0;
}

double kdbo_baseline_group_by_mt(const int32_t* date, const int32_t* rf, const int32_t* ls, const double* qty,
                                 const double* price, const double* disc, const double* tax, int64_t n,
                                 int32_t date_leq, const int32_t* rank_rf, const int32_t* rank_ls, double* out,
                                 int32_t max_groups, int32_t* ngroups, int32_t threads) {
  double t0 = Now();
  const int T = std::max(1, int(threads));
  std::vector<Q1Part> parts(T);
  ParallelRanges(T, n, [&](int t, int64_t b, int64_t e) {
    Q1Range(date, rf, ls, qty, price, disc, tax, b, e, date_leq, parts[t].ht);
  });
  Q1Output(parts, rank_rf, rank_ls, out, max_groups, ngroups);
  return Now() - t0;
}

// Q3 shape: build = ScanSelect(customer: date < date_lt AND segment == seg)
// into runtime::HashTable keyed by HashCombine(key); probe = Scan(orders)
// -> bucket loop -> CheckEquality -> GroupBy(custkey) SUM(price*(1-disc))
// -> ORDER BY sum DESC.  Writes the first `top` (key, sum) pairs.
double kdbo_baseline_join_group(const int32_t* ckey, const int32_t* cdate, const int32_t* cseg,
                                int64_t nb, int32_t date_lt, int32_t seg, const int32_t* okey,
                                const double* oprice, const double* odisc, int64_t np,
                                int32_t top, int32_t* out_keys, double* out_sums,
                                int32_t* ngroups) {
  double t0 = Now();
  JoinTable ht;
  for (int64_t i = 0; i < nb; i++) {
    if (!(cdate[i] < date_lt)) continue;
    if (!(cseg[i] == seg)) continue;
    ht[KeyHash(ckey[i])].push_back(ckey[i]);
  }
  AggTable agg(sizeof(Q3Payload));
  Q3ProbeRange(ht, okey, oprice, odisc, 0, np, agg);
  std::vector<AggTable*> parts{&agg};
  Q3Output(parts, top, out_keys, out_sums, ngroups);
  return Now() - t0;
}

// Multi-threaded: the build side is filtered in parallel and inserted in
// row order into one shared table; probe rows are split over the threads,
// each aggregating into its own table; the tables merge by key.
double kdbo_baseline_join_group_mt(const int32_t* ckey, const int32_t* cdate, const int32_t* cseg, int64_t nb,
                                   int32_t date_lt, int32_t seg, const int32_t* okey, const double* oprice,
                                   const double* odisc, int64_t np, int32_t top, int32_t* out_keys,
                                   double* out_sums, int32_t* ngroups, int32_t threads) {
  double t0 = Now();
  const int T = std::max(1, int(threads));
  std::vector<std::vector<int32_t>> pass(T);
  ParallelRanges(T, nb, [&](int t, int64_t b, int64_t e) {
    for (int64_t i = b; i < e; i++)
      if (cdate[i] < date_lt && cseg[i] == seg) pass[t].push_back(ckey[i]);
  });
  JoinTable ht;
  for (auto& v : pass)
    for (int32_t k : v) ht[KeyHash(k)].push_back(k);
  std::vector<std::unique_ptr<AggTable>> aggs;
  for (int t = 0; t < T; t++) aggs.push_back(std::make_unique<AggTable>(sizeof(Q3Payload)));
  ParallelRanges(T, np, [&](int t, int64_t b, int64_t e) { Q3ProbeRange(ht, okey, oprice, odisc, b, e, *aggs[t]); });
  std::vector<AggTable*> parts;
  for (auto& a : aggs) parts.push_back(a.get());
  Q3Output(parts, top, out_keys, out_sums, ngroups);
  return Now() - t0;
}

}  // extern "C"
