// CPU oracle for the KushDB hot path -- TEST INFRASTRUCTURE ONLY.
//
// Row-at-a-time, push-based restatement of what the reference's translators
// generate.  Each rule cites the reference file:line it follows.  Compiled
// with -ffp-contract=off so per-row float arithmetic is plain IEEE mul/add
// like the reference backends (khir/asm/asm_backend.cc:1834-1864,
// khir/llvm/llvm_backend.cc:140-141).
//
// Parity of this restatement with the reference is pinned by the reference's
// own golden tables (end_to_end_test/**/ *_expected.tbl, copied into
// tests/golden/ by tests/golden/make_fixtures.py).

#include "oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <random>
#include <set>
#include <string>
#include <string_view>
#include <unordered_map>
#include <vector>

#include "../kushdb_b200/csrc/host_result.h"
#include "../kushdb_b200/csrc/plan.h"

using namespace kdb::plan;

namespace {

struct Col {
  Type type;
  int64_t n = 0;
  std::vector<int64_t> i;
  std::vector<double> f;
  std::vector<int64_t> toff;
  std::string chars;
  std::vector<int8_t> null;  // empty = not nullable
};

struct Table {
  std::map<std::string, Col> cols;
  int64_t rows = -1;
};

struct Val {
  bool null = false;
  int64_t i = 0;
  double f = 0;
  std::string_view s;
};

using Row = std::vector<Val>;
using Consumer = std::function<void(const Row&)>;

struct Ctx {
  std::map<std::string, Table> tables;
  kdb::EnumDicts enums;
  std::string err;
  double last_exec_s = 0;
  int32_t skinner_budget = 10000;
  int32_t skinner_seed = 0;
};

struct EvalEnv {
  const Row* child[16] = {nullptr};
  const Row* virt = nullptr;
};

class Executor {
 public:
  explicit Executor(Ctx& ctx) : ctx_(ctx) {}

  // ------------------------------------------------------------------------
  // Expressions (compile/translators/expression_translator.cc:43-360,
  // compile/proxy/evaluate.cc)
  // ------------------------------------------------------------------------
  std::string_view EnumStr(int32_t enum_id, int64_t key) const {
    auto it = ctx_.enums.find(enum_id);
    if (it == ctx_.enums.end() || key < 0 || key >= (int64_t)it->second.size())
      throw std::runtime_error("enum key out of range");
    return it->second[key];
  }

  static Val Null() {
    Val v;
    v.null = true;
    return v;
  }
  static Val Bool(bool b) {
    Val v;
    v.i = b ? 1 : 0;
    return v;
  }

  // Arithmetic in the column type with wrap-around (evaluate.cc:84-140).
  static int64_t IntArith(TypeId t, BinOp op, int64_t a, int64_t b) {
    uint64_t ua = (uint64_t)a, ub = (uint64_t)b, r;
    switch (op) {
      case BinOp::ADD: r = ua + ub; break;
      case BinOp::SUB: r = ua - ub; break;
      case BinOp::MUL: r = ua * ub; break;
      default: throw std::runtime_error("Invalid arguments to div");
    }
    if (t == TypeId::SMALLINT) return (int16_t)(uint16_t)r;
    if (t == TypeId::INT) return (int32_t)(uint32_t)r;
    return (int64_t)r;
  }

  template <typename T>
  static bool Cmp(BinOp op, const T& a, const T& b) {
    switch (op) {
      case BinOp::EQ: return a == b;
      case BinOp::NEQ: return a != b;
      case BinOp::LT: return a < b;
      case BinOp::LEQ: return a <= b;
      case BinOp::GT: return a > b;
      case BinOp::GEQ: return a >= b;
      default: throw std::runtime_error("bad comparison");
    }
  }

  // Full match of LIKE tokens (literal byte / any byte but '\n' / any run of
  // bytes without '\n') by dynamic programming over (token, position).
  static bool LikeMatch(const std::vector<std::pair<int, unsigned char>>& tok, std::string_view s) {
    const size_t n = tok.size(), m = s.size();
    // ok[j] = tokens [i, n) match s[j, m)
    std::vector<char> ok(m + 1, 0), next(m + 1, 0);
    ok[m] = 1;
    for (size_t i = n; i-- > 0;) {
      std::fill(next.begin(), next.end(), 0);
      for (size_t j = m + 1; j-- > 0;) {
        const int kind = tok[i].first;
        if (kind == 2) {
          next[j] = ok[j] || (j < m && s[j] != '\n' && next[j + 1]);
        } else if (j < m) {
          const bool hit = kind == 1 ? s[j] != '\n' : (unsigned char)s[j] == tok[i].second;
          next[j] = hit && ok[j + 1];
        }
      }
      ok.swap(next);
    }
    return ok[0];
  }

  Val Eval(const Expr& e, const EvalEnv& env) const {
    switch (e.kind) {
      case ExprKind::ColRef: {
        const Row* r = env.child[e.child_idx];
        if (!r) throw std::runtime_error("column reference to unbound child");
        return (*r)[e.column_idx];
      }
      case ExprKind::VirtColRef:
        return (*env.virt)[e.column_idx];
      case ExprKind::Literal: {
        Val v;
        v.null = e.lit_null;
        v.i = e.ival;
        v.f = e.fval;
        v.s = e.sval;
        return v;
      }
      case ExprKind::Unary: {
        Val c = Eval(e.kid(0), env);
        if (e.uop == UnOp::IS_NULL) return Bool(c.null);
        // NOT: NULL stays NULL (expression_translator.cc:53-67)
        if (c.null) return Null();
        return Bool(!c.i);
      }
      case ExprKind::Case: {
        // cond NULL or false -> else (expression_translator.cc:180-192)
        Val c = Eval(e.kid(0), env);
        if (!c.null && c.i) return Eval(e.kid(1), env);
        return Eval(e.kid(2), env);
      }
      case ExprKind::IntToFloat: {
        // NULL input gives a non-NULL 0.0 (expression_translator.cc:232-262)
        Val c = Eval(e.kid(0), env);
        Val v;
        v.f = c.null ? 0.0 : (double)c.i;
        return v;
      }
      case ExprKind::Extract: {
        Val c = Eval(e.kid(0), env);
        if (c.null) return Null();
        Val v;
        v.i = kdb::ExtractYear((int32_t)c.i);
        return v;
      }
      case ExprKind::EnumIn: {
        // NULL -> false (expression_translator.cc:332-350)
        Val c = Eval(e.kid(0), env);
        if (c.null) return Bool(false);
        for (int32_t x : e.in_values)
          if (x == c.i) return Bool(true);
        return Bool(false);
      }
      case ExprKind::Regexp: {
        // RE2::FullMatch of the planner's ^...$ pattern
        // (expression_translator.cc:277-297, planner.cc:283-321): NULL ->
        // false; an ENUM matches through its string
        Val c = Eval(e.kid(0), env);
        if (c.null) return Bool(false);
        const Type& ct = e.kid(0).type;
        std::string_view s = ct.id == TypeId::ENUM ? EnumStr(ct.enum_id, c.i) : std::string_view(c.s);
        return Bool(LikeMatch(LikeTokens(e.regex), s));
      }
      case ExprKind::Agg:
        throw std::runtime_error("Aggregate expression can't be derived");
      case ExprKind::Binary: break;
    }

    // Binary
    if (e.bop == BinOp::AND) {
      // left NULL -> NULL; left false -> false; else right
      // (expression_translator.cc:74-91)
      Val l = Eval(e.kid(0), env);
      if (l.null) return Null();
      if (!l.i) return Bool(false);
      return Eval(e.kid(1), env);
    }
    if (e.bop == BinOp::OR) {
      // left NULL -> right; left true -> true; else right
      // (expression_translator.cc:93-108)
      Val l = Eval(e.kid(0), env);
      if (l.null) return Eval(e.kid(1), env);
      if (l.i) return Bool(true);
      return Eval(e.kid(1), env);
    }
    Val l = Eval(e.kid(0), env);
    Val r = Eval(e.kid(1), env);
    if (l.null || r.null) return Null();
    const Type& lt = e.kid(0).type;
    const Type& rt = e.kid(1).type;
    switch (lt.id) {
      case TypeId::BOOLEAN:
        return Bool(Cmp(e.bop, l.i != 0, r.i != 0));
      case TypeId::SMALLINT:
      case TypeId::INT:
      case TypeId::BIGINT:
      case TypeId::DATE:
        if (e.bop == BinOp::ADD || e.bop == BinOp::SUB || e.bop == BinOp::MUL ||
            e.bop == BinOp::DIV) {
          Val v;
          v.i = IntArith(lt.id, e.bop, l.i, r.i);
          return v;
        }
        return Bool(Cmp(e.bop, l.i, r.i));
      case TypeId::REAL: {
        Val v;
        switch (e.bop) {
          case BinOp::ADD: v.f = l.f + r.f; return v;
          case BinOp::SUB: v.f = l.f - r.f; return v;
          case BinOp::MUL: v.f = l.f * r.f; return v;
          case BinOp::DIV: v.f = l.f / r.f; return v;
          default: return Bool(Cmp(e.bop, l.f, r.f));
        }
      }
      case TypeId::TEXT: {
        switch (e.bop) {
          case BinOp::STARTS_WITH: return Bool(l.s.rfind(r.s, 0) == 0);
          case BinOp::ENDS_WITH:
            return Bool(l.s.size() >= r.s.size() &&
                        l.s.compare(l.s.size() - r.s.size(), r.s.size(), r.s) == 0);
          case BinOp::CONTAINS: return Bool(l.s.find(r.s) != std::string_view::npos);
          default: return Bool(Cmp(e.bop, l.s, r.s));
        }
      }
      case TypeId::ENUM: {
        // EQ/NEQ on keys; ordering and string ops on the key's string
        // (evaluate.cc:186-268)
        if (e.bop == BinOp::EQ) return Bool(l.i == r.i);
        if (e.bop == BinOp::NEQ) return Bool(l.i != r.i);
        std::string_view ls = EnumStr(lt.enum_id, l.i);
        std::string_view rs = rt.id == TypeId::ENUM ? EnumStr(rt.enum_id, r.i) : r.s;
        switch (e.bop) {
          case BinOp::STARTS_WITH: return Bool(ls.rfind(rs, 0) == 0);
          case BinOp::ENDS_WITH:
            return Bool(ls.size() >= rs.size() &&
                        ls.compare(ls.size() - rs.size(), rs.size(), rs) == 0);
          case BinOp::CONTAINS: return Bool(ls.find(rs) != std::string_view::npos);
          default: return Bool(Cmp(e.bop, ls, rs));
        }
      }
    }
    throw std::runtime_error("unhandled binary expression");
  }

  // proxy::Equal (evaluate.cc:404-470): NULL equals NULL.
  bool Equal(const Type& t, const Val& a, const Val& b) const {
    if (a.null && b.null) return true;
    if (a.null || b.null) return false;
    switch (t.id) {
      case TypeId::REAL: return a.f == b.f;
      case TypeId::TEXT: return a.s == b.s;
      case TypeId::BOOLEAN: return (a.i != 0) == (b.i != 0);
      default: return a.i == b.i;
    }
  }

  // proxy::LessThan (evaluate.cc:339-402): NULL sorts after every value.
  bool LessThan(const Type& t, const Val& a, const Val& b) const {
    if (a.null && b.null) return false;
    if (a.null) return false;
    if (b.null) return true;
    switch (t.id) {
      case TypeId::REAL: return a.f < b.f;
      case TypeId::TEXT: return a.s < b.s;
      case TypeId::ENUM: return EnumStr(t.enum_id, a.i) < EnumStr(t.enum_id, b.i);
      case TypeId::BOOLEAN: throw std::runtime_error("Can't be less than.");
      default: return a.i < b.i;
    }
  }

  // ------------------------------------------------------------------------
  // Aggregators (compile/proxy/aggregator.cc)
  // ------------------------------------------------------------------------
  struct AggState {
    Val v;         // SUM/MIN/MAX value, AVG cma
    double cnt = 0;  // AVG record count (stored as REAL, aggregator.cc:189-195)
    int64_t count = 0;
  };

  void AggInit(const Expr& agg, AggState& s, const EvalEnv& env) const {
    Val next = Eval(agg.kid(0), env);
    switch (agg.agg) {
      case AggType::SUM:
      case AggType::MIN:
      case AggType::MAX:
        // Initialize stores the first value, NULL or not (aggregator.cc:28-30,
        // :100-102)
        s.v = next;
        break;
      case AggType::AVG:
        // value = NULL ? (0, null) : float(value); count = 1 (aggregator.cc:197-216)
        s.v = Val();
        if (next.null) {
          s.v.null = true;
          s.v.f = 0;
        } else {
          s.v.f = agg.kid(0).type.id == TypeId::REAL ? next.f : (double)next.i;
        }
        s.cnt = 1;
        break;
      case AggType::COUNT:
        // COUNT starts at 1 for the first row whether or not it is NULL
        // (aggregator.cc:285-287)
        s.count = 1;
        break;
    }
  }

  void AggUpdate(const Expr& agg, AggState& s, const EvalEnv& env) const {
    Val next = Eval(agg.kid(0), env);
    if (next.null) return;
    const Type& t = agg.kid(0).type;
    switch (agg.agg) {
      case AggType::SUM:
        // aggregator.cc:32-82
        if (s.v.null) {
          s.v = next;
        } else if (t.id == TypeId::REAL) {
          s.v.f = s.v.f + next.f;
        } else {
          s.v.i = IntArith(t.id, BinOp::ADD, s.v.i, next.i);
        }
        break;
      case AggType::MIN:
      case AggType::MAX: {
        // aggregator.cc:104-178; ENUM compares strings
        if (s.v.null) {
          s.v = next;
          break;
        }
        bool is_min = agg.agg == AggType::MIN;
        bool take;
        switch (t.id) {
          case TypeId::REAL: take = is_min ? next.f < s.v.f : s.v.f < next.f; break;
          case TypeId::TEXT: take = is_min ? next.s < s.v.s : s.v.s < next.s; break;
          case TypeId::ENUM: {
            auto a = EnumStr(t.enum_id, next.i), b = EnumStr(t.enum_id, s.v.i);
            take = is_min ? a < b : b < a;
            break;
          }
          default: take = is_min ? next.i < s.v.i : s.v.i < next.i; break;
        }
        if (take) s.v = next;
        break;
      }
      case AggType::AVG: {
        // cumulative moving average (aggregator.cc:239-268)
        double x = t.id == TypeId::REAL ? next.f : (double)next.i;
        if (s.v.null) {
          s.v.null = false;
          s.v.f = x;
        } else {
          double n = s.cnt + 1;
          s.v.f = s.v.f + (x - s.v.f) / n;
          s.cnt = n;
        }
        break;
      }
      case AggType::COUNT:
        s.count += 1;  // aggregator.cc:289-295
        break;
    }
  }

  Val AggGet(const Expr& agg, const AggState& s) const {
    if (agg.agg == AggType::COUNT) {
      Val v;
      v.i = s.count;
      return v;
    }
    return s.v;
  }

  // ------------------------------------------------------------------------
  // Operators
  // ------------------------------------------------------------------------
  const Table& GetTable(const std::string& name) const {
    auto it = ctx_.tables.find(name);
    if (it == ctx_.tables.end()) throw std::runtime_error("unknown relation " + name);
    return it->second;
  }

  const Col& GetCol(const Table& t, const std::string& name) const {
    auto it = t.cols.find(name);
    if (it == t.cols.end()) throw std::runtime_error("unknown column " + name);
    return it->second;
  }

  static Val Load(const Col& c, int64_t r) {
    Val v;
    if (!c.null.empty() && c.null[r]) {
      v.null = true;
      return v;
    }
    switch (c.type.id) {
      case TypeId::REAL: v.f = c.f[r]; break;
      case TypeId::TEXT:
        v.s = std::string_view(c.chars.data() + c.toff[r], c.toff[r + 1] - c.toff[r]);
        break;
      default: v.i = c.i[r]; break;
    }
    return v;
  }

  void Produce(const Operator& op, const Consumer& consume) {
    switch (op.kind) {
      case OpKind::SCAN: return ProduceScan(op, consume);
      case OpKind::SCAN_SELECT: return ProduceScanSelect(op, consume);
      case OpKind::SELECT: return ProduceSelect(op, consume);
      case OpKind::HASH_JOIN: return ProduceHashJoin(op, consume);
      case OpKind::CROSS_PRODUCT: return ProduceCrossProduct(op, consume);
      case OpKind::GROUP_BY_AGGREGATE: return ProduceGroupBy(op, consume);
      case OpKind::AGGREGATE: return ProduceAggregate(op, consume);
      case OpKind::ORDER_BY: return ProduceOrderBy(op, consume);
      case OpKind::SKINNER_JOIN: return ProduceSkinner(op, consume);
      case OpKind::OUTPUT: return Produce(op.child(), consume);
    }
  }

  // scan_translator.cc:140-168: every row, every catalog column.
  void ProduceScan(const Operator& op, const Consumer& consume) {
    const Table& t = GetTable(op.relation);
    std::vector<const Col*> cols;
    for (const auto& c : op.scan_columns) cols.push_back(&GetCol(t, c.name));
    int64_t n = cols.empty() ? 0 : cols[0]->n;
    Row scan(cols.size()), out(op.output.size());
    EvalEnv env;
    env.child[0] = &scan;
    for (int64_t r = 0; r < n; r++) {
      for (size_t k = 0; k < cols.size(); k++) scan[k] = Load(*cols[k], r);
      for (size_t k = 0; k < op.output.size(); k++) out[k] = Eval(*op.output[k].expr, env);
      consume(out);
    }
  }

  // scan_select_translator.cc:92-156: filters in order over the scan schema
  // (virtual values); NULL or false drops the row; then the output schema.
  void ProduceScanSelect(const Operator& op, const Consumer& consume) {
    const Table& t = GetTable(op.relation);
    std::vector<const Col*> cols;
    for (const auto& c : op.scan_columns) cols.push_back(&GetCol(t, c.name));
    int64_t n = cols.empty() ? 0 : cols[0]->n;
    Row scan(cols.size()), out(op.output.size());
    EvalEnv env;
    env.virt = &scan;
    for (int64_t r = 0; r < n; r++) {
      for (size_t k = 0; k < cols.size(); k++) scan[k] = Load(*cols[k], r);
      bool keep = true;
      for (const auto& f : op.filters) {
        Val v = Eval(*f, env);
        if (v.null || !v.i) {
          keep = false;
          break;
        }
      }
      if (!keep) continue;
      for (size_t k = 0; k < op.output.size(); k++) out[k] = Eval(*op.output[k].expr, env);
      consume(out);
    }
  }

  // select_translator.cc:19-37
  void ProduceSelect(const Operator& op, const Consumer& consume) {
    Row out(op.output.size());
    Produce(op.child(), [&](const Row& in) {
      EvalEnv env;
      env.child[0] = &in;
      Val v = Eval(*op.filters[0], env);
      if (v.null || !v.i) return;
      for (size_t k = 0; k < op.output.size(); k++) out[k] = Eval(*op.output[k].expr, env);
      consume(out);
    });
  }

  // Key tuples with proxy::Equal semantics (NULL == NULL, -0.0 == 0.0).
  struct KeyPart {
    bool null;
    int64_t i;
    double f;
    std::string s;
    bool operator<(const KeyPart& o) const {
      if (null != o.null) return null < o.null;
      if (null) return false;
      if (i != o.i) return i < o.i;
      if (f != o.f) return f < o.f;
      return s < o.s;
    }
  };
  static KeyPart MakeKeyPart(const Type& t, const Val& v) {
    KeyPart k{v.null, 0, 0.0, {}};
    if (v.null) return k;
    switch (t.id) {
      case TypeId::REAL: k.f = v.f == 0.0 ? 0.0 : v.f; break;
      case TypeId::TEXT: k.s = std::string(v.s); break;
      case TypeId::BOOLEAN: k.i = v.i != 0; break;
      default: k.i = v.i; break;
    }
    return k;
  }

  // cross_product_translator.cc:19-74: the left child is buffered in its
  // stream order; every right row then meets every buffered left row.
  void ProduceCrossProduct(const Operator& op, const Consumer& consume) {
    std::vector<Row> left;
    Produce(op.child(0), [&](const Row& in) { left.push_back(in); });
    Row out(op.output.size());
    Produce(op.child(1), [&](const Row& in) {
      EvalEnv env;
      env.child[1] = &in;
      for (const Row& l : left) {
        env.child[0] = &l;
        for (size_t k = 0; k < op.output.size(); k++) out[k] = Eval(*op.output[k].expr, env);
        consume(out);
      }
    });
  }

  // hash_join_translator.cc:34-139.  Build = left child, rows with a NULL key
  // skipped (:86-101).  A probe row visits the bucket of its hash in insertion
  // order and keeps the rows whose keys are Equal (:106-138); the bucket
  // restricted to equal keys is exactly the equal-key build rows in insertion
  // order, which is what this map holds.
  void ProduceHashJoin(const Operator& op, const Consumer& consume) {
    std::map<std::vector<KeyPart>, std::vector<Row>> table;
    Produce(op.child(0), [&](const Row& in) {
      EvalEnv env;
      env.child[0] = &in;
      std::vector<KeyPart> key;
      for (const auto& k : op.left_keys) {
        Val v = Eval(*k, env);
        if (v.null) return;
        key.push_back(MakeKeyPart(k->type, v));
      }
      table[key].push_back(in);
    });
    Row out(op.output.size());
    Produce(op.child(1), [&](const Row& in) {
      EvalEnv env;
      env.child[1] = &in;
      std::vector<KeyPart> key;
      for (const auto& k : op.right_keys) {
        Val v = Eval(*k, env);
        if (v.null) return;  // a NULL probe key is never Equal to a non-NULL build key
        key.push_back(MakeKeyPart(k->type, v));
      }
      auto it = table.find(key);
      if (it == table.end()) return;
      for (const Row& left : it->second) {
        env.child[0] = &left;
        for (size_t k = 0; k < op.output.size(); k++) out[k] = Eval(*op.output[k].expr, env);
        consume(out);
      }
    });
  }

  // group_by_aggregate_translator.cc:36-111 + AggregateHashTable: groups are
  // emitted by ForEach over the payload blocks, i.e. in first-insertion order
  // (compile/proxy/aggregate_hash_table.cc:245-291, runtime Insert appends).
  void ProduceGroupBy(const Operator& op, const Consumer& consume) {
    std::map<std::vector<KeyPart>, size_t> index;
    std::vector<Row> keys;
    std::vector<std::vector<AggState>> states;
    Produce(op.child(), [&](const Row& in) {
      EvalEnv env;
      env.child[0] = &in;
      Row kv;
      std::vector<KeyPart> key;
      for (const auto& g : op.group_by) {
        Val v = Eval(*g, env);
        kv.push_back(v);
        key.push_back(MakeKeyPart(g->type, v));
      }
      auto it = index.find(key);
      if (it == index.end()) {
        index.emplace(std::move(key), keys.size());
        // key string views point into column / literal storage that outlives
        // the query
        keys.push_back(kv);
        states.emplace_back(op.aggs.size());
        for (size_t a = 0; a < op.aggs.size(); a++) AggInit(*op.aggs[a], states.back()[a], env);
      } else {
        auto& st = states[it->second];
        for (size_t a = 0; a < op.aggs.size(); a++) AggUpdate(*op.aggs[a], st[a], env);
      }
    });
    Row virt, out(op.output.size());
    for (size_t g = 0; g < keys.size(); g++) {
      virt = keys[g];
      for (size_t a = 0; a < op.aggs.size(); a++) virt.push_back(AggGet(*op.aggs[a], states[g][a]));
      EvalEnv env;
      env.virt = &virt;
      for (size_t k = 0; k < op.output.size(); k++) out[k] = Eval(*op.output[k].expr, env);
      consume(out);
    }
  }

  // aggregate_translator.cc:34-126: the first row initialises, later rows
  // update; an empty input emits one all-NULL row (:82-89).
  void ProduceAggregate(const Operator& op, const Consumer& consume) {
    std::vector<AggState> st(op.aggs.size());
    bool empty = true;
    Produce(op.child(), [&](const Row& in) {
      EvalEnv env;
      env.child[0] = &in;
      if (empty) {
        for (size_t a = 0; a < op.aggs.size(); a++) AggInit(*op.aggs[a], st[a], env);
        empty = false;
      } else {
        for (size_t a = 0; a < op.aggs.size(); a++) AggUpdate(*op.aggs[a], st[a], env);
      }
    });
    Row out(op.output.size());
    if (empty) {
      for (auto& v : out) v = Null();
      consume(out);
      return;
    }
    Row virt;
    for (size_t a = 0; a < op.aggs.size(); a++) virt.push_back(AggGet(*op.aggs[a], st[a]));
    EvalEnv env;
    env.virt = &virt;
    for (size_t k = 0; k < op.output.size(); k++) out[k] = Eval(*op.output[k].expr, env);
    consume(out);
  }

  // order_by_translator.cc:35-110 + runtime::Vector::Sort (vector.cc:45-110):
  // top-down merge sort whose merge takes the left element only when
  // comp(left, right) is true, so ties take the right run first.
  void MergeSort(std::vector<Row>& v, const std::function<bool(const Row&, const Row&)>& comp,
                 int l, int r) {
    if (l >= r) return;
    int m = l + (r - l) / 2;
    MergeSort(v, comp, l, m);
    MergeSort(v, comp, m + 1, r);
    std::vector<Row> a(v.begin() + l, v.begin() + m + 1), b(v.begin() + m + 1, v.begin() + r + 1);
    size_t i = 0, j = 0;
    int k = l;
    while (i < a.size() && j < b.size()) {
      if (comp(a[i], b[j])) v[k++] = a[i++];
      else v[k++] = b[j++];
    }
    while (i < a.size()) v[k++] = a[i++];
    while (j < b.size()) v[k++] = b[j++];
  }

  void ProduceOrderBy(const Operator& op, const Consumer& consume) {
    std::vector<Row> buf;
    Produce(op.child(), [&](const Row& in) { buf.push_back(in); });
    const auto& child_schema = SchemaOf(op.child());
    auto comp = [&](const Row& s1, const Row& s2) {
      for (size_t k = 0; k < op.sort_keys.size(); k++) {
        int idx = op.sort_keys[k]->column_idx;
        const Type& t = child_schema[idx].expr->type;
        bool asc = op.asc[k];
        if (LessThan(t, s1[idx], s2[idx])) return asc;
        if (LessThan(t, s2[idx], s1[idx])) return !asc;
      }
      return false;
    };
    if (!buf.empty()) MergeSort(buf, comp, 0, (int)buf.size() - 1);
    Row out(op.output.size());
    for (const Row& in : buf) {
      EvalEnv env;
      env.child[0] = &in;
      for (size_t k = 0; k < op.output.size(); k++) out[k] = Eval(*op.output[k].expr, env);
      consume(out);
    }
  }

  // SkinnerJoin: the result is the set of child-tuple combinations that
  // satisfy every condition, each emitted once (the TupleIdxTable dedup of
  // permutable_skinner_join_translator.cc:842-912); join order only changes
  // the emission order, which the reference's tests do not compare
  // (end_to_end_test/skinner_join/*_test.cc sort both sides).  Restated here
  // as a left-deep join in child order with each condition checked as soon
  // as every child it references is bound.
  void ProduceSkinner(const Operator& op, const Consumer& consume) {
    size_t nt = op.children.size();
    std::vector<std::vector<Row>> rows(nt);
    for (size_t t = 0; t < nt; t++)
      Produce(op.child(t), [&](const Row& in) { rows[t].push_back(in); });
    // tables referenced by each condition
    std::vector<std::vector<int>> cond_tables(op.conditions.size());
    std::function<void(const Expr&, std::set<int>&)> collect = [&](const Expr& e,
                                                                   std::set<int>& s) {
      if (e.kind == ExprKind::ColRef) s.insert(e.child_idx);
      for (const auto& k : e.kids) collect(*k, s);
    };
    std::vector<int> ready_at(op.conditions.size(), 0);
    for (size_t c = 0; c < op.conditions.size(); c++) {
      std::set<int> s;
      collect(*op.conditions[c], s);
      ready_at[c] = s.empty() ? 0 : *s.rbegin();
    }
    // Equality conditions between the new table and an earlier one are
    // answered through a hash index on the new table's column.
    struct EqIdx {
      int cond;
      int other_table, other_col;
      std::map<KeyPart, std::vector<int64_t>> idx;
    };
    std::vector<std::vector<EqIdx>> eq(nt);
    for (size_t c = 0; c < op.conditions.size(); c++) {
      const Expr& e = *op.conditions[c];
      if (e.kind != ExprKind::Binary || e.bop != BinOp::EQ) continue;
      const Expr& a = e.kid(0);
      const Expr& b = e.kid(1);
      if (a.kind != ExprKind::ColRef || b.kind != ExprKind::ColRef) continue;
      if (a.child_idx == b.child_idx) continue;
      const Expr& hi = a.child_idx > b.child_idx ? a : b;
      const Expr& lo = a.child_idx > b.child_idx ? b : a;
      EqIdx ix;
      ix.cond = (int)c;
      ix.other_table = lo.child_idx;
      ix.other_col = lo.column_idx;
      for (int64_t r = 0; r < (int64_t)rows[hi.child_idx].size(); r++) {
        const Val& v = rows[hi.child_idx][r][hi.column_idx];
        if (v.null) continue;
        ix.idx[MakeKeyPart(hi.type, v)].push_back(r);
      }
      eq[hi.child_idx].push_back(std::move(ix));
    }
    EvalEnv env;
    Row out(op.output.size());
    std::function<void(size_t)> rec = [&](size_t t) {
      if (t == nt) {
        for (size_t k = 0; k < op.output.size(); k++) out[k] = Eval(*op.output[k].expr, env);
        consume(out);
        return;
      }
      auto try_row = [&](int64_t r) {
        env.child[t] = &rows[t][r];
        for (size_t c = 0; c < op.conditions.size(); c++) {
          if (ready_at[c] != (int)t) continue;
          Val v = Eval(*op.conditions[c], env);
          if (v.null || !v.i) return;
        }
        rec(t + 1);
      };
      if (!eq[t].empty()) {
        const EqIdx& ix = eq[t][0];
        const Val& key = (*env.child[ix.other_table])[ix.other_col];
        if (key.null) return;
        auto it = ix.idx.find(MakeKeyPart(op.conditions[ix.cond]->kid(0).type, key));
        if (it == ix.idx.end()) return;
        for (int64_t r : it->second) try_row(r);
      } else {
        for (int64_t r = 0; r < (int64_t)rows[t].size(); r++) try_row(r);
      }
      env.child[t] = nullptr;
    };
    rec(0);
  }

  Ctx& ctx_;
};

void Collect(const Operator& root, const Row& row, kdb::HostResult& res) {
  const auto& schema = SchemaOf(root);
  if (res.cols.empty()) {
    for (const auto& c : schema) {
      kdb::HostColumn hc;
      hc.name = c.name;
      hc.type = c.expr->type;
      res.cols.push_back(std::move(hc));
    }
  }
  for (size_t k = 0; k < row.size(); k++) {
    auto& hc = res.cols[k];
    const Val& v = row[k];
    hc.null.push_back(v.null ? 1 : 0);
    switch (hc.type.id) {
      case TypeId::REAL: hc.f.push_back(v.null ? 0.0 : v.f); break;
      case TypeId::TEXT: hc.s.emplace_back(v.null ? std::string_view() : v.s); break;
      default: hc.i.push_back(v.null ? 0 : v.i); break;
    }
  }
  res.rows++;
}

}  // namespace

struct kdbo_ctx {
  Ctx c;
};
struct kdbo_result {
  kdb::HostResult r;
};

extern "C" {

kdbo_ctx* kdbo_create(void) { return new kdbo_ctx(); }
void kdbo_destroy(kdbo_ctx* ctx) { delete ctx; }
const char* kdbo_last_error(kdbo_ctx* ctx) { return ctx ? ctx->c.err.c_str() : "null ctx"; }

static int SetTableRows(Ctx& c, Table& t, int64_t n) {
  if (t.rows >= 0 && t.rows != n) {
    c.err = "column length differs from the table's other columns";
    return -1;
  }
  t.rows = n;
  return 0;
}

int kdbo_register_column(kdbo_ctx* ctx, const char* table, const char* column, const char* type,
                         const void* data, int64_t n, const int8_t* nulls) {
  try {
    Table& t = ctx->c.tables[table];
    if (SetTableRows(ctx->c, t, n)) return -1;
    Col col;
    col.type = ParseType(type);
    col.n = n;
    switch (col.type.id) {
      case TypeId::REAL: {
        const double* d = (const double*)data;
        col.f.assign(d, d + n);
        break;
      }
      case TypeId::BOOLEAN: {
        const int8_t* d = (const int8_t*)data;
        col.i.assign(d, d + n);
        break;
      }
      case TypeId::SMALLINT: {
        const int16_t* d = (const int16_t*)data;
        col.i.assign(d, d + n);
        break;
      }
      case TypeId::BIGINT: {
        const int64_t* d = (const int64_t*)data;
        col.i.assign(d, d + n);
        break;
      }
      case TypeId::TEXT: ctx->c.err = "use kdbo_register_text_column"; return -1;
      default: {
        const int32_t* d = (const int32_t*)data;
        col.i.assign(d, d + n);
        break;
      }
    }
    if (nulls) col.null.assign(nulls, nulls + n);
    t.cols[column] = std::move(col);
    return 0;
  } catch (const std::exception& e) {
    ctx->c.err = e.what();
    return -1;
  }
}

int kdbo_register_text_column(kdbo_ctx* ctx, const char* table, const char* column,
                              const int64_t* offsets, const char* chars, int64_t n,
                              const int8_t* nulls) {
  Table& t = ctx->c.tables[table];
  if (SetTableRows(ctx->c, t, n)) return -1;
  Col col;
  col.type = Type{TypeId::TEXT, 0};
  col.n = n;
  col.toff.assign(offsets, offsets + n + 1);
  col.chars.assign(chars, chars + offsets[n]);
  if (nulls) col.null.assign(nulls, nulls + n);
  t.cols[column] = std::move(col);
  return 0;
}

int kdbo_register_enum(kdbo_ctx* ctx, int32_t enum_id, const int64_t* offsets, const char* chars,
                       int32_t n) {
  std::vector<std::string> v;
  for (int32_t k = 0; k < n; k++) v.emplace_back(chars + offsets[k], offsets[k + 1] - offsets[k]);
  ctx->c.enums[enum_id] = std::move(v);
  return 0;
}

void kdbo_set_skinner_options(kdbo_ctx* ctx, int32_t budget, int32_t seed) {
  ctx->c.skinner_budget = budget;
  ctx->c.skinner_seed = seed;
}

int kdbo_execute(kdbo_ctx* ctx, const char* plan_json, kdbo_result** out) {
  try {
    auto plan = ParsePlan(plan_json);
    auto res = std::make_unique<kdbo_result>();
    Executor ex(ctx->c);
    auto t0 = std::chrono::steady_clock::now();
    // Column metadata comes from the root schema even when no row is produced.
    const auto& schema = SchemaOf(*plan);
    for (const auto& c : schema) {
      kdb::HostColumn hc;
      hc.name = c.name;
      hc.type = c.expr->type;
      res->r.cols.push_back(std::move(hc));
    }
    ex.Produce(*plan, [&](const Row& row) { Collect(*plan, row, res->r); });
    auto t1 = std::chrono::steady_clock::now();
    ctx->c.last_exec_s = std::chrono::duration<double>(t1 - t0).count();
    *out = res.release();
    return 0;
  } catch (const std::exception& e) {
    ctx->c.err = e.what();
    return -1;
  }
}

double kdbo_last_exec_seconds(kdbo_ctx* ctx) { return ctx->c.last_exec_s; }

int64_t kdbo_result_num_rows(const kdbo_result* r) { return r->r.rows; }
int32_t kdbo_result_num_cols(const kdbo_result* r) { return (int32_t)r->r.cols.size(); }

int kdbo_result_col_type(const kdbo_result* r, int32_t col, char* buf, int32_t cap) {
  if (col < 0 || col >= (int32_t)r->r.cols.size()) return -1;
  const auto& t = r->r.cols[col].type;
  std::string s = t.id == TypeId::ENUM ? "ENUM:" + std::to_string(t.enum_id) : TypeName(t.id);
  std::snprintf(buf, cap, "%s", s.c_str());
  return 0;
}

int kdbo_result_get_i64(const kdbo_result* r, int32_t col, int64_t* out) {
  if (col < 0 || col >= (int32_t)r->r.cols.size()) return -1;
  const auto& c = r->r.cols[col];
  if (c.i.size() != (size_t)r->r.rows) return -1;
  std::copy(c.i.begin(), c.i.end(), out);
  return 0;
}

int kdbo_result_get_f64(const kdbo_result* r, int32_t col, double* out) {
  if (col < 0 || col >= (int32_t)r->r.cols.size()) return -1;
  const auto& c = r->r.cols[col];
  if (c.f.size() != (size_t)r->r.rows) return -1;
  std::copy(c.f.begin(), c.f.end(), out);
  return 0;
}

int kdbo_result_get_nulls(const kdbo_result* r, int32_t col, int8_t* out) {
  if (col < 0 || col >= (int32_t)r->r.cols.size()) return -1;
  const auto& c = r->r.cols[col];
  std::copy(c.null.begin(), c.null.end(), out);
  return 0;
}

int64_t kdbo_result_get_text(const kdbo_result* r, int32_t col, int64_t row, char* buf,
                             int64_t cap) {
  if (col < 0 || col >= (int32_t)r->r.cols.size()) return -1;
  const auto& c = r->r.cols[col];
  if (row < 0 || row >= (int64_t)c.s.size()) return -1;
  const std::string& s = c.s[row];
  if (buf && cap > 0) std::memcpy(buf, s.data(), std::min<int64_t>(cap, s.size()));
  return (int64_t)s.size();
}

int64_t kdbo_result_format(kdbo_ctx* ctx, const kdbo_result* r, char* buf, int64_t cap) {
  std::string s = kdb::FormatResult(r->r, ctx->c.enums);
  if (buf && cap > 0) {
    int64_t n = std::min<int64_t>(cap - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return (int64_t)s.size() + 1;
}

void kdbo_result_free(kdbo_result* r) { delete r; }

}  // extern "C"
