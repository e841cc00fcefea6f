// Plan executor + pipeline code generator.
//
// Follows the reference's produce/consume translation
// (compile/translators/operator_translator.h:13-38): a plan is cut into
// pipelines at the same breakers the reference uses -- hash-join build side
// (hash_join_translator.cc:34-55), group-by / aggregate
// (group_by_aggregate_translator.cc:36-111, aggregate_translator.cc:34-126),
// order-by materialisation (order_by_translator.cc:35-110) and Skinner
// children (permutable_skinner_join_translator.cc:111-204).  Each pipeline
// becomes ONE CUDA kernel (the reference's body_N becomes a grid-stride loop
// over the source rows): streaming operators (scan-select filters,
// projections, hash-join probes, Skinner index lookups) are fused into the
// loop body, and the sink (materialisation, aggregate, group table, join
// table) is written into the same kernel.  Kernels are compiled for sm_100a by
// NVRTC with -fmad=false so per-row float arithmetic rounds exactly like the
// reference's mulsd/addsd (khir/asm/asm_backend.cc:1834-1864).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <functional>
#include <limits>
#include <list>
#include <map>
#include <random>
#include <set>
#include <sstream>

#include "engine.h"
#include "join_prior.h"
#include "operators.h"

namespace kdb {
namespace {

using namespace plan;

// ---------------------------------------------------------------------------
// Source building
// ---------------------------------------------------------------------------

std::string CType(TypeId t) {
  switch (t) {
    case TypeId::SMALLINT: return "int16_t";
    case TypeId::INT:
    case TypeId::DATE:
    case TypeId::ENUM: return "int32_t";
    case TypeId::BIGINT: return "int64_t";
    case TypeId::REAL: return "double";
    case TypeId::BOOLEAN: return "bool";
    case TypeId::TEXT: return "kdb_str";
  }
  return "void";
}

// Storage type of a materialised column.
std::string StoreType(TypeId t) {
  switch (t) {
    case TypeId::BOOLEAN: return "int8_t";
    case TypeId::TEXT: return "kdb_str";
    default: return CType(t);
  }
}

size_t StoreWidth(TypeId t) {
  switch (t) {
    case TypeId::BOOLEAN: return 1;
    case TypeId::SMALLINT: return 2;
    case TypeId::INT:
    case TypeId::DATE:
    case TypeId::ENUM: return 4;
    case TypeId::BIGINT:
    case TypeId::REAL: return 8;
    case TypeId::TEXT: return 16;
  }
  return 8;
}

bool IsIntLike(TypeId t) {
  return t == TypeId::SMALLINT || t == TypeId::INT || t == TypeId::BIGINT || t == TypeId::DATE ||
         t == TypeId::ENUM || t == TypeId::BOOLEAN;
}

std::string F64Lit(double d) {
  if (std::isnan(d)) return "__longlong_as_double(0x7ff8000000000000LL)";
  if (std::isinf(d)) return d > 0 ? "__longlong_as_double(0x7ff0000000000000LL)"
                                  : "__longlong_as_double((long long)0xfff0000000000000ULL)";
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%.17g", d);
  std::string s = buf;
  if (s.find_first_of(".eE") == std::string::npos) s += ".0";
  return s;
}

std::string I64Lit(int64_t v) {
  if (v == INT64_MIN) return "(-9223372036854775807LL - 1)";
  return "(" + std::to_string(v) + "LL)";
}

struct CVal {
  Type type;
  std::string v;  // C expression / variable holding the value
  std::string n;  // C bool expression: is NULL ("false" when never NULL)
};

struct Scope {
  std::vector<std::vector<CVal>> child;
  std::vector<CVal> virt;
  const std::vector<CVal>& Child(int i) const {
    if (i < 0 || i >= static_cast<int>(child.size()) || child[i].empty())
      throw Error(-1, "column reference to unbound child " + std::to_string(i));
    return child[i];
  }
};

class KernelSource {
 public:
  std::ostringstream globals;
  std::ostringstream pre;
  std::ostringstream body;
  std::vector<uint64_t> args;
  int indent = 1;
  int tmp = 0;
  int lits = 0;

  std::string Fresh(const char* p) { return std::string(p) + std::to_string(tmp++); }

  void L(const std::string& s) { body << std::string(indent * 2, ' ') << s << "\n"; }
  void Open(const std::string& s) {
    L(s + " {");
    indent++;
  }
  void Close() {
    indent--;
    L("}");
  }

  int Arg(uint64_t w) {
    if (args.size() >= 384) throw Error(-5, "pipeline needs more than 384 kernel argument words");
    args.push_back(w);
    return static_cast<int>(args.size()) - 1;
  }
  std::string Word(uint64_t w) { return "a.w[" + std::to_string(Arg(w)) + "]"; }
  // Declares a typed device pointer local in the prologue.
  std::string Ptr(const void* p, const std::string& type, bool is_const = false) {
    std::string name = "p" + std::to_string(tmp++);
    pre << "  " << (is_const ? "const " : "") << type << "* __restrict__ " << name << " = ("
        << (is_const ? "const " : "") << type << "*)a.w[" << Arg(reinterpret_cast<uint64_t>(p))
        << "];\n";
    return name;
  }
  std::string Lit(const std::string& s) {
    std::string name = "kdb_lit" + std::to_string(lits++);
    globals << "__device__ const char " << name << "[" << (s.size() + 1) << "] = {";
    for (unsigned char c : s) globals << static_cast<int>(c) << ",";
    globals << "0};\n";
    return "kdb_mkstr(" + name + ", " + std::to_string(s.size()) + ")";
  }

  std::string Kernel(const std::string& name, int block, int min_blocks = 1) const {
    int words = 16;
    while (words < static_cast<int>(args.size())) words *= 2;
    if (words > 384) words = 384;
    std::ostringstream o;
    o << globals.str() << "\nextern \"C\" __global__ void __launch_bounds__(" << block << ", " << min_blocks
      << ") " << name << "(KArgsN<" << words << "> a) {\n"
      << kGridDependencyWait << pre.str() << body.str() << "}\n";
    return o.str();
  }

  KArgs Args() const {
    KArgs k;
    std::memset(&k, 0, sizeof(k));
    for (size_t i = 0; i < args.size(); i++) k.w[i] = args[i];
    return k;
  }
};

// ---------------------------------------------------------------------------
// Expression emission (mirrors compile/translators/expression_translator.cc
// and compile/proxy/evaluate.cc; NULL rules as in the oracle)
// ---------------------------------------------------------------------------

class ExprGen {
 public:
  ExprGen(Context& ctx, KernelSource& ks) : ctx_(ctx), ks_(ks) {}

  CVal Bind(const Type& t, const std::string& v, const std::string& n) {
    CVal out{t, ks_.Fresh("v"), ks_.Fresh("n")};
    ks_.L(CType(t.id) + " " + out.v + " = " + v + ";");
    if (n == "false" || n == "true") {
      out.n = n;
      ks_.tmp--;
    } else {
      ks_.L("bool " + out.n + " = " + n + ";");
    }
    return out;
  }

  const DevEnum& EnumOf(const Type& t) { return ctx_.Enum(t.enum_id); }

  std::string EnumRank(const Type& t, const std::string& key) {
    auto it = rank_ptr_.find(t.enum_id);
    if (it == rank_ptr_.end())
      it = rank_ptr_.emplace(t.enum_id, ks_.Ptr(EnumOf(t).d_rank, "int32_t", true)).first;
    return it->second + "[" + key + "]";
  }
  std::string EnumString(const Type& t, const std::string& key) {
    auto it = str_ptr_.find(t.enum_id);
    if (it == str_ptr_.end()) {
      const DevEnum& e = EnumOf(t);
      std::string off = ks_.Ptr(e.d_off, "int64_t", true);
      std::string ch = ks_.Ptr(e.d_chars, "char", true);
      it = str_ptr_.emplace(t.enum_id, std::make_pair(off, ch)).first;
    }
    return "kdb_enum_str(" + it->second.first + ", " + it->second.second + ", " + key + ")";
  }

  std::string HashOf(const CVal& c) {
    switch (c.type.id) {
      case TypeId::REAL: return "kdb_mix64(kdb_dbits(" + c.v + "))";
      case TypeId::TEXT: return "kdb_hash_str(" + c.v + ")";
      case TypeId::BOOLEAN: return "kdb_mix64((uint64_t)(" + c.v + " ? 1 : 0))";
      default: return "kdb_mix64((uint64_t)(int64_t)" + c.v + ")";
    }
  }

  // 32-bit join key hash; equal values of any integer width hash alike
  std::string KeyHash32(const CVal& c) {
    switch (c.type.id) {
      case TypeId::REAL: return "kdb_hash64to32(kdb_dbits(" + c.v + "))";
      case TypeId::TEXT: return "(uint32_t)(kdb_hash_str(" + c.v + ") >> 32)";
      case TypeId::BOOLEAN: return "kdb_hash64to32((uint64_t)(" + c.v + " ? 1 : 0))";
      default: return "kdb_hash64to32((uint64_t)(int64_t)" + c.v + ")";
    }
  }

  std::string EqOf(const CVal& a, const CVal& b) {
    switch (a.type.id) {
      case TypeId::TEXT: return "kdb_str_eq(" + a.v + ", " + b.v + ")";
      case TypeId::BOOLEAN: return "(" + a.v + " == " + b.v + ")";
      default: return "(" + a.v + " == " + b.v + ")";
    }
  }

  CVal Emit(const Expr& e, const Scope& s) {
    switch (e.kind) {
      case ExprKind::ColRef: return s.Child(e.child_idx).at(e.column_idx);
      case ExprKind::VirtColRef: return s.virt.at(e.column_idx);
      case ExprKind::Literal: {
        // numeric literals travel as kernel argument words, so queries that
        // differ only in their constants share one compiled pipeline
        std::string v;
        switch (e.type.id) {
          case TypeId::REAL: {
            uint64_t bits;
            std::memcpy(&bits, &e.fval, 8);
            v = "__longlong_as_double((long long)" + ks_.Word(bits) + ")";
            break;
          }
          case TypeId::TEXT: v = ks_.Lit(e.sval); break;
          case TypeId::BOOLEAN: v = "(" + ks_.Word(e.ival ? 1 : 0) + " != 0)"; break;
          case TypeId::BIGINT: v = "(int64_t)" + ks_.Word(static_cast<uint64_t>(e.ival)); break;
          case TypeId::SMALLINT: v = "(int16_t)(int64_t)" + ks_.Word(static_cast<uint64_t>(e.ival)); break;
          default: v = "(int32_t)(int64_t)" + ks_.Word(static_cast<uint64_t>(e.ival)); break;
        }
        return CVal{e.type, v, e.lit_null ? "true" : "false"};
      }
      case ExprKind::Unary: {
        CVal c = Emit(e.kid(0), s);
        if (e.uop == UnOp::IS_NULL) return Bind(e.type, c.n, "false");
        return Bind(e.type, "!" + c.v, c.n);
      }
      case ExprKind::Case: {
        CVal c = Emit(e.kid(0), s);
        CVal t = Emit(e.kid(1), s);
        CVal f = Emit(e.kid(2), s);
        std::string take = "(!(" + c.n + ") && " + c.v + ")";
        return Bind(e.type, take + " ? " + t.v + " : " + f.v, take + " ? " + t.n + " : " + f.n);
      }
      case ExprKind::IntToFloat: {
        CVal c = Emit(e.kid(0), s);
        return Bind(e.type, "(" + c.n + ") ? 0.0 : (double)" + c.v, "false");
      }
      case ExprKind::Extract: {
        CVal c = Emit(e.kid(0), s);
        return Bind(e.type, "kdb_extract_year(" + c.v + ")", c.n);
      }
      case ExprKind::EnumIn: {
        CVal c = Emit(e.kid(0), s);
        std::string cond = "false";
        for (int32_t x : e.in_values) cond += " || " + c.v + " == " + std::to_string(x);
        return Bind(e.type, "!(" + c.n + ") && (" + cond + ")", "false");
      }
      case ExprKind::Regexp: {
        // expression_translator.cc:277-297: NULL -> false; an ENUM matches
        // through its string
        CVal c = Emit(e.kid(0), s);
        const auto tok = LikeTokens(e.regex);
        if (tok.size() > 63) throw Error(-5, "LIKE pattern of more than 63 tokens");
        uint64_t tr[256] = {0}, star = 0;
        for (size_t i = 0; i < tok.size(); i++) {
          if (tok[i].first == 0) tr[tok[i].second] |= 1ULL << i;
          else if (tok[i].first == 1) {
            for (int b = 0; b < 256; b++)
              if (b != '\n') tr[b] |= 1ULL << i;
          } else {
            star |= 1ULL << i;
          }
        }
        const std::string name = "kdb_like_tr" + std::to_string(ks_.lits++);
        ks_.globals << "__device__ const unsigned long long " << name << "[256] = {";
        for (int b = 0; b < 256; b++) ks_.globals << tr[b] << "ULL,";
        ks_.globals << "};\n";
        const std::string str = c.type.id == TypeId::ENUM ? EnumString(c.type, c.v) : c.v;
        return Bind(e.type, "!(" + c.n + ") && kdb_like(" + str + ", " + name + ", " + std::to_string(star) + "ULL, " +
                                std::to_string(tok.size()) + ")",
                    "false");
      }
      case ExprKind::Agg: throw Error(-1, "Aggregate expression can't be derived");
      case ExprKind::Binary: break;
    }
    CVal l = Emit(e.kid(0), s);
    CVal r = Emit(e.kid(1), s);
    if (e.bop == BinOp::AND) {
      // expression_translator.cc:74-91
      return Bind(e.type, "(" + l.n + ") ? false : (" + l.v + " ? " + r.v + " : false)",
                  "(" + l.n + ") ? true : (" + l.v + " ? (" + r.n + ") : false)");
    }
    if (e.bop == BinOp::OR) {
      // expression_translator.cc:93-108
      return Bind(e.type, "(" + l.n + ") ? " + r.v + " : (" + l.v + " ? true : " + r.v + ")",
                  "(" + l.n + ") ? (" + r.n + ") : (" + l.v + " ? false : (" + r.n + "))");
    }
    std::string n = "(" + l.n + ") || (" + r.n + ")";
    if (l.n == "false" && r.n == "false") n = "false";
    const Type& lt = l.type;
    auto cmp = [&](const std::string& a, const std::string& b) -> std::string {
      switch (e.bop) {
        case BinOp::EQ: return "(" + a + " == " + b + ")";
        case BinOp::NEQ: return "(" + a + " != " + b + ")";
        case BinOp::LT: return "(" + a + " < " + b + ")";
        case BinOp::LEQ: return "(" + a + " <= " + b + ")";
        case BinOp::GT: return "(" + a + " > " + b + ")";
        case BinOp::GEQ: return "(" + a + " >= " + b + ")";
        default: throw Error(-1, "bad comparison");
      }
    };
    switch (lt.id) {
      case TypeId::BOOLEAN: return Bind(e.type, cmp(l.v, r.v), n);
      case TypeId::SMALLINT:
      case TypeId::INT:
      case TypeId::BIGINT:
      case TypeId::DATE: {
        if (e.bop == BinOp::ADD || e.bop == BinOp::SUB || e.bop == BinOp::MUL) {
          // arithmetic in the column type, two's-complement wrap (evaluate.cc:84-113)
          std::string ut = lt.id == TypeId::SMALLINT ? "uint16_t"
                           : lt.id == TypeId::BIGINT ? "uint64_t"
                                                     : "uint32_t";
          const char* op = e.bop == BinOp::ADD ? " + " : e.bop == BinOp::SUB ? " - " : " * ";
          std::string expr = "(" + CType(lt.id) + ")(" + ut + ")((" + ut + ")" + l.v + op + "(" +
                             ut + ")" + r.v + ")";
          if (lt.id == TypeId::SMALLINT)
            expr = "(int16_t)(uint16_t)((uint32_t)(uint16_t)" + l.v + op + "(uint32_t)(uint16_t)" +
                   r.v + ")";
          return Bind(e.type, expr, n);
        }
        if (e.bop == BinOp::DIV) throw Error(-1, "Invalid arguments to div");
        return Bind(e.type, cmp(l.v, r.v), n);
      }
      case TypeId::REAL: {
        switch (e.bop) {
          case BinOp::ADD: return Bind(e.type, "__dadd_rn(" + l.v + ", " + r.v + ")", n);
          case BinOp::SUB: return Bind(e.type, "__dsub_rn(" + l.v + ", " + r.v + ")", n);
          case BinOp::MUL: return Bind(e.type, "__dmul_rn(" + l.v + ", " + r.v + ")", n);
          case BinOp::DIV: return Bind(e.type, "__ddiv_rn(" + l.v + ", " + r.v + ")", n);
          default: return Bind(e.type, cmp(l.v, r.v), n);
        }
      }
      case TypeId::TEXT: {
        switch (e.bop) {
          case BinOp::STARTS_WITH:
            return Bind(e.type, "kdb_str_starts_with(" + l.v + ", " + r.v + ")", n);
          case BinOp::ENDS_WITH:
            return Bind(e.type, "kdb_str_ends_with(" + l.v + ", " + r.v + ")", n);
          case BinOp::CONTAINS:
            return Bind(e.type, "kdb_str_contains(" + l.v + ", " + r.v + ")", n);
          case BinOp::EQ: return Bind(e.type, "kdb_str_eq(" + l.v + ", " + r.v + ")", n);
          case BinOp::NEQ: return Bind(e.type, "!kdb_str_eq(" + l.v + ", " + r.v + ")", n);
          default: return Bind(e.type, cmp("kdb_str_cmp(" + l.v + ", " + r.v + ")", "0"), n);
        }
      }
      case TypeId::ENUM: {
        // evaluate.cc:186-268: EQ/NEQ on keys, ordering and string ops on the
        // key's string (ranks when both sides are the same enum)
        if (e.bop == BinOp::EQ || e.bop == BinOp::NEQ) return Bind(e.type, cmp(l.v, r.v), n);
        if (r.type.id == TypeId::ENUM && r.type.enum_id == lt.enum_id &&
            (e.bop == BinOp::LT || e.bop == BinOp::LEQ || e.bop == BinOp::GT || e.bop == BinOp::GEQ))
          return Bind(e.type, cmp(EnumRank(lt, l.v), EnumRank(lt, r.v)), n);
        std::string ls = EnumString(lt, l.v);
        std::string rs = r.type.id == TypeId::ENUM ? EnumString(r.type, r.v) : r.v;
        switch (e.bop) {
          case BinOp::STARTS_WITH: return Bind(e.type, "kdb_str_starts_with(" + ls + ", " + rs + ")", n);
          case BinOp::ENDS_WITH: return Bind(e.type, "kdb_str_ends_with(" + ls + ", " + rs + ")", n);
          case BinOp::CONTAINS: return Bind(e.type, "kdb_str_contains(" + ls + ", " + rs + ")", n);
          default: return Bind(e.type, cmp("kdb_str_cmp(" + ls + ", " + rs + ")", "0"), n);
        }
      }
    }
    throw Error(-1, "unhandled binary expression");
  }

 private:
  Context& ctx_;
  KernelSource& ks_;
  std::map<int32_t, std::string> rank_ptr_;
  std::map<int32_t, std::pair<std::string, std::string>> str_ptr_;
};

// ---------------------------------------------------------------------------
// Aggregate state layout (compile/proxy/aggregator.cc semantics)
// ---------------------------------------------------------------------------

enum class StateKind { SumF64, SumI64, AvgF64, Count, MinMaxKey, MinMaxText };

// How two partial states of one accumulator word combine.
enum class WordKind { AddF64, AddI64, MinU64, MaxU64 };

struct DenseWord {
  WordKind kind;
  std::string init;   // C initialiser
  std::string ctype;  // register type
};

// C expression combining two uint64 bit patterns of a word of kind `k`.
std::string CombineBits(WordKind k, const std::string& a, const std::string& b) {
  switch (k) {
    case WordKind::AddF64:
      return "(uint64_t)__double_as_longlong(__dadd_rn(__longlong_as_double((long long)" + a +
             "), __longlong_as_double((long long)" + b + ")))";
    case WordKind::AddI64: return "(" + a + " + " + b + ")";
    case WordKind::MinU64: return "(" + b + " < " + a + " ? " + b + " : " + a + ")";
    case WordKind::MaxU64: return "(" + b + " > " + a + " ? " + b + " : " + a + ")";
  }
  return a;
}

// Emits a block-wide reduction of per-CTA partials part[k * G + b] (word-
// major, so a warp's loads of one word are contiguous) over `G` blocks into
// shared tot[k]: one warp per word, lanes striding over the blocks in a
// fixed order, then a shuffle tree (deterministic).
void EmitPartialReduce(KernelSource& ks, const std::string& part, const std::string& G, int nw,
                       const std::vector<WordKind>& kinds) {
  // the words' kinds as a table (one compact loop for every word, instead
  // of a loop body per word: the latter overflowed the instruction cache)
  const std::string kt = "kdb_kinds" + std::to_string(ks.lits++);
  ks.globals << "__device__ const unsigned char " << kt << "[" << nw << "] = {";
  for (int w = 0; w < nw; w++) ks.globals << static_cast<int>(kinds[w]) << ",";
  ks.globals << "};\n";
  ks.L("__shared__ uint64_t tot[" + std::to_string(nw) + "];");
  ks.Open("");
  ks.L("const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;");
  ks.Open("for (int k = warp; k < " + std::to_string(nw) + "; k += blockDim.x / 32)");
  ks.L("const int kind = " + kt + "[k];");
  ks.L("uint64_t x = kdb_word_identity(kind);");
  ks.Open("for (int64_t b0 = lane; b0 < (int64_t)" + G + "; b0 += 256)");
  ks.L("uint64_t v[8];");
  ks.L("_Pragma(\"unroll\") for (int u = 0; u < 8; u++) { const int64_t b = b0 + 32 * u; v[u] = b < (int64_t)" + G +
       " ? " + part + "[(int64_t)k * (int64_t)" + G + " + b] : 0ULL; }");
  ks.L("_Pragma(\"unroll\") for (int u = 0; u < 8; u++) if (b0 + 32 * u < (int64_t)" + G +
       ") x = kdb_word_combine(kind, x, v[u]);");
  ks.Close();
  ks.L("for (int o = 16; o > 0; o >>= 1) x = kdb_word_combine(kind, x, __shfl_down_sync(0xffffffffu, x, o));");
  ks.L("if (lane == 0) tot[k] = x;");
  ks.Close();
  ks.Close();
  ks.L("__syncthreads();");
}



struct AggPlan {
  const Expr* agg;
  StateKind kind;
  bool is_min = false;
  bool child_nullable = false;
  int count_flag = -1;  // bit in the first-row flags (COUNT(col) quirk)
};

AggPlan PlanAgg(const Expr& a, int& flags) {
  AggPlan p{&a, StateKind::Count};
  const Type& ct = a.kid(0).type;
  p.child_nullable = a.kid(0).nullable;
  switch (a.agg) {
    case AggType::SUM: p.kind = ct.id == TypeId::REAL ? StateKind::SumF64 : StateKind::SumI64; break;
    case AggType::AVG: p.kind = StateKind::AvgF64; break;
    case AggType::COUNT:
      p.kind = StateKind::Count;
      // COUNT initialises to 1 on the group's first row even when that row's
      // value is NULL (aggregator.cc:285-287)
      if (p.child_nullable) {
        if (flags >= 8) throw Error(-5, "more than 8 nullable COUNT(col) aggregates");
        p.count_flag = flags++;
      }
      break;
    case AggType::MIN:
    case AggType::MAX:
      p.is_min = a.agg == AggType::MIN;
      if (ct.id == TypeId::BOOLEAN) throw Error(-1, "cannot compute min of non-numeric col");
      p.kind = ct.id == TypeId::TEXT ? StateKind::MinMaxText : StateKind::MinMaxKey;
      break;
  }
  return p;
}

// Order-preserving 64-bit key of a MIN/MAX input value.
std::string OKey(ExprGen& eg, const CVal& c) {
  switch (c.type.id) {
    case TypeId::REAL: return "kdb_dord(" + c.v + ")";
    case TypeId::ENUM:
      return "(((uint64_t)(uint32_t)" + eg.EnumRank(c.type, c.v) + " << 32) | (uint64_t)(uint32_t)" +
             c.v + ")";
    default: return "((uint64_t)(int64_t)" + c.v + " ^ 0x8000000000000000ULL)";
  }
}

// Value from an order-preserving key.
std::string OKeyInv(const Type& t, const std::string& k) {
  switch (t.id) {
    case TypeId::REAL: return "kdb_dord_inv(" + k + ")";
    case TypeId::ENUM: return "(int32_t)(uint32_t)(" + k + " & 0xffffffffULL)";
    default: return "(" + CType(t.id) + ")(int64_t)(" + k + " ^ 0x8000000000000000ULL)";
  }
}

// ---------------------------------------------------------------------------
// Executor
// ---------------------------------------------------------------------------

using Consume = std::function<void(const std::vector<CVal>&, const std::string& pos)>;

constexpr int64_t kSmallOrder = 4096;

struct KeyLayout {
  bool packed = true;
  std::vector<int> offset, width;
  std::vector<bool> nullable;
  std::vector<uint64_t> card;
  int bits = 0;
  uint64_t domain = 1;  // number of distinct keys when all keys are enum/bool
  bool small_domain = true;
};

struct JoinTable {
  MatBuffer build;
  uint64_t* slots = nullptr;
  uint64_t mask = 0;
  // one-bit-per-position filter of the build keys' hashes (about 8 bits per
  // build row, 2^bloom_log2 bits): a probe whose bit is clear skips the
  // table; the filter is small enough to stay in L1 / L2 where the table
  // does not
  uint32_t* bloom = nullptr;
  int bloom_log2 = 0;
  // one 32-bit-or-narrower build key: the slot holds the key itself in its
  // high word (instead of the hash), so a probe compares it there and never
  // loads the build row's key; `key_col` is that column
  bool key_in_slot = false;
  int key_col = -1;
  // key-in-slot tables: device word set by the build when two non-NULL
  // build rows share the key (the join key is then not unique)
  uint64_t* dup = nullptr;
  // grouped form (Skinner indexes): rows sorted by key hash (`srow`, with
  // their hashes `sh`), and `slots` holding one entry per distinct hash
  // (hash << 32 | first sorted index + 1) with the group's length in `lens`
  uint32_t* lens = nullptr;
  uint64_t* sh = nullptr;
  uint32_t* srow = nullptr;
  int64_t n = 0;
};

// An ungrouped aggregate over a Skinner join evaluated inside the episode
// kernel: no result row is materialised.  `state` holds, per aggregate, a
// value word and a count word, then the row count and the first position
// (the layout of the aggregate's per-CTA partials).
struct SkinnerAgg {
  const std::vector<AggPlan>* plans = nullptr;
  uint64_t* state = nullptr;
  int nw = 0;
};

}  // namespace

// One cached Skinner child: its filtered rows and the grouped indexes of the
// join columns, in device memory owned by the entry.  `ready` is recorded on
// the building stream after the last kernel that fills them; a request that
// finds the entry waits on it before its own kernels read the entry.
struct BuildEntry {
  explicit BuildEntry(Context& ctx) : arena(ctx) {
    if (!ctx.dry) KDB_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  }
  ~BuildEntry() {
    if (ready) cudaEventDestroy(ready);
  }
  BuildEntry(const BuildEntry&) = delete;
  BuildEntry& operator=(const BuildEntry&) = delete;
  Arena arena;  // frees the entry's memory when the last holder lets go
  MatBuffer mat;
  std::vector<JoinTable> index;  // per child column (empty where none)
  cudaEvent_t ready = nullptr;
};

// Shared by the slots of one server.  Entries leave the map oldest first
// once the cached bytes pass max_bytes; their memory goes when the last
// query holding them is destroyed, after its own synchronisation, so no
// kernel still reads it.  The server's tables do not change while it runs
// (a documented condition of the serving slots), so entries never go stale.
struct BuildCache {
  explicit BuildCache(size_t max) : max_bytes(max) {}
  std::mutex mu;
  size_t max_bytes;
  size_t bytes = 0;
  std::list<std::string> lru;  // least recently used first
  struct Slot {
    std::shared_ptr<BuildEntry> entry;
    std::list<std::string>::iterator at;
  };
  std::unordered_map<std::string, Slot> map;
  int64_t hits = 0, misses = 0;

  std::shared_ptr<BuildEntry> Find(const std::string& key) {
    std::lock_guard<std::mutex> lock(mu);
    auto it = map.find(key);
    if (it == map.end()) {
      misses++;
      return nullptr;
    }
    hits++;
    lru.splice(lru.end(), lru, it->second.at);
    return it->second.entry;
  }
  // Keeps `e` (or an entry another slot inserted for the same key first,
  // which the caller then uses instead of its own).
  std::shared_ptr<BuildEntry> Insert(const std::string& key, std::shared_ptr<BuildEntry> e) {
    std::lock_guard<std::mutex> lock(mu);
    auto it = map.find(key);
    if (it != map.end()) return e;  // both built it; each uses its own
    lru.push_back(key);
    map[key] = Slot{e, std::prev(lru.end())};
    bytes += e->arena.bytes();
    while (bytes > max_bytes && lru.size() > 1) {
      auto victim = map.find(lru.front());
      bytes -= victim->second.entry->arena.bytes();
      map.erase(victim);
      lru.pop_front();
    }
    return e;
  }
};

std::shared_ptr<BuildCache> MakeBuildCache(size_t max_bytes) { return std::make_shared<BuildCache>(max_bytes); }

void BuildCacheStats(BuildCache& c, int64_t* hits, int64_t* misses, int64_t* bytes, int64_t* entries) {
  std::lock_guard<std::mutex> lock(c.mu);
  *hits = c.hits;
  *misses = c.misses;
  *bytes = static_cast<int64_t>(c.bytes);
  *entries = static_cast<int64_t>(c.map.size());
}

namespace {

class Executor {
 public:
  Executor(Context& ctx, Arena& arena) : ctx_(ctx), arena_(arena) {}

  HostResult Run(const Operator& root);
  MatBuffer MaterializeRoot(const Operator& root) { return Materialize(root); }
  // the root's rows from the device into a host result
  HostResult Download(const MatBuffer& m, const Operator& root, bool check_error = false);
  int64_t bytes_scanned = 0;

 private:
  Context& ctx_;
  Arena& arena_;
  std::map<const Operator*, MatBuffer> mats_;
  std::map<const Operator*, JoinTable> joins_;
  // build-cache entries this query reads: kept until the executor (whose
  // query has synchronised by then) is destroyed
  std::vector<std::shared_ptr<BuildEntry>> held_;
  std::string ChildSig(const Operator& child, const std::set<int>& index_cols) const;

  // --- helpers -----------------------------------------------------------
  // Upper bound (or, for joins, an estimate) of the rows a stream produces.
  int64_t RowBound(const Operator& o) {
    switch (o.kind) {
      case OpKind::SCAN:
      case OpKind::SCAN_SELECT: {
        auto it = ctx_.tables.find(o.relation);
        return it == ctx_.tables.end() ? 0 : std::max<int64_t>(it->second.rows, 0);
      }
      case OpKind::SELECT: return RowBound(o.child());
      case OpKind::HASH_JOIN:
        return 2 * std::max<int64_t>(RowBound(o.child(1)), joins_.count(&o) ? joins_.at(&o).build.rows : 0);
      case OpKind::CROSS_PRODUCT:
        return std::max<int64_t>(1, RowBound(o.child(1)) * (mats_.count(&o.child(0)) ? mats_.at(&o.child(0)).rows : 1));
      default: {
        auto it = mats_.find(&o);
        return it == mats_.end() ? 1024 : it->second.rows;
      }
    }
  }
  static bool Streamable(const Operator& op) {
    return op.kind == OpKind::SCAN || op.kind == OpKind::SCAN_SELECT || op.kind == OpKind::SELECT ||
           op.kind == OpKind::HASH_JOIN || op.kind == OpKind::CROSS_PRODUCT;
  }

  // Reads a device counter.  In a compile-only context it reports 2 rows so
  // the downstream pipelines (sorts, outputs) are still generated.
  int64_t ReadU64(const uint64_t* d) {
    uint64_t h = 0;
    ctx_.D2H(&h, d, sizeof(h));
    if (ctx_.dry) h = 2;
    return static_cast<int64_t>(h);
  }

  MatBuffer AllocMat(const std::vector<SchemaCol>& schema, int64_t cap) {
    MatBuffer m;
    m.cap = std::max<int64_t>(cap, 1);
    for (const auto& c : schema) {
      MatCol mc;
      mc.type = c.expr->type;
      mc.nullable = c.expr->nullable;
      mc.data = arena_.Alloc(StoreWidth(mc.type.id) * m.cap);
      if (mc.nullable) mc.nulls = arena_.AllocT<int8_t>(m.cap);
      m.cols.push_back(mc);
    }
    m.pos = arena_.AllocT<uint64_t>(m.cap);
    return m;
  }

  // Prepare everything a stream over `op` needs: materialise non-streamable
  // inputs, build hash-join tables and Skinner indexes.
  void Prepare(const Operator& op) {
    switch (op.kind) {
      case OpKind::SCAN:
      case OpKind::SCAN_SELECT: return;
      case OpKind::SELECT:
        PrepareInput(op.child());
        return;
      case OpKind::HASH_JOIN:
        BuildJoin(op);
        PrepareInput(op.child(1));
        return;
      case OpKind::CROSS_PRODUCT:
        // the left child is buffered (cross_product_translator.cc:19-40)
        if (!mats_.count(&op.child(0))) mats_[&op.child(0)] = Materialize(op.child(0));
        PrepareCrossLeft(op);
        PrepareInput(op.child(1));
        return;
      default: return;
    }
  }
  void PrepareInput(const Operator& op) {
    if (Streamable(op)) Prepare(op);
    else if (!mats_.count(&op)) mats_[&op] = Materialize(op);
  }

  // --- stream emission ---------------------------------------------------
  void EmitStream(KernelSource& ks, ExprGen& eg, const Operator& op, const Consume& consume,
                  int64_t& src_rows);
  void EmitMatScan(KernelSource& ks, const MatBuffer& m, const uint32_t* indirection,
                   const Consume& consume, int64_t& src_rows);
  // The output values of a SCAN / SCAN_SELECT at base-table row `row` (a
  // row the scan's filters already passed), its columns read there.
  std::vector<CVal> EmitScanRowAt(KernelSource& ks, ExprGen& eg, const Operator& op, const std::string& row);
  MatBuffer EmitOrderedMaterialize(KernelSource& ks, ExprGen& eg, const Operator& op, const uint32_t* order,
                                   const MatBuffer& src, int64_t& src_rows);
  std::vector<CVal> LoadMatRow(KernelSource& ks, ExprGen& eg, const MatBuffer& m,
                               const std::string& row, std::vector<std::string>* col_ptrs_cache);

  // --- pipelines ---------------------------------------------------------
  MatBuffer Materialize(const Operator& op);
  MatBuffer MaterializeStream(const Operator& op, const uint32_t* order = nullptr,
                              const MatBuffer* ordered_src = nullptr);
  // `on_count(rows)` runs between the counting and the writing pass; `on_row`
  // emits extra per-row work into the writing pass (values, row index).
  using RowHook = std::function<void(KernelSource&, ExprGen&, const std::vector<CVal>&, const std::string&)>;
  MatBuffer MaterializeCounted(const Operator& op, const std::function<void(int64_t)>& on_count = nullptr,
                               const RowHook& on_row = nullptr);
  // left rows of a CROSS_PRODUCT in the left child's stream order (null:
  // the buffer already is in that order)
  std::map<const Operator*, uint32_t*> cross_order_;
  void PrepareCrossLeft(const Operator& op);
  static bool StreamHasJoin(const Operator& op) {
    if (op.kind == OpKind::HASH_JOIN || op.kind == OpKind::CROSS_PRODUCT) return true;
    return op.kind == OpKind::SELECT && Streamable(op.child()) && StreamHasJoin(op.child());
  }
  MatBuffer RunAggregate(const Operator& op);
  // any_order: the consumer (an ORDER BY) orders the rows itself, so the
  // groups may come out in any order with their first-appearance key as the
  // stream position (pos_is_index false) instead of being sorted by it
  MatBuffer RunGroupBy(const Operator& op, bool any_order = false, const Operator* order_by = nullptr);
  MatBuffer RunOrderBy(const Operator& op);
  MatBuffer RunSkinner(const Operator& op, const SkinnerAgg* agg = nullptr);
  MatBuffer SmallOrderBy(const Operator& op, MatBuffer& m);
  MatBuffer LargeOrderBy(const Operator& op, MatBuffer& m);
  // Returns true when it also counted ties into *ties (range sort taken).
  bool SortItems(uint64_t* items, int64_t n, unsigned long long* ties = nullptr, uint32_t tie_mask = 0,
                 const unsigned long long* key_range = nullptr);
  // KDB_ORDER_FUSED_RANGE: the kernel that makes the items also reduces
  // their key range for the range-bucket sort (one 64-bit atomic min and max
  // per warp).  Measured slower on the Q3 ORDER BY (step 217-219 against
  // 214-216 us): thousands of warps' atomics queue on the two words, where
  // the sort's own 32-CTA pass issues 64.
  bool KeyRangeWanted() const {
    return ctx_.OptStr("KDB_ORDER_FUSED_RANGE") && !ctx_.OptStr("KDB_ORDER_MERGE") && !ctx_.OptStr("KDB_ORDER_SAMPLE");
  }
  // set while materialising an ORDER BY's output: the sorted items, whose
  // high words hold the rows (read by EmitMatScan instead of an index array)
  const uint64_t* order_items_ = nullptr;
  MatBuffer RunGroupByDense(const Operator& op, const std::vector<AggPlan>& plans, const KeyLayout& kl,
                            const Operator* order_by = nullptr);
  // the ORDER BY was done by its GROUP BY child (dense path)
  bool group_sorted_ = false;
  bool BuildRowGroups(const Operator& op, std::vector<int>* key_cols);
  MatBuffer RunGroupByBuildRows(const Operator& op, const std::vector<AggPlan>& plans,
                                const std::vector<int>& key_cols, bool any_order);
  void BuildJoin(const Operator& op);
  JoinTable BuildIndex(const MatBuffer& m, const std::vector<int>& key_cols);
  // The table of BuildIndex for `rows` build rows of buffer m's layout
  // (allocated and cleared), and the insert of one row into it.
  JoinTable PrepareJoinTable(const MatBuffer& m, int64_t rows, const std::vector<int>& key_cols);
  void EmitJoinInsert(KernelSource& ks, ExprGen& eg, const JoinTable& jt, const std::vector<CVal>& vals,
                      const std::vector<int>& key_cols, const std::string& row);
  JoinTable BuildGroupedIndex(const MatBuffer& m, int key_col);
  std::string probe_br_;  // inside an on_match callback: the matched build row's index
  // set while emitting a probe whose kernel staged the join filter in
  // shared memory: the array's name
  std::string smem_bloom_;
  // set while emitting a join's probe side: its scan takes one row per
  // thread per iteration (the probe's dependent table accesses, not the
  // column loads, bound such a pipeline, and the 4-row vector's registers
  // cost occupancy)
  bool probe_side_scan_ = false;
  // set with probe_side_scan_: the scan prefetches only these columns (the
  // probe keys and the filters); the others load where they are used
  const std::set<int>* prefetch_only_ = nullptr;
  // set while materialising a join's build side (rows in any order)
  bool build_side_mat_ = false;
  // TMA-staged scan: set by a consumer before emitting its scan (rows per
  // tile, stages); the scan reports the dynamic shared memory it needs in
  // tma_smem_ (0 when it fell back to register loads).
  int tma_tile_ = 0, tma_stages_ = 0;
  size_t tma_smem_ = 0;
  // Probe-ahead (KDB_PROBE_AHEAD=1, or =word for the filter word alone): a
  // join whose probe side is a plain scan of its key column has that scan
  // load the key two rows ahead and, one row ahead, the row's join-filter
  // word and first table slot, so the probe of a row starts with its
  // dependent table reads done.  Measured on the Q3 shape it is slower (69
  // vs 52 us for the probe + group-by kernel: the speculative loads of the
  // rows the filter rejects crowd the load queues), so it is off by
  // default.  ahead_jt_/ahead_out_col_ go from the join to its scan; the
  // ahead_* names come back from the scan to EmitProbe.
  const JoinTable* ahead_jt_ = nullptr;
  int ahead_out_col_ = -1;
  const JoinTable* ahead_probe_jt_ = nullptr;
  bool ahead_slot_on_ = true;
  std::string ahead_key_var_, ahead_word_, ahead_slot_;
  void SetProbeAhead(const Operator& join, const JoinTable& jt) {
    ahead_jt_ = nullptr;
    ahead_out_col_ = -1;
    const char* mode = ctx_.OptStr("KDB_PROBE_AHEAD");
    if ((!mode && !ctx_.OptStr("KDB_PROBE_VEC")) || ctx_.OptStr("KDB_LAZY_PROBE_COLUMNS") ||
        join.right_keys.size() != 1)
      return;
    const Expr& k = *join.right_keys[0];
    const OpKind ck = join.child(1).kind;
    if (k.kind != ExprKind::ColRef || k.child_idx != 1 || (ck != OpKind::SCAN && ck != OpKind::SCAN_SELECT)) return;
    ahead_jt_ = &jt;
    ahead_out_col_ = k.column_idx;
    ahead_slot_on_ = !mode || std::string(mode) != "word";
  }
  void EmitProbe(KernelSource& ks, ExprGen& eg, const JoinTable& jt,
                 const std::vector<int>& build_key_cols, const std::vector<CVal>& probe_keys,
                 const std::function<void(const std::vector<CVal>&, const std::string&)>& on_match);
  std::string JoinHash(ExprGen& eg, const std::vector<CVal>& keys);

  // Kernel symbol for a pipeline role: "group by" -> kdb_group_by.
  static std::string KernelName(const char* what) {
    std::string n = "kdb_";
    for (const char* c = what; *c; c++) n += (*c == ' ') ? '_' : *c;
    return n;
  }

  void LaunchPipeline(KernelSource& ks, int64_t src_rows, const char* what, int block = 256, int min_blocks = 1) {
    std::string name = KernelName(what);
    std::string src = ks.Kernel(name, block, min_blocks);
    CUfunction f = ctx_.Kernel(src, name);
    int grid = ctx_.GridFor(std::max<int64_t>(src_rows, 1), block);
    ctx_.Launch(f, grid, block, ks.Args(), 0, what);
  }
};

std::string Executor::JoinHash(ExprGen& eg, const std::vector<CVal>& keys) {
  std::string h;
  for (const auto& k : keys) h = h.empty() ? eg.KeyHash32(k) : "kdb_hash_combine32(" + h + ", " + eg.KeyHash32(k) + ")";
  return h;
}

std::vector<CVal> Executor::LoadMatRow(KernelSource& ks, ExprGen& eg, const MatBuffer& m,
                                       const std::string& row, std::vector<std::string>* cache) {
  std::vector<CVal> vals;
  for (size_t c = 0; c < m.cols.size(); c++) {
    const MatCol& mc = m.cols[c];
    std::string dp, np;
    if (cache && (*cache).size() > 2 * c && !(*cache)[2 * c].empty()) {
      dp = (*cache)[2 * c];
      np = (*cache)[2 * c + 1];
    } else {
      dp = ks.Ptr(mc.data, StoreType(mc.type.id), true);
      np = mc.nullable ? ks.Ptr(mc.nulls, "int8_t", true) : "";
      if (cache) {
        if (cache->size() < 2 * m.cols.size()) cache->resize(2 * m.cols.size());
        (*cache)[2 * c] = dp;
        (*cache)[2 * c + 1] = np;
      }
    }
    std::string v = dp + "[" + row + "]";
    if (mc.type.id == TypeId::BOOLEAN) v = "(" + v + " != 0)";
    vals.push_back(eg.Bind(mc.type, v, mc.nullable ? "(" + np + "[" + row + "] != 0)" : "false"));
  }
  return vals;
}

void Executor::EmitMatScan(KernelSource& ks, const MatBuffer& m, const uint32_t* indirection,
                           const Consume& consume, int64_t& src_rows) {
  ExprGen eg(ctx_, ks);
  src_rows = m.rows;
  std::string n = ks.Word(static_cast<uint64_t>(m.rows));
  // sorted items instead of an index array: row = the item's high word
  const uint64_t* items = indirection ? order_items_ : nullptr;
  order_items_ = nullptr;
  std::string ind = items ? ks.Ptr(items, "uint64_t", true)
                          : indirection ? ks.Ptr(indirection, "uint32_t", true) : "";
  std::string pos = ks.Ptr(m.pos, "uint64_t", true);
  ks.Open("for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < (int64_t)" + n +
          "; r += (int64_t)gridDim.x * blockDim.x)");
  std::string row = "r";
  if (items) {
    ks.L("int64_t rr = (int64_t)(uint32_t)(" + ind + "[2 * r + 1] >> 32);");
    row = "rr";
  } else if (indirection) {
    ks.L("int64_t rr = (int64_t)" + ind + "[r];");
    row = "rr";
  }
  auto vals = LoadMatRow(ks, eg, m, row, nullptr);
  // ordered sources (ORDER BY output) emit in sorted order: position = r
  consume(vals, indirection ? "(uint64_t)r" : pos + "[" + row + "]");
  ks.Close();
}

std::vector<CVal> Executor::EmitScanRowAt(KernelSource& ks, ExprGen& eg, const Operator& op,
                                          const std::string& row) {
  if (op.kind != OpKind::SCAN && op.kind != OpKind::SCAN_SELECT) throw Error(-1, "row access of a non-scan");
  std::vector<CVal> scan;
  for (const auto& sc : op.scan_columns) {
    const DevColumn& c = ctx_.Column(op.relation, sc.name);
    std::string v;
    if (c.type.id == TypeId::TEXT) {
      v = "kdb_text_at(" + ks.Ptr(c.toff, "int64_t", true) + ", " + ks.Ptr(c.tchars, "char", true) + ", " + row + ")";
    } else {
      v = ks.Ptr(c.data, StoreType(c.type.id), true) + "[" + row + "]";
      if (c.type.id == TypeId::BOOLEAN) v = "(" + v + " != 0)";
    }
    const std::string nul = c.nulls ? "(" + ks.Ptr(c.nulls, "int8_t", true) + "[" + row + "] != 0)" : "false";
    // bound where used: columns the consumer never reads are never loaded
    scan.push_back(CVal{c.type, "(" + v + ")", nul});
  }
  Scope s;
  if (op.kind == OpKind::SCAN) s.child.push_back(scan);
  else s.virt = scan;
  std::vector<CVal> out;
  for (const auto& c : op.output) out.push_back(eg.Emit(*c.expr, s));
  return out;
}

void Executor::EmitStream(KernelSource& ks, ExprGen& eg, const Operator& op, const Consume& consume,
                          int64_t& src_rows) {
  switch (op.kind) {
    case OpKind::SCAN:
    case OpKind::SCAN_SELECT: {
      // scan_translator.cc:140-168 / scan_select_translator.cc:92-156
      const DevTable* t = nullptr;
      auto it = ctx_.tables.find(op.relation);
      if (it == ctx_.tables.end()) throw Error(-1, "unknown relation " + op.relation);
      t = &it->second;
      int64_t rows = std::max<int64_t>(t->rows, 0);
      src_rows = rows;
      std::string n = ks.Word(static_cast<uint64_t>(rows));
      // columns used by the filters load first, the rest only for rows that
      // pass (scan_select_translator.cc:115-134 loads lazily the same way)
      std::set<int> filter_cols;
      std::function<void(const Expr&)> collect = [&](const Expr& e) {
        if (e.kind == ExprKind::VirtColRef || e.kind == ExprKind::ColRef) filter_cols.insert(e.column_idx);
        for (const auto& k : e.kids) collect(*k);
      };
      for (const auto& f : op.filters) collect(*f);
      std::vector<const DevColumn*> cols;
      std::vector<std::string> dp, np, tp;
      for (const auto& sc : op.scan_columns) {
        const DevColumn& c = ctx_.Column(op.relation, sc.name);
        if (c.type.id != sc.type.id) throw Error(-1, "column " + sc.name + " type mismatch");
        cols.push_back(&c);
        if (c.type.id == TypeId::TEXT) {
          dp.push_back(ks.Ptr(c.toff, "int64_t", true));
          tp.push_back(ks.Ptr(c.tchars, "char", true));
        } else {
          dp.push_back(ks.Ptr(c.data, StoreType(c.type.id), true));
          tp.push_back("");
        }
        np.push_back(c.nulls ? ks.Ptr(c.nulls, "int8_t", true) : "");
        bytes_scanned += static_cast<int64_t>(c.bytes);
      }
      bool any_text = false;
      for (const DevColumn* c : cols) any_text |= c->type.id == TypeId::TEXT;
      const bool probe_side = probe_side_scan_;
      probe_side_scan_ = false;
      const std::set<int>* prefetch_only = probe_side ? prefetch_only_ : nullptr;
      prefetch_only_ = nullptr;
      // probe-ahead: the scan column that is the join's probe key
      const JoinTable* ajt = ahead_jt_;
      ahead_jt_ = nullptr;
      int ak = -1;
      if (probe_side && ajt && ahead_out_col_ >= 0 && ahead_out_col_ < static_cast<int>(op.output.size())) {
        const Expr& oe = *op.output[ahead_out_col_].expr;
        const bool direct = (oe.kind == ExprKind::ColRef && oe.child_idx == 0) || oe.kind == ExprKind::VirtColRef;
        if (direct && oe.column_idx >= 0 && oe.column_idx < static_cast<int>(cols.size())) {
          const TypeId t = cols[oe.column_idx]->type.id;
          if (t == TypeId::INT || t == TypeId::DATE || t == TypeId::ENUM || t == TypeId::SMALLINT ||
              t == TypeId::BIGINT)
            ak = oe.column_idx;
        }
      }
      // KDB_PROBE_VEC: the probe side too takes 4-row vectors, and each
      // vector's join-filter words, then (for the rows that pass) first
      // table slots, load together before its rows are probed
      const bool vec_probe = probe_side && ak >= 0 && ctx_.OptStr("KDB_PROBE_VEC") != nullptr;
      const bool vec = !any_text && (!probe_side || vec_probe) && !ctx_.OptStr("KDB_NO_VECTOR_SCAN");
      std::vector<CVal> scan(cols.size());
      std::function<void(size_t)> load;
      // TMA staging needs every column (and null array) 16-byte aligned
      const int TT = tma_tile_, TS = tma_stages_;
      tma_tile_ = tma_stages_ = 0;
      tma_smem_ = 0;
      bool tma = vec && TT > 0 && TS > 0 && TT % 16 == 0;
      for (size_t k = 0; k < cols.size() && tma; k++) {
        tma = reinterpret_cast<uintptr_t>(cols[k]->data) % 16 == 0 &&
              (!cols[k]->nulls || reinterpret_cast<uintptr_t>(cols[k]->nulls) % 16 == 0);
      }
      if (tma) {
        // Persistent CTAs walk tiles of TT rows (tile t = blockIdx.x + i *
        // gridDim.x).  Thread 0 keeps TS tiles in flight: per tile one
        // 1-D bulk copy per column into that stage's shared memory, all
        // completing on the stage's mbarrier; the threads read 4 rows at a
        // time from shared memory.  The last tile's bytes past its last whole
        // 16-byte unit are loaded by the threads themselves.
        std::vector<size_t> off(cols.size(), 0), noff(cols.size(), 0);
        std::vector<int> width(cols.size());
        size_t sb = 0;
        auto place = [&](size_t bytes) {
          const size_t o = sb;
          sb += (bytes + 127) / 128 * 128;
          return o;
        };
        for (size_t k = 0; k < cols.size(); k++) {
          width[k] = static_cast<int>(StoreWidth(cols[k]->type.id));
          off[k] = place(static_cast<size_t>(TT) * width[k]);
          if (!np[k].empty()) noff[k] = place(static_cast<size_t>(TT));
        }
        const size_t stage_bytes = sb;
        tma_smem_ = stage_bytes * TS;
        if (tma_smem_ > (size_t(160) << 10)) {
          // too wide a row for the stages beside the consumer's own shared
          // memory: register loads instead
          tma = false;
          tma_smem_ = 0;
        }
      }
      if (tma) {
        std::vector<size_t> off(cols.size(), 0), noff(cols.size(), 0);
        std::vector<int> width(cols.size());
        size_t sb = 0;
        auto place = [&](size_t bytes) {
          const size_t o = sb;
          sb += (bytes + 127) / 128 * 128;
          return o;
        };
        for (size_t k = 0; k < cols.size(); k++) {
          width[k] = static_cast<int>(StoreWidth(cols[k]->type.id));
          off[k] = place(static_cast<size_t>(TT) * width[k]);
          if (!np[k].empty()) noff[k] = place(static_cast<size_t>(TT));
        }
        const size_t stage_bytes = sb;
        const std::string ERR = ks.Ptr(ctx_.d_err, "int");
        const std::string sT = std::to_string(TT), sS = std::to_string(TS), sB = std::to_string(stage_bytes);
        ks.L("extern __shared__ __align__(128) unsigned char kdb_dsm[];");
        ks.L("__shared__ __align__(8) uint64_t kdb_tbar[" + sS + "];");
        ks.L("const int64_t nrows = (int64_t)" + n + ";");
        ks.L("const int64_t kdb_nt = (nrows + " + sT + " - 1) / " + sT + ";");
        ks.L("auto kdb_issue = [&](int64_t t, int st) {");
        ks.indent++;
        ks.L("const int64_t tb = t * " + sT + ";");
        ks.L("const int64_t tn = nrows - tb < " + sT + " ? nrows - tb : " + sT + ";");
        ks.L("unsigned char* sb = kdb_dsm + (size_t)st * " + sB + ";");
        std::vector<std::string> bn(cols.size()), nbn(cols.size());
        std::string tot = "0u";
        for (size_t k = 0; k < cols.size(); k++) {
          bn[k] = ks.Fresh("tb");
          ks.L("const uint32_t " + bn[k] + " = (uint32_t)((tn * " + std::to_string(width[k]) + ") & ~15LL);");
          tot += " + " + bn[k];
          if (!np[k].empty()) {
            nbn[k] = ks.Fresh("tnb");
            ks.L("const uint32_t " + nbn[k] + " = (uint32_t)(tn & ~15LL);");
            tot += " + " + nbn[k];
          }
        }
        ks.L("kdb_bar_expect(&kdb_tbar[st], " + tot + ");");
        for (size_t k = 0; k < cols.size(); k++) {
          ks.L("if (" + bn[k] + ") kdb_bulk_copy(sb + " + std::to_string(off[k]) + ", (const unsigned char*)" + dp[k] +
               " + tb * " + std::to_string(width[k]) + ", " + bn[k] + ", &kdb_tbar[st]);");
          if (!np[k].empty())
            ks.L("if (" + nbn[k] + ") kdb_bulk_copy(sb + " + std::to_string(noff[k]) + ", (const unsigned char*)" +
                 np[k] + " + tb, " + nbn[k] + ", &kdb_tbar[st]);");
        }
        ks.indent--;
        ks.L("};");
        ks.L("if (threadIdx.x == 0) { for (int s = 0; s < " + sS +
             "; s++) kdb_bar_init(&kdb_tbar[s]); kdb_fence_proxy_async(); }");
        ks.L("__syncthreads();");
        ks.L("if (threadIdx.x == 0) for (int s = 0; s < " + sS +
             "; s++) { const int64_t t = blockIdx.x + (int64_t)s * gridDim.x; if (t < kdb_nt) kdb_issue(t, s); }");
        ks.Open("for (int64_t kdb_it = 0;; kdb_it++)");
        ks.L("const int64_t kdb_t = blockIdx.x + kdb_it * (int64_t)gridDim.x;");
        ks.L("if (kdb_t >= kdb_nt) break;");
        ks.L("const int kdb_st = (int)(kdb_it % " + sS + ");");
        ks.Open("if (!kdb_bar_wait_all(&kdb_tbar[kdb_st], (uint32_t)((kdb_it / " + sS + ") & 1), " + ERR + "))");
        // give up: wait (bounded) for every copy this block still has in
        // flight into its shared memory, then leave
        ks.Open("if (threadIdx.x == 0)");
        ks.L("for (int64_t j = kdb_it; j < kdb_it + " + sS + "; j++) if (blockIdx.x + j * (int64_t)gridDim.x < kdb_nt) "
             "kdb_bar_wait(&kdb_tbar[j % " + sS + "], (uint32_t)((j / " + sS + ") & 1));");
        ks.Close();
        ks.L("break;");
        ks.Close();
        ks.L("const int64_t kdb_tb = kdb_t * " + sT + ";");
        ks.L("const int kdb_tn = (int)(nrows - kdb_tb < " + sT + " ? nrows - kdb_tb : " + sT + ");");
        ks.L("unsigned char* kdb_sb = kdb_dsm + (size_t)kdb_st * " + sB + ";");
        ks.Open("if (kdb_tn < " + sT + ")");
        for (size_t k = 0; k < cols.size(); k++) {
          const std::string st = StoreType(cols[k]->type.id), w = std::to_string(width[k]);
          ks.L("for (int i = (int)(((kdb_tn * " + w + ") & ~15) / " + w + ") + threadIdx.x; i < kdb_tn; i += blockDim.x) ((" +
               st + "*)(kdb_sb + " + std::to_string(off[k]) + "))[i] = " + dp[k] + "[kdb_tb + i];");
          if (!np[k].empty())
            ks.L("for (int i = (kdb_tn & ~15) + threadIdx.x; i < kdb_tn; i += blockDim.x) ((int8_t*)(kdb_sb + " +
                 std::to_string(noff[k]) + "))[i] = " + np[k] + "[kdb_tb + i];");
        }
        // these generic writes precede later bulk copies into the stage
        ks.L("kdb_fence_proxy_async();");
        ks.L("__syncthreads();");
        ks.Close();
        std::vector<std::string> arr(cols.size()), narr(cols.size());
        ks.Open("for (int q = threadIdx.x; q * 4 < kdb_tn; q += blockDim.x)");
        ks.L("const int64_t base = kdb_tb + (int64_t)q * 4;");
        for (size_t k = 0; k < cols.size(); k++) {
          const std::string st = StoreType(cols[k]->type.id);
          arr[k] = ks.Fresh("L");
          ks.L(st + " " + arr[k] + "[4];");
          ks.L("kdb_lds4((const " + st + "*)(kdb_sb + " + std::to_string(off[k]) + "), q * 4, " + arr[k] + ");");
          if (!np[k].empty()) {
            narr[k] = ks.Fresh("N");
            ks.L("int8_t " + narr[k] + "[4];");
            ks.L("kdb_lds4((const int8_t*)(kdb_sb + " + std::to_string(noff[k]) + "), q * 4, " + narr[k] + ");");
          }
        }
        load = [&, arr, narr](size_t k) {
          const DevColumn& c = *cols[k];
          std::string v = c.type.id == TypeId::BOOLEAN ? "(" + arr[k] + "[u] != 0)" : arr[k] + "[u]";
          scan[k] = eg.Bind(c.type, v, narr[k].empty() ? "false" : "(" + narr[k] + "[u] != 0)");
        };
        ks.L("#pragma unroll");
        ks.Open("for (int u = 0; u < 4; u++)");
        ks.L("const int64_t r = base + u;");
        ks.Open("if (r < nrows)");
      } else if (vec) {
        // 4 consecutive rows per thread, every column loaded with vector
        // loads up front (all loads of an iteration in flight together)
        // With prefetch (default), the next iteration's vectors are loaded
        // before this iteration's rows are processed, so a warp keeps two
        // iterations of loads in flight.
        // KDB_SCAN_BATCH=B (B > 1, not on a probe side): B vectors per
        // thread and iteration (vectors q, q + stride, ..., so each load
        // instruction stays coalesced), all loaded before any is processed,
        // instead of the one-vector prefetch
        const char* batch_opt = ctx_.OptStr("KDB_SCAN_BATCH");
        const int VB = (batch_opt && !probe_side) ? std::max(1, std::min(8, std::atoi(batch_opt))) : 1;
        const std::string R = std::to_string(4 * VB);
        const bool prefetch = VB == 1 && !ctx_.OptStr("KDB_NO_SCAN_PREFETCH");
        ks.L("const int64_t nrows = (int64_t)" + n + ";");
        ks.L("const int64_t qstride = (int64_t)gridDim.x * blockDim.x;");
        std::vector<std::string> arr(cols.size()), narr(cols.size()), parr(cols.size()), pnarr(cols.size());
        // loads of the 4 rows of vector `qv` into the arrays `dst` / `ndst`
        // from element `off` on
        auto fetch = [&](const std::string& qv, const std::vector<std::string>& dst,
                         const std::vector<std::string>& ndst, int off = 0) {
          ks.Open("");
          ks.L("const int64_t fb = (" + qv + ") * 4;");
          ks.L("const bool ffull = fb + 4 <= nrows;");
          const std::string o = off ? " + " + std::to_string(off) : "";
          for (size_t k = 0; k < cols.size(); k++) {
            const DevColumn& c = *cols[k];
            std::string st = StoreType(c.type.id);
            ks.L("if (ffull) kdb_ld4(" + dp[k] + ", fb, " + dst[k] + o + "); else for (int u = 0; u < 4; u++) (" +
                 dst[k] + o + ")[u] = fb + u < nrows ? " + dp[k] + "[fb + u] : (" + st + ")0;");
            if (!np[k].empty())
              ks.L("if (ffull) kdb_ld4(" + np[k] + ", fb, " + ndst[k] + o + "); else for (int u = 0; u < 4; u++) (" +
                   ndst[k] + o + ")[u] = fb + u < nrows ? " + np[k] + "[fb + u] : (int8_t)0;");
          }
          ks.Close();
        };
        if (prefetch) {
          for (size_t k = 0; k < cols.size(); k++) {
            parr[k] = ks.Fresh("P");
            ks.L(StoreType(cols[k]->type.id) + " " + parr[k] + "[4];");
            if (!np[k].empty()) {
              pnarr[k] = ks.Fresh("PN");
              ks.L("int8_t " + pnarr[k] + "[4];");
            }
          }
          ks.L("const int64_t q0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;");
          ks.Open("if (q0 * 4 < nrows)");
          fetch("q0", parr, pnarr);
          ks.Close();
        }
        ks.Open("for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q * 4 < nrows; q += qstride * " +
                std::to_string(VB) + ")");
        ks.L("const int64_t base = q * 4;");
        for (size_t k = 0; k < cols.size(); k++) {
          arr[k] = ks.Fresh("L");
          ks.L(StoreType(cols[k]->type.id) + " " + arr[k] + "[" + R + "];");
          if (!np[k].empty()) {
            narr[k] = ks.Fresh("N");
            ks.L("int8_t " + narr[k] + "[" + R + "];");
          }
        }
        if (prefetch) {
          for (size_t k = 0; k < cols.size(); k++) {
            ks.L("for (int u = 0; u < 4; u++) " + arr[k] + "[u] = " + parr[k] + "[u];");
            if (!np[k].empty()) ks.L("for (int u = 0; u < 4; u++) " + narr[k] + "[u] = " + pnarr[k] + "[u];");
          }
          ks.Open("if ((q + qstride) * 4 < nrows)");
          fetch("q + qstride", parr, pnarr);
          ks.Close();
        } else {
          for (int b = 0; b < VB; b++) fetch("q + qstride * " + std::to_string(b), arr, narr, 4 * b);
        }
        if (vec_probe) {
          // the vector's 4 join-filter words, then the first table slots of
          // the rows that pass, all in flight together (indexes masked:
          // always in bounds; rows past the end carry key 0)
          const std::string vs = ks.Ptr(ajt->slots, "uint64_t", true), vm = ks.Word(ajt->mask);
          const std::string vb = ajt->bloom ? ks.Ptr(ajt->bloom, "uint32_t", true) : "";
          const std::string lg = std::to_string(ajt->bloom_log2);
          const std::string h = JoinHash(eg, {CVal{cols[ak]->type, arr[ak] + "[u]", "false"}});
          ks.L("uint32_t VW[4];");
          ks.L("uint64_t VS[4];");
          ks.L("#pragma unroll");
          ks.L("for (int u = 0; u < 4; u++) VW[u] = " +
               (vb.empty() ? std::string("~0u") : "__ldg(&" + vb + "[kdb_bloom_bit(" + h + ", " + lg + ") >> 5])") + ";");
          ks.L("#pragma unroll");
          ks.Open("for (int u = 0; u < 4; u++)");
          ks.L("const uint32_t vh = " + h + ";");
          if (vb.empty())
            ks.L("VS[u] = " + vs + "[vh & (uint32_t)" + vm + "];");
          else
            ks.L("VS[u] = ((VW[u] >> (kdb_bloom_bit(vh, " + lg + ") & 31)) & 1u) ? " + vs + "[vh & (uint32_t)" + vm +
                 "] : 0ULL;");
          ks.Close();
          ahead_probe_jt_ = ajt;
          ahead_word_ = "VW[u]";
          ahead_slot_ = "VS[u]";
          ahead_slot_on_ = true;
        }
        load = [&, arr, narr, ak](size_t k) {
          const DevColumn& c = *cols[k];
          std::string v = c.type.id == TypeId::BOOLEAN ? "(" + arr[k] + "[u] != 0)" : arr[k] + "[u]";
          scan[k] = eg.Bind(c.type, v, narr[k].empty() ? "false" : "(" + narr[k] + "[u] != 0)");
          if (static_cast<int>(k) == ak) ahead_key_var_ = scan[k].v;
        };
        ks.L("#pragma unroll");
        ks.Open("for (int u = 0; u < " + R + "; u++)");
        ks.L(VB == 1 ? "const int64_t r = base + u;" : "const int64_t r = base + (int64_t)(u >> 2) * qstride * 4 + (u & 3);");
        ks.Open("if (r < nrows)");
      } else {
        // On a join's probe side (one row per thread and iteration) the next
        // iteration's values of every fixed-width column are loaded before
        // this iteration's row is probed, so their HBM latency overlaps the
        // probe's dependent L2 accesses (KDB_NO_PROBE_PREFETCH: off).
        const bool pf = probe_side && !ctx_.OptStr("KDB_NO_PROBE_PREFETCH") && !ctx_.OptStr("KDB_LAZY_PROBE_COLUMNS");
        std::vector<std::string> nxt(cols.size()), nnx(cols.size());
        if (!pf || !ctx_.OptStr("KDB_PROBE_AHEAD")) ak = -1;
        std::string a_key2, a_word, a_slot, a_slots, a_bloom;
        auto ahead_loads = [&](const std::string& key) {
          // the join-filter word and the first table slot of the row whose
          // probe key is `key` (indexes masked: always in bounds)
          const std::string h = ks.Fresh("AH");
          ks.L("const uint32_t " + h + " = " + JoinHash(eg, {CVal{cols[ak]->type, key, "false"}}) + ";");
          if (ajt->bloom)
            ks.L(a_word + " = __ldg(&" + a_bloom + "[kdb_bloom_bit(" + h + ", " + std::to_string(ajt->bloom_log2) +
                 ") >> 5]);");
          if (ahead_slot_on_) ks.L(a_slot + " = " + a_slots + "[" + h + " & (uint32_t)" + ks.Word(ajt->mask) + "];");
        };
        if (pf) {
          ks.L("const int64_t kdb_pstride = (int64_t)gridDim.x * blockDim.x;");
          ks.L("const int64_t kdb_p0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;");
          for (size_t k = 0; k < cols.size(); k++) {
            if (cols[k]->type.id == TypeId::TEXT) continue;
            if (prefetch_only && !prefetch_only->count(static_cast<int>(k))) continue;
            const std::string st = StoreType(cols[k]->type.id);
            nxt[k] = ks.Fresh("X");
            ks.L(st + " " + nxt[k] + " = kdb_p0 < (int64_t)" + n + " ? " + dp[k] + "[kdb_p0] : (" + st + ")0;");
            if (!np[k].empty()) {
              nnx[k] = ks.Fresh("XN");
              ks.L("int8_t " + nnx[k] + " = kdb_p0 < (int64_t)" + n + " ? " + np[k] + "[kdb_p0] : (int8_t)0;");
            }
          }
          if (ak >= 0) {
            const std::string st = StoreType(cols[ak]->type.id);
            a_key2 = ks.Fresh("XA");
            ks.L(st + " " + a_key2 + " = kdb_p0 + kdb_pstride < (int64_t)" + n + " ? " + dp[ak] +
                 "[kdb_p0 + kdb_pstride] : (" + st + ")0;");
            a_slots = ks.Ptr(ajt->slots, "uint64_t", true);
            if (ajt->bloom) a_bloom = ks.Ptr(ajt->bloom, "uint32_t", true);
            a_word = ks.Fresh("AW");
            a_slot = ks.Fresh("AS");
            ks.L("uint32_t " + a_word + " = 0;");
            ks.L("uint64_t " + a_slot + " = 0;");
            ks.Open("if (kdb_p0 < (int64_t)" + n + ")");
            ahead_loads(nxt[ak]);
            ks.Close();
          }
        }
        ks.Open("for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < (int64_t)" + n +
                "; r += (int64_t)gridDim.x * blockDim.x)");
        std::vector<std::string> cur(cols.size()), ncur(cols.size());
        if (pf) {
          for (size_t k = 0; k < cols.size(); k++) {
            if (nxt[k].empty()) continue;
            const std::string st = StoreType(cols[k]->type.id);
            cur[k] = ks.Fresh("C");
            ks.L("const " + st + " " + cur[k] + " = " + nxt[k] + ";");
            if (!nnx[k].empty()) {
              ncur[k] = ks.Fresh("CN");
              ks.L("const int8_t " + ncur[k] + " = " + nnx[k] + ";");
            }
          }
          std::string cword, cslot;
          if (ak >= 0) {
            cword = ks.Fresh("CW");
            cslot = ks.Fresh("CS");
            ks.L("const uint32_t " + cword + " = " + a_word + ";");
            ks.L("const uint64_t " + cslot + " = " + a_slot + ";");
          }
          ks.Open("if (r + kdb_pstride < (int64_t)" + n + ")");
          for (size_t k = 0; k < cols.size(); k++) {
            if (nxt[k].empty()) continue;
            if (static_cast<int>(k) == ak) ks.L(nxt[k] + " = " + a_key2 + ";");
            else ks.L(nxt[k] + " = " + dp[k] + "[r + kdb_pstride];");
            if (!nnx[k].empty()) ks.L(nnx[k] + " = " + np[k] + "[r + kdb_pstride];");
          }
          if (ak >= 0) {
            ahead_loads(nxt[ak]);
            ks.L("if (r + 2 * kdb_pstride < (int64_t)" + n + ") " + a_key2 + " = " + dp[ak] + "[r + 2 * kdb_pstride];");
          }
          ks.Close();
          if (ak >= 0) {
            ahead_probe_jt_ = ajt;
            ahead_word_ = cword;
            ahead_slot_ = cslot;
          }
        }
        // With KDB_LAZY_PROBE_COLUMNS the probe side of a join reads its
        // columns where the consumer uses them (non-key columns only inside
        // the match branch).  Measured on the Q3 shape it is slower (61 vs
        // 55 us for the probe + group-by kernel): the loads then wait behind
        // the probe's dependent accesses instead of overlapping them, which
        // costs more than the sectors saved, so all columns load up front.
        const bool lazy = probe_side && ctx_.OptStr("KDB_LAZY_PROBE_COLUMNS");
        load = [&, lazy, cur, ncur, ak](size_t k) {
          const DevColumn& c = *cols[k];
          std::string v;
          const std::string raw = cur[k].empty() ? dp[k] + "[r]" : cur[k];
          if (c.type.id == TypeId::TEXT) v = "kdb_text_at(" + dp[k] + ", " + tp[k] + ", r)";
          else if (c.type.id == TypeId::BOOLEAN) v = "(" + raw + " != 0)";
          else v = raw;
          const std::string nul = np[k].empty() ? "false"
                                  : ncur[k].empty() ? "(" + np[k] + "[r] != 0)" : "(" + ncur[k] + " != 0)";
          if (lazy || (prefetch_only && !prefetch_only->count(static_cast<int>(k))))
            scan[k] = CVal{c.type, "(" + v + ")", nul};
          else scan[k] = eg.Bind(c.type, v, nul);
          if (static_cast<int>(k) == ak) ahead_key_var_ = scan[k].v;
        };
      }
      auto close_loop = [&]() {
        if (vec) {
          ks.Close();
          ks.Close();
        }
        ks.Close();
        if (tma) {
          // the stage is free once every thread has read it: refill it with
          // the tile TS iterations ahead
          ks.L("__syncthreads();");
          ks.L("if (threadIdx.x == 0) { const int64_t kdb_nx = kdb_t + (int64_t)" + std::to_string(TS) +
               " * gridDim.x; if (kdb_nx < kdb_nt) { kdb_fence_proxy_async(); kdb_issue(kdb_nx, kdb_st); } }");
          ks.Close();
        }
      };
      Scope s;
      if (op.kind == OpKind::SCAN) {
        for (size_t k = 0; k < cols.size(); k++) load(k);
        s.child.push_back(scan);
        std::vector<CVal> out;
        for (const auto& c : op.output) out.push_back(eg.Emit(*c.expr, s));
        consume(out, "(uint64_t)r");
        close_loop();
        return;
      }
      for (int k : filter_cols)
        if (k < static_cast<int>(cols.size())) load(k);
      int opened = 0;
      for (const auto& f : op.filters) {
        s.virt = scan;
        CVal v = eg.Emit(*f, s);
        ks.Open("if (!(" + v.n + ") && " + v.v + ")");
        opened++;
      }
      for (size_t k = 0; k < cols.size(); k++)
        if (!filter_cols.count(static_cast<int>(k))) load(k);
      s.virt = scan;
      std::vector<CVal> out;
      for (const auto& c : op.output) out.push_back(eg.Emit(*c.expr, s));
      consume(out, "(uint64_t)r");
      for (int i = 0; i < opened; i++) ks.Close();
      close_loop();
      return;
    }
    case OpKind::SELECT: {
      // select_translator.cc:19-37
      auto body = [&](const std::vector<CVal>& in, const std::string& pos) {
        Scope s;
        s.child.push_back(in);
        CVal v = eg.Emit(*op.filters[0], s);
        ks.Open("if (!(" + v.n + ") && " + v.v + ")");
        std::vector<CVal> out;
        for (const auto& c : op.output) out.push_back(eg.Emit(*c.expr, s));
        consume(out, pos);
        ks.Close();
      };
      if (Streamable(op.child())) EmitStream(ks, eg, op.child(), body, src_rows);
      else EmitMatScan(ks, mats_.at(&op.child()), nullptr, body, src_rows);
      return;
    }
    case OpKind::HASH_JOIN: {
      // probe side: hash_join_translator.cc:106-138
      const JoinTable& jt = joins_.at(&op);
      std::vector<int> bkeys;
      for (const auto& k : op.left_keys) bkeys.push_back(k->column_idx);
      auto body = [&](const std::vector<CVal>& right, const std::string& pos) {
        Scope s;
        s.child.resize(2);
        s.child[1] = right;
        std::vector<CVal> pk;
        for (const auto& k : op.right_keys) pk.push_back(eg.Emit(*k, s));
        EmitProbe(ks, eg, jt, bkeys, pk, [&](const std::vector<CVal>& left, const std::string& bpos) {
          Scope s2;
          s2.child.push_back(left);
          s2.child.push_back(right);
          std::vector<CVal> out;
          for (const auto& c : op.output) out.push_back(eg.Emit(*c.expr, s2));
          consume(out, "((" + pos + ") << 32) | ((" + bpos + ") & 0xffffffffULL)");
        });
      };
      probe_side_scan_ = !ctx_.OptStr("KDB_VECTOR_PROBE_SCAN");
      if (probe_side_scan_) SetProbeAhead(op, jt);
      if (Streamable(op.child(1))) EmitStream(ks, eg, op.child(1), body, src_rows);
      else EmitMatScan(ks, mats_.at(&op.child(1)), nullptr, body, src_rows);
      probe_side_scan_ = false;
      ahead_jt_ = nullptr;
      ahead_probe_jt_ = nullptr;
      return;
    }
    case OpKind::CROSS_PRODUCT: {
      // cross_product_translator.cc:43-74: every right row meets the
      // buffered left rows in their stream order; the pair's position is
      // (right position, left stream rank)
      const MatBuffer& lm = mats_.at(&op.child(0));
      const uint32_t* lorder = cross_order_.count(&op) ? cross_order_.at(&op) : nullptr;
      const std::string NL = "(int64_t)" + ks.Word(static_cast<uint64_t>(lm.rows));
      const std::string LO = lorder ? ks.Ptr(lorder, "uint32_t", true) : "";
      auto body = [&](const std::vector<CVal>& right, const std::string& pos) {
        const std::string li = ks.Fresh("li"), lr = ks.Fresh("lr");
        ks.Open("for (int64_t " + li + " = 0; " + li + " < " + NL + "; " + li + "++)");
        ks.L("const int64_t " + lr + " = " + (lorder ? "(int64_t)" + LO + "[" + li + "]" : li) + ";");
        std::vector<CVal> left = LoadMatRow(ks, eg, lm, lr, nullptr);
        Scope s2;
        s2.child.push_back(left);
        s2.child.push_back(right);
        std::vector<CVal> out;
        for (const auto& c : op.output) out.push_back(eg.Emit(*c.expr, s2));
        consume(out, "((" + pos + ") << 32) | (uint64_t)" + li);
        ks.Close();
      };
      if (Streamable(op.child(1))) EmitStream(ks, eg, op.child(1), body, src_rows);
      else EmitMatScan(ks, mats_.at(&op.child(1)), nullptr, body, src_rows);
      return;
    }
    default: {
      EmitMatScan(ks, mats_.at(&op), nullptr, consume, src_rows);
      return;
    }
  }
}

void Executor::PrepareCrossLeft(const Operator& op) {
  const MatBuffer& lm = mats_.at(&op.child(0));
  if (lm.rows >= (int64_t(1) << 32)) throw Error(-5, "CrossProduct left side of 2^32 rows or more");
  if (lm.pos_is_index || lm.rows <= 1 || cross_order_.count(&op)) return;
  // buffer rows not in stream order: sort their positions once
  uint64_t* keys = arena_.AllocT<uint64_t>(lm.rows);
  uint32_t* idx = arena_.AllocT<uint32_t>(lm.rows);
  KernelSource ks;
  const std::string K = ks.Ptr(keys, "uint64_t"), I = ks.Ptr(idx, "uint32_t");
  const std::string P = ks.Ptr(lm.pos, "uint64_t", true), N = ks.Word(static_cast<uint64_t>(lm.rows));
  ks.Open("for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)" + N +
          "; i += (int64_t)gridDim.x * blockDim.x)");
  ks.L(K + "[i] = " + P + "[i]; " + I + "[i] = (uint32_t)i;");
  ks.Close();
  LaunchPipeline(ks, lm.rows, "cross order");
  ctx_.RadixSortPairs(keys, idx, lm.rows, arena_, 64);
  cross_order_[&op] = idx;
}

void Executor::EmitProbe(KernelSource& ks, ExprGen& eg, const JoinTable& jt,
                         const std::vector<int>& bkeys, const std::vector<CVal>& pk,
                         const std::function<void(const std::vector<CVal>&, const std::string&)>& on_match) {
  // NULL probe keys never equal a (non-NULL) build key
  std::string nn = "true";
  for (const auto& k : pk) nn += " && !(" + k.n + ")";
  ks.Open("if (" + nn + ")");
  std::string h = ks.Fresh("h");
  ks.L("uint32_t " + h + " = " + JoinHash(eg, pk) + ";");
  std::string slots = ks.Ptr(jt.slots, "uint64_t", true);
  std::string mask = "(uint32_t)" + ks.Word(jt.mask);
  // the probe-side scan loaded this row's filter word and first slot ahead
  const bool ahead = ahead_probe_jt_ == &jt && pk.size() == 1 && pk[0].v == ahead_key_var_;
  if (ahead) ahead_probe_jt_ = nullptr;
  if (jt.bloom) {
    if (ahead)
      ks.Open("if ((" + ahead_word_ + " >> (kdb_bloom_bit(" + h + ", " + std::to_string(jt.bloom_log2) +
              ") & 31)) & 1u)");
    else if (!smem_bloom_.empty())
      ks.Open("if ((" + smem_bloom_ + "[kdb_bloom_bit(" + h + ", " + std::to_string(jt.bloom_log2) + ") >> 5] >> (kdb_bloom_bit(" +
              h + ", " + std::to_string(jt.bloom_log2) + ") & 31)) & 1u)");
    else
      ks.Open("if (kdb_bloom_test(" + ks.Ptr(jt.bloom, "uint32_t", true) + ", " + h + ", " +
              std::to_string(jt.bloom_log2) + "))");
  }
  std::string i = ks.Fresh("i"), k = ks.Fresh("k"), e = ks.Fresh("e");
  ks.L("uint32_t " + i + " = " + h + " & " + mask + ";");
  ks.Open("for (uint32_t " + k + " = 0; " + k + " <= " + mask + "; " + k + "++, " + i + " = (" + i +
          " + 1) & " + mask + ")");
  if (ahead && ahead_slot_on_)
    ks.L("uint64_t " + e + " = " + k + " == 0 ? " + ahead_slot_ + " : " + slots + "[" + i + "];");
  else ks.L("uint64_t " + e + " = " + slots + "[" + i + "];");
  ks.L("if (" + e + " == 0) break;");
  std::string br = ks.Fresh("br");
  std::vector<CVal> left;
  if (jt.key_in_slot && bkeys.size() == 1 && bkeys[0] == jt.key_col && pk[0].type.id != TypeId::REAL &&
      pk[0].type.id != TypeId::TEXT && pk[0].type.id != TypeId::BOOLEAN) {
    // the stored key, sign-extended, against the probe value in 64 bits
    ks.Open("if ((int64_t)(int32_t)(uint32_t)(" + e + " >> 32) == (int64_t)(" + pk[0].v + "))");
    ks.L("int64_t " + br + " = (int64_t)(uint32_t)" + e + " - 1;");
    left = LoadMatRow(ks, eg, jt.build, br, nullptr);
    const MatCol& kc = jt.build.cols.at(jt.key_col);
    left.at(jt.key_col) = eg.Bind(kc.type, "(" + CType(kc.type.id) + ")(" + pk[0].v + ")", "false");
    ks.Open("");
  } else {
    if (jt.key_in_slot) throw Error(-5, "join probe does not match its key-in-slot table");
    ks.Open("if ((uint32_t)(" + e + " >> 32) == " + h + ")");
    ks.L("int64_t " + br + " = (int64_t)(uint32_t)" + e + " - 1;");
    left = LoadMatRow(ks, eg, jt.build, br, nullptr);
    std::string eq = "true";
    for (size_t j = 0; j < bkeys.size(); j++) eq += " && " + eg.EqOf(left.at(bkeys[j]), pk[j]);
    ks.Open("if (" + eq + ")");
  }
  std::string bpos = ks.Ptr(jt.build.pos, "uint64_t", true) + "[" + br + "]";
  probe_br_ = br;
  on_match(left, bpos);
  ks.Close();
  ks.Close();
  ks.Close();
  if (jt.bloom) ks.Close();
  ks.Close();
}

// Join table over materialised rows (runtime::HashTable equivalent,
// runtime/hash_table.cc:13-36): build rows with a NULL key are skipped
// (hash_join_translator.cc:86-101).
JoinTable Executor::PrepareJoinTable(const MatBuffer& m, int64_t rows, const std::vector<int>& key_cols) {
  JoinTable jt;
  jt.build = m;
  uint64_t cap = 1024;
  while (cap < static_cast<uint64_t>(rows) * 2) cap <<= 1;
  if (cap > (uint64_t(1) << 31)) throw Error(-5, "join build side of more than 2^30 rows");
  jt.mask = cap - 1;
  jt.slots = arena_.AllocT<uint64_t>(cap);
  ctx_.Memset(jt.slots, 0, cap * sizeof(uint64_t));
  if (!ctx_.OptStr("KDB_NO_JOIN_FILTER")) {
    jt.bloom_log2 = 14;
    // KDB_SMEM_BLOOM: at most 2^20 bits, so that a probe kernel can hold
    // the filter in shared memory
    const int max_log2 = ctx_.OptStr("KDB_SMEM_BLOOM") ? 20 : 26;
    while (jt.bloom_log2 < max_log2 && (int64_t(1) << jt.bloom_log2) < rows * 8) jt.bloom_log2++;
    const size_t words = (size_t(1) << jt.bloom_log2) / 32;
    jt.bloom = arena_.AllocT<uint32_t>(words);
    ctx_.Memset(jt.bloom, 0, words * sizeof(uint32_t));
  }
  if (key_cols.size() == 1 && !ctx_.OptStr("KDB_NO_KEY_IN_SLOT")) {
    const TypeId t = m.cols.at(key_cols[0]).type.id;
    jt.key_in_slot = t == TypeId::INT || t == TypeId::DATE || t == TypeId::ENUM || t == TypeId::SMALLINT;
    jt.key_col = key_cols[0];
  }
  if (jt.key_in_slot) {
    jt.dup = arena_.AllocT<uint64_t>(1);
    ctx_.Memset(jt.dup, 0, sizeof(uint64_t));
  }
  return jt;
}

void Executor::EmitJoinInsert(KernelSource& ks, ExprGen& eg, const JoinTable& jt, const std::vector<CVal>& vals,
                              const std::vector<int>& key_cols, const std::string& row) {
  std::string slots = ks.Ptr(jt.slots, "uint64_t");
  std::string mask = ks.Word(jt.mask);
  std::vector<CVal> keys;
  std::string nn = "true";
  for (int c : key_cols) {
    keys.push_back(vals.at(c));
    nn += " && !(" + vals.at(c).n + ")";
  }
  // build rows with a NULL key are skipped (hash_join_translator.cc:86-101)
  ks.Open("if (" + nn + ")");
  const std::string h = ks.Fresh("jh");
  ks.L("const uint32_t " + h + " = " + JoinHash(eg, keys) + ";");
  if (jt.key_in_slot)
    ks.L("if (kdb_join_insert_keyed(" + slots + ", " + mask + ", " + h + ", (uint32_t)(int32_t)" + keys[0].v +
         ", (uint32_t)(" + row + "))) atomicOr((unsigned long long*)" + ks.Ptr(jt.dup, "uint64_t") + ", 1ULL);");
  else
    ks.L("kdb_join_insert(" + slots + ", " + mask + ", " + h + ", (uint32_t)(" + row + "));");
  if (jt.bloom)
    ks.L("kdb_bloom_set(" + ks.Ptr(jt.bloom, "uint32_t") + ", " + h + ", " + std::to_string(jt.bloom_log2) + ");");
  ks.Close();
}

JoinTable Executor::BuildIndex(const MatBuffer& m, const std::vector<int>& key_cols) {
  JoinTable jt = PrepareJoinTable(m, m.rows, key_cols);
  if (m.rows == 0) return jt;
  KernelSource ks;
  ExprGen eg(ctx_, ks);
  std::string n = ks.Word(static_cast<uint64_t>(m.rows));
  ks.Open("for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < (int64_t)" + n +
          "; r += (int64_t)gridDim.x * blockDim.x)");
  auto vals = LoadMatRow(ks, eg, m, "r", nullptr);
  EmitJoinInsert(ks, eg, jt, vals, key_cols, "r");
  ks.Close();
  LaunchPipeline(ks, m.rows, "join build");
  return jt;
}

// Index for the Skinner join's lookups (the role of the reference's column
// indexes, runtime/column_index.cc / memory_column_index.cc: key -> rows):
// rows sorted by key hash, and a table of distinct hashes pointing at each
// run.  A lookup costs one probe of the distinct table plus its matches, so
// heavily repeated keys (Zipf) neither form long probe clusters nor slow
// the lookups of other keys.  Rows with a NULL key are left out.
JoinTable Executor::BuildGroupedIndex(const MatBuffer& m, int key_col) {
  JoinTable jt;
  jt.build = m;
  const int64_t n = m.rows;
  jt.n = n;
  uint64_t cap = 1024;
  while (cap < static_cast<uint64_t>(n) * 2) cap <<= 1;
  if (cap > (uint64_t(1) << 31)) throw Error(-5, "join index over more than 2^30 rows");
  jt.mask = cap - 1;
  jt.slots = arena_.AllocT<uint64_t>(cap);
  jt.lens = arena_.AllocT<uint32_t>(cap);
  jt.sh = arena_.AllocT<uint64_t>(std::max<int64_t>(n, 1));
  jt.srow = arena_.AllocT<uint32_t>(std::max<int64_t>(n, 1));
  ctx_.Memset(jt.slots, 0, cap * sizeof(uint64_t));
  ctx_.Memset(jt.lens, 0, cap * sizeof(uint32_t));
  if (n == 0) return jt;
  const uint64_t kNullHash = 1ULL << 32;  // sorts after every real hash
  {
    KernelSource ks;
    ExprGen eg(ctx_, ks);
    std::string N = ks.Word(static_cast<uint64_t>(n));
    std::string SH = ks.Ptr(jt.sh, "uint64_t"), SR = ks.Ptr(jt.srow, "uint32_t");
    ks.Open("for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < (int64_t)" + N +
            "; r += (int64_t)gridDim.x * blockDim.x)");
    auto vals = LoadMatRow(ks, eg, m, "r", nullptr);
    const CVal& key = vals.at(key_col);
    ks.L(SH + "[r] = (" + key.n + ") ? " + std::to_string(kNullHash) + "ULL : (uint64_t)" + JoinHash(eg, {key}) + ";");
    ks.L(SR + "[r] = (uint32_t)r;");
    ks.Close();
    LaunchPipeline(ks, n, "index keys");
  }
  ctx_.RadixSortPairs(jt.sh, jt.srow, n, arena_, 33);
  for (int pass = 0; pass < 2; pass++) {
    // pass 0: the first row of every run claims a slot; pass 1: the last row
    // of every run writes the run's length into that slot
    KernelSource ks;
    std::string N = ks.Word(static_cast<uint64_t>(n));
    std::string SH = ks.Ptr(jt.sh, "uint64_t", true), SL = ks.Ptr(jt.slots, "uint64_t");
    std::string LN = ks.Ptr(jt.lens, "uint32_t"), M = ks.Word(jt.mask);
    ks.Open("for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)" + N +
            "; i += (int64_t)gridDim.x * blockDim.x)");
    ks.L("const uint64_t h = " + SH + "[i];");
    ks.L("if (h >= " + std::to_string(kNullHash) + "ULL) continue;");
    if (pass == 0) {
      ks.L("if (i > 0 && " + SH + "[i - 1] == h) continue;");
      ks.L("kdb_join_insert(" + SL + ", " + M + ", (uint32_t)h, (uint32_t)i);");
    } else {
      ks.L("if (i + 1 < (int64_t)" + N + " && " + SH + "[i + 1] == h) continue;");
      ks.L("uint32_t s = (uint32_t)h & (uint32_t)" + M + ";");
      ks.Open("for (uint32_t k = 0; k <= (uint32_t)" + M + "; k++, s = (s + 1) & (uint32_t)" + M + ")");
      ks.L("const uint64_t e = " + SL + "[s];");
      ks.L("if (e == 0) break;");
      ks.Open("if ((uint32_t)(e >> 32) == (uint32_t)h)");
      ks.L(LN + "[s] = (uint32_t)(i + 1 - ((int64_t)(uint32_t)e - 1));");
      ks.L("break;");
      ks.Close();
      ks.Close();
    }
    ks.Close();
    LaunchPipeline(ks, n, pass == 0 ? "index runs" : "index lengths");
  }
  return jt;
}

void Executor::BuildJoin(const Operator& op) {
  if (joins_.count(&op)) return;
  // a join's build rows need no particular buffer order (their stream
  // positions travel with them): with KDB_BUILD_MAT_ATOMIC the build side
  // is written in one pass with block-level slot claims
  std::vector<int> keys;
  for (const auto& k : op.left_keys) {
    if (k->kind != ExprKind::ColRef) throw Error(-5, "hash join keys must be column references");
    keys.push_back(k->column_idx);
  }
  const Operator& child = op.child(0);
  if (Streamable(child) && !StreamHasJoin(child) && !ctx_.OptStr("KDB_BUILD_MAT_ATOMIC") &&
      !ctx_.OptStr("KDB_MATERIALIZE_ATOMIC") && !ctx_.OptStr("KDB_JOIN_BUILD_PASS")) {
    // The build side's writing pass inserts every row into the join table
    // as it writes it (sized from the counting pass): no separate build
    // kernel re-reads the rows.
    Prepare(child);
    JoinTable jt;
    MatBuffer layout;  // column types only: the table is sized before the rows exist
    for (const auto& c : child.output) {
      MatCol mc;
      mc.type = c.expr->type;
      mc.nullable = c.expr->nullable;
      layout.cols.push_back(mc);
    }
    auto on_count = [&](int64_t rows) { jt = PrepareJoinTable(layout, rows, keys); };
    auto on_row = [&](KernelSource& ks, ExprGen& eg, const std::vector<CVal>& vals, const std::string& row) {
      EmitJoinInsert(ks, eg, jt, vals, keys, row);
    };
    MatBuffer left = MaterializeCounted(child, on_count, on_row);
    jt.build = left;
    joins_[&op] = jt;
    return;
  }
  build_side_mat_ = ctx_.OptStr("KDB_BUILD_MAT_ATOMIC") != nullptr && Streamable(child);
  MatBuffer left = Materialize(child);
  build_side_mat_ = false;
  joins_[&op] = BuildIndex(left, keys);
}


// Materialise a streamable operator's rows (with stream positions), or, when
// `ordered_src` is given, project `op.output` over that buffer read in
// `order`.  Capacity: exact bound for scans; join outputs are counted and the
// pipeline reruns once at the counted size if the first guess was short.
// Projection of `op.output` over `src` read in sorted order (row r of the
// result is src row order[r]), emitted into `ks`; returns the output buffer.
MatBuffer Executor::EmitOrderedMaterialize(KernelSource& ks, ExprGen& eg, const Operator& op, const uint32_t* order,
                                           const MatBuffer& src, int64_t& src_rows) {
  const auto& schema = op.output;
  MatBuffer out = AllocMat(schema, src.rows);
  std::vector<std::string> optr, onull;
  for (const auto& c : out.cols) {
    optr.push_back(ks.Ptr(c.data, StoreType(c.type.id)));
    onull.push_back(c.nullable ? ks.Ptr(c.nulls, "int8_t") : "");
  }
  std::string posp = ks.Ptr(out.pos, "uint64_t");
  auto body = [&](const std::vector<CVal>& in, const std::string& pos) {
    Scope s;
    s.child.push_back(in);
    std::vector<CVal> vals;
    for (const auto& c : schema) vals.push_back(eg.Emit(*c.expr, s));
    ks.Open("");
    ks.L("const uint64_t slot = (uint64_t)r;");
    for (size_t c = 0; c < vals.size(); c++) {
      const CVal& v = vals[c];
      std::string val = v.type.id == TypeId::BOOLEAN ? "(int8_t)(" + v.v + " ? 1 : 0)" : v.v;
      ks.L(optr[c] + "[slot] = " + val + ";");
      if (!onull[c].empty()) ks.L(onull[c] + "[slot] = (" + v.n + ") ? 1 : 0;");
    }
    ks.L(posp + "[slot] = " + pos + ";");
    ks.Close();
  };
  EmitMatScan(ks, src, order, body, src_rows);
  out.rows = src.rows;
  out.pos_is_index = true;
  return out;
}

MatBuffer Executor::MaterializeStream(const Operator& op, const uint32_t* order,
                                      const MatBuffer* ordered_src) {
  if (ordered_src) {
    // every row r is written at index r: the count is known without a
    // read-back (device errors surface at the next synchronisation)
    KernelSource ks;
    ExprGen eg(ctx_, ks);
    int64_t src_rows = 0;
    MatBuffer out = EmitOrderedMaterialize(ks, eg, op, order, *ordered_src, src_rows);
    LaunchPipeline(ks, src_rows, "materialize");
    return out;
  }
  Prepare(op);
  const bool any_order = build_side_mat_;
  build_side_mat_ = false;
  if (!StreamHasJoin(op) && !any_order && !ctx_.OptStr("KDB_MATERIALIZE_ATOMIC")) return MaterializeCounted(op);
  int64_t cap = RowBound(op);
  for (int attempt = 0; attempt < 3; attempt++) {
    const auto mark = ctx_.RecordMark();
    KernelSource ks;
    ExprGen eg(ctx_, ks);
    const auto& schema = op.output;
    MatBuffer out = AllocMat(schema, cap);
    uint64_t* counter = arena_.AllocT<uint64_t>(1);
    ctx_.Memset(counter, 0, sizeof(uint64_t));
    std::vector<std::string> optr, onull;
    for (const auto& c : out.cols) {
      optr.push_back(ks.Ptr(c.data, StoreType(c.type.id)));
      onull.push_back(c.nullable ? ks.Ptr(c.nulls, "int8_t") : "");
    }
    std::string posp = ks.Ptr(out.pos, "uint64_t");
    std::string cnt = ks.Ptr(counter, "uint64_t");
    std::string capw = "(uint64_t)" + ks.Word(static_cast<uint64_t>(out.cap));
    auto sink = [&](const std::vector<CVal>& vals, const std::string& pos) {
      ks.Open("");
      // rows append through the warp-aggregated counter
      ks.L("uint64_t slot = kdb_alloc_slot((unsigned long long*)" + cnt + ");");
      ks.Open("if (slot < " + capw + ")");
      for (size_t c = 0; c < vals.size(); c++) {
        const CVal& v = vals[c];
        std::string val = v.type.id == TypeId::BOOLEAN ? "(int8_t)(" + v.v + " ? 1 : 0)" : v.v;
        ks.L(optr[c] + "[slot] = " + val + ";");
        if (!onull[c].empty()) ks.L(onull[c] + "[slot] = (" + v.n + ") ? 1 : 0;");
      }
      ks.L(posp + "[slot] = " + pos + ";");
      ks.Close();
      ks.Close();
    };
    int64_t src_rows = 0;
    EmitStream(ks, eg, op, sink, src_rows);
    LaunchPipeline(ks, src_rows, "materialize");
    int64_t produced = ReadU64(counter);
    ctx_.CheckDeviceError("materialize");
    if (produced <= out.cap) {
      out.rows = produced;
      return out;
    }
    cap = produced;
    ctx_.RecordTruncate(mark);
  }
  throw Error(-4, "materialisation did not converge");
}

// Join-free streams (scans and filters) materialise in two passes over the
// same grid: the first counts each block's rows, an exclusive scan turns the
// counts into block offsets, and the second writes each block's rows at its
// offset through a shared-memory slot counter.  One global atomic per
// produced warp-row would serialise on the counter's L2 line (tens of
// microseconds for a filtered scan of a few million rows); the count pass
// reads only the filter columns.
MatBuffer Executor::MaterializeCounted(const Operator& op, const std::function<void(int64_t)>& on_count,
                                       const RowHook& on_row) {
  const int block = 256;
  const auto& schema = op.output;
  const std::string shared_init =
      "  __shared__ unsigned kdb_block_rows;\n"
      "  if (threadIdx.x == 0) kdb_block_rows = 0;\n"
      "  __syncthreads();\n";
  int64_t src_rows = 0;
  KernelSource kc;
  ExprGen egc(ctx_, kc);
  kc.pre << shared_init;
  auto count_sink = [&](const std::vector<CVal>&, const std::string&) {
    kc.L("kdb_alloc_block_slot(&kdb_block_rows);");
  };
  EmitStream(kc, egc, op, count_sink, src_rows);
  const int grid = ctx_.GridFor(std::max<int64_t>(src_rows, 1), block);
  uint64_t* offsets = arena_.AllocT<uint64_t>(grid + 1);
  const std::string offp = kc.Ptr(offsets, "uint64_t");
  kc.L("__syncthreads();");
  kc.L("if (threadIdx.x == 0) " + offp + "[blockIdx.x] = kdb_block_rows;");
  LaunchPipeline(kc, src_rows, "materialize count", block);
  ctx_.ScanU64(offsets, grid, "materialize offsets");
  const int64_t produced = ReadU64(offsets + grid);
  ctx_.CheckDeviceError("materialize");
  if (on_count) on_count(produced);

  KernelSource ks;
  ExprGen eg(ctx_, ks);
  MatBuffer out = AllocMat(schema, std::max<int64_t>(produced, 1));
  std::vector<std::string> optr, onull;
  for (const auto& c : out.cols) {
    optr.push_back(ks.Ptr(c.data, StoreType(c.type.id)));
    onull.push_back(c.nullable ? ks.Ptr(c.nulls, "int8_t") : "");
  }
  const std::string posp = ks.Ptr(out.pos, "uint64_t");
  const std::string offr = ks.Ptr(offsets, "uint64_t", true);
  const std::string capw = "(uint64_t)" + ks.Word(static_cast<uint64_t>(out.cap));
  ks.pre << shared_init;
  ks.pre << "  const uint64_t kdb_block_base = " << offr << "[blockIdx.x];\n";
  auto sink = [&](const std::vector<CVal>& vals, const std::string& pos) {
    ks.Open("");
    ks.L("const uint64_t slot = kdb_block_base + kdb_alloc_block_slot(&kdb_block_rows);");
    ks.Open("if (slot < " + capw + ")");
    for (size_t c = 0; c < vals.size(); c++) {
      const CVal& v = vals[c];
      std::string val = v.type.id == TypeId::BOOLEAN ? "(int8_t)(" + v.v + " ? 1 : 0)" : v.v;
      ks.L(optr[c] + "[slot] = " + val + ";");
      if (!onull[c].empty()) ks.L(onull[c] + "[slot] = (" + v.n + ") ? 1 : 0;");
    }
    ks.L(posp + "[slot] = " + pos + ";");
    if (on_row) on_row(ks, eg, vals, "slot");
    ks.Close();
    ks.Close();
  };
  int64_t src_rows2 = 0;
  EmitStream(ks, eg, op, sink, src_rows2);
  LaunchPipeline(ks, src_rows2, "materialize", block);
  out.rows = produced;
  return out;
}

MatBuffer Executor::Materialize(const Operator& op) {
  switch (op.kind) {
    case OpKind::OUTPUT: return Materialize(op.child());
    case OpKind::AGGREGATE: return RunAggregate(op);
    case OpKind::GROUP_BY_AGGREGATE: return RunGroupBy(op);
    case OpKind::ORDER_BY: return RunOrderBy(op);
    case OpKind::SKINNER_JOIN: return RunSkinner(op);
    default: return MaterializeStream(op);
  }
}

// Emits the per-row update of one aggregate at group slot `g` (atomics).
// Whether an aggregate needs its per-group count of non-NULL inputs: COUNT
// and AVG always; SUM, MIN and MAX only to tell an all-NULL group (NULL
// result), which cannot happen when the input is never NULL.
bool NeedsCount(const AggPlan& p, const CVal& c) {
  const bool value_only = p.kind == StateKind::SumF64 || p.kind == StateKind::SumI64 || p.kind == StateKind::MinMaxKey;
  return !(value_only && c.n == "false");
}

void EmitGroupUpdate(KernelSource& ks, ExprGen& eg, const AggPlan& p, const CVal& c,
                     const std::string& sv, const std::string& sc, const std::string& g, bool count = true) {
  ks.Open("if (!(" + c.n + "))");
  switch (p.kind) {
    case StateKind::SumF64: ks.L("atomicAdd((double*)&" + sv + "[" + g + "], " + c.v + ");"); break;
    case StateKind::AvgF64: ks.L("atomicAdd((double*)&" + sv + "[" + g + "], (double)" + c.v + ");"); break;
    case StateKind::SumI64:
      ks.L("atomicAdd((unsigned long long*)&" + sv + "[" + g + "], (unsigned long long)(int64_t)" + c.v + ");");
      break;
    case StateKind::MinMaxKey:
      ks.L(std::string(p.is_min ? "kdb_atomic_min_u64(&" : "kdb_atomic_max_u64(&") + sv + "[" + g + "], " +
           OKey(eg, c) + ");");
      break;
    case StateKind::MinMaxText:
      ks.L("kdb_atomic_str_minmax(&" + sv + "[" + g + "], " + c.v + ", " + (p.is_min ? "true" : "false") + ");");
      break;
    case StateKind::Count: break;
  }
  if (count) ks.L("atomicAdd((unsigned long long*)&" + sc + "[" + g + "], 1ULL);");
  ks.Close();
}

// The aggregate's result value from its state at slot `g`.
// `counted`: the group's count of non-NULL inputs was kept (NeedsCount);
// without it a group's SUM / MIN / MAX is never NULL.
CVal GroupResult(ExprGen& eg, const AggPlan& p, const std::string& sv, const std::string& sc,
                 const std::string& g, const std::string& first, bool counted = true) {
  const Type& rt = p.agg->type;
  const Type& ct = p.agg->kid(0).type;
  std::string v = sv + "[" + g + "]", c = "(int64_t)" + sc + "[" + g + "]";
  const std::string none = counted ? c + " == 0" : "false";
  switch (p.kind) {
    case StateKind::SumF64: return eg.Bind(rt, "__longlong_as_double((long long)" + v + ")", none);
    case StateKind::SumI64: return eg.Bind(rt, "(" + CType(rt.id) + ")(int64_t)" + v, none);
    case StateKind::AvgF64:
      return eg.Bind(rt, "__ddiv_rn(__longlong_as_double((long long)" + v + "), (double)" + c + ")", c + " == 0");
    case StateKind::Count: {
      std::string val = c;
      if (p.count_flag >= 0) val = "(" + c + " + (int64_t)((" + first + " >> " + std::to_string(p.count_flag) + ") & 1ULL))";
      return eg.Bind(rt, val, "false");
    }
    case StateKind::MinMaxKey: return eg.Bind(rt, OKeyInv(ct, v), none);
    case StateKind::MinMaxText: return eg.Bind(rt, "kdb_str_from_handle(" + v + ")", c + " == 0");
  }
  throw Error(-1, "bad aggregate");
}

// ---------------------------------------------------------------------------
// Ungrouped aggregate (aggregate_translator.cc:34-126): per-thread register
// state, block reduction to per-block partials, one finalize thread that
// combines the partials in block order and evaluates the output schema.
// ---------------------------------------------------------------------------

MatBuffer Executor::RunAggregate(const Operator& op) {
  int flags = 0;
  std::vector<AggPlan> plans;
  for (const auto& a : op.aggs) plans.push_back(PlanAgg(*a, flags));
  const int nw = static_cast<int>(plans.size()) * 2 + 2;  // per agg: value, count; + rows, first
  const int block = 256;
  // An aggregate of exact, order-free states (COUNT, MIN/MAX of keys,
  // integer SUM) over non-NULL inputs directly above a Skinner join is
  // evaluated inside the join's episode kernel, without materialising the
  // join's result (JOB-style MIN(...) queries).
  bool fuse = op.child().kind == OpKind::SKINNER_JOIN && !ctx_.OptStr("KDB_NO_SKINNER_AGG");
  for (const auto& p : plans)
    fuse = fuse && !p.child_nullable && p.count_flag < 0 &&
           (p.kind == StateKind::Count || p.kind == StateKind::MinMaxKey || p.kind == StateKind::SumI64);
  int grid = 1;
  uint64_t* part = nullptr;
  uint64_t* text_state = arena_.AllocT<uint64_t>(plans.size() + 1);
  bool any_text = false;  // only TEXT MIN/MAX read the text state
  for (const auto& p : plans) any_text |= p.kind == StateKind::MinMaxText;
  if (any_text) ctx_.Memset(text_state, 0, sizeof(uint64_t) * (plans.size() + 1));
  // Finalize.  Every output column gets a NULL array: an empty input emits a
  // single all-NULL row even for COUNT (aggregate_translator.cc:82-89).
  MatBuffer out = AllocMat(op.output, 1);
  for (auto& mc : out.cols)
    if (!mc.nulls) {
      mc.nullable = true;
      mc.nulls = arena_.AllocT<int8_t>(1);
    }
  bool fused_finalize = false;
  // (the finalize is emitted into the aggregate kernel's last CTA, or into
  // a one-block kernel after a fused Skinner join)
  auto emit_finalize = [&](KernelSource& fk, ExprGen& fg, const std::string& fp, const std::string& G) {
  std::string ftp = fk.Ptr(text_state, "uint64_t", true);
  {
    std::vector<WordKind> kinds(nw, WordKind::AddI64);
    for (size_t j = 0; j < plans.size(); j++) {
      const AggPlan& p = plans[j];
      if (p.kind == StateKind::SumF64 || p.kind == StateKind::AvgF64) kinds[j * 2] = WordKind::AddF64;
      if (p.kind == StateKind::MinMaxKey) kinds[j * 2] = p.is_min ? WordKind::MinU64 : WordKind::MaxU64;
    }
    kinds[nw - 1] = WordKind::MinU64;
    EmitPartialReduce(fk, fp, G, nw, kinds);
  }
  fk.Open("if (threadIdx.x == 0)");
  for (size_t j = 0; j < plans.size(); j++) {
    const AggPlan& p = plans[j];
    std::string J = std::to_string(j), W = std::to_string(j * 2), C = std::to_string(j * 2 + 1);
    switch (p.kind) {
      case StateKind::SumF64:
      case StateKind::AvgF64: fk.L("double s" + J + " = __longlong_as_double((long long)tot[" + W + "]);"); break;
      case StateKind::MinMaxKey: fk.L("uint64_t s" + J + " = tot[" + W + "];"); break;
      default: fk.L("int64_t s" + J + " = (int64_t)tot[" + W + "];"); break;
    }
    fk.L("int64_t c" + J + " = (int64_t)tot[" + C + "];");
  }
  fk.L("int64_t rows = (int64_t)tot[" + std::to_string(nw - 2) + "];");
  fk.L("uint64_t first = tot[" + std::to_string(nw - 1) + "];");
  std::vector<CVal> virt;
  for (size_t j = 0; j < plans.size(); j++) {
    const AggPlan& p = plans[j];
    std::string J = std::to_string(j);
    const Type& rt = p.agg->type;
    const Type& ct = p.agg->kid(0).type;
    switch (p.kind) {
      case StateKind::SumF64: virt.push_back(fg.Bind(rt, "s" + J, "c" + J + " == 0")); break;
      case StateKind::SumI64: virt.push_back(fg.Bind(rt, "(" + CType(rt.id) + ")s" + J, "c" + J + " == 0")); break;
      case StateKind::AvgF64:
        virt.push_back(fg.Bind(rt, "__ddiv_rn(s" + J + ", (double)c" + J + ")", "c" + J + " == 0"));
        break;
      case StateKind::Count: {
        std::string v = "c" + J;
        if (p.count_flag >= 0) v = "(c" + J + " + (int64_t)((first >> " + std::to_string(p.count_flag) + ") & 1ULL))";
        virt.push_back(fg.Bind(rt, v, "false"));
        break;
      }
      case StateKind::MinMaxKey: virt.push_back(fg.Bind(rt, OKeyInv(ct, "s" + J), "c" + J + " == 0")); break;
      case StateKind::MinMaxText:
        virt.push_back(fg.Bind(rt, "kdb_str_from_handle(" + ftp + "[" + J + "])", "c" + J + " == 0"));
        break;
    }
  }
  Scope s;
  s.virt = virt;
  std::vector<CVal> vals;
  for (const auto& c : op.output) vals.push_back(fg.Emit(*c.expr, s));
  for (size_t c = 0; c < out.cols.size(); c++) {
    const MatCol& mc = out.cols[c];
    std::string dp = fk.Ptr(mc.data, StoreType(mc.type.id));
    std::string val = mc.type.id == TypeId::BOOLEAN ? "(int8_t)(" + vals[c].v + " ? 1 : 0)" : vals[c].v;
    fk.L(dp + "[0] = " + val + ";");
    std::string np = fk.Ptr(mc.nulls, "int8_t");
    fk.L(np + "[0] = (rows == 0 || (" + vals[c].n + ")) ? 1 : 0;");
  }
  std::string posp = fk.Ptr(out.pos, "uint64_t");
  fk.L(posp + "[0] = 0;");
  fk.Close();
  };
  if (fuse) {
    part = arena_.AllocT<uint64_t>(nw);
    std::vector<uint64_t> init(nw, 0);
    for (size_t j = 0; j < plans.size(); j++)
      if (plans[j].kind == StateKind::MinMaxKey && plans[j].is_min) init[2 * j] = ~0ULL;
    init[nw - 1] = ~0ULL;
    ctx_.H2D(part, init.data(), sizeof(uint64_t) * nw);
    SkinnerAgg sa;
    sa.plans = &plans;
    sa.state = part;
    sa.nw = nw;
    RunSkinner(op.child(), &sa);
  } else {
  PrepareInput(op.child());

  KernelSource ks;
  ExprGen eg(ctx_, ks);
  int64_t src_rows = 0;
  for (size_t j = 0; j < plans.size(); j++) {
    const AggPlan& p = plans[j];
    std::string J = std::to_string(j);
    switch (p.kind) {
      case StateKind::SumF64:
      case StateKind::AvgF64: ks.L("double s" + J + " = 0.0;"); break;
      case StateKind::MinMaxKey: ks.L("uint64_t s" + J + " = " + (p.is_min ? "~0ULL;" : "0ULL;")); break;
      default: ks.L("int64_t s" + J + " = 0;"); break;
    }
    ks.L("int64_t c" + J + " = 0;");
  }
  ks.L("int64_t rows = 0;");
  ks.L("uint64_t first = ~0ULL;");
  std::string tsp = ks.Ptr(text_state, "uint64_t");
  auto consume = [&](const std::vector<CVal>& in, const std::string& pos) {
    Scope s;
    s.child.push_back(in);
    std::string fl = "0ULL";
    for (size_t j = 0; j < plans.size(); j++) {
      const AggPlan& p = plans[j];
      CVal c = eg.Emit(p.agg->kid(0), s);
      std::string J = std::to_string(j);
      if (p.count_flag >= 0) fl += " | ((" + c.n + ") ? " + std::to_string(1 << p.count_flag) + "ULL : 0ULL)";
      ks.Open("if (!(" + c.n + "))");
      switch (p.kind) {
        case StateKind::SumF64: ks.L("s" + J + " = __dadd_rn(s" + J + ", " + c.v + ");"); break;
        case StateKind::AvgF64: ks.L("s" + J + " = __dadd_rn(s" + J + ", (double)" + c.v + ");"); break;
        case StateKind::SumI64:
          ks.L("s" + J + " = (int64_t)((uint64_t)s" + J + " + (uint64_t)(int64_t)" + c.v + ");");
          break;
        case StateKind::MinMaxKey:
          ks.L("{ uint64_t k = " + OKey(eg, c) + "; s" + J + " = " + (p.is_min ? "(k < s" : "(k > s") + J +
               ") ? k : s" + J + "; }");
          break;
        case StateKind::MinMaxText:
          ks.L("kdb_atomic_str_minmax(&" + tsp + "[" + J + "], " + c.v + ", " + (p.is_min ? "true" : "false") + ");");
          break;
        case StateKind::Count: break;
      }
      ks.L("c" + J + "++;");
      ks.Close();
    }
    ks.L("rows++;");
    ks.L("{ uint64_t f = ((uint64_t)(" + pos + ") << 8) | (" + fl + "); first = f < first ? f : first; }");
  };
  if (Streamable(op.child())) EmitStream(ks, eg, op.child(), consume, src_rows);
  else EmitMatScan(ks, mats_.at(&op.child()), nullptr, consume, src_rows);

  // Enough rows per thread that every thread runs a few prefetched
  // iterations (at 1M rows one row group per thread left most of the
  // kernel's time to ramp-up and the block reductions), at least one CTA
  // per SM.
  {
    const int64_t rpt = ctx_.OptStr("KDB_AGG_ROWS_PER_THREAD") ? std::atoll(ctx_.OptStr("KDB_AGG_ROWS_PER_THREAD"))
                                                               : 16;
    const int64_t want = (std::max<int64_t>(src_rows, 1) + block * rpt - 1) / (block * rpt);
    grid = static_cast<int>(std::max<int64_t>(std::min<int64_t>(ctx_.GridFor(std::max<int64_t>(src_rows, 1), block),
                                                                want),
                                              std::min<int64_t>(ctx_.num_sms, ctx_.GridFor(std::max<int64_t>(src_rows, 1), block))));
  }
  part = arena_.AllocT<uint64_t>(static_cast<size_t>(grid) * nw);
  std::string pp = ks.Ptr(part, "uint64_t");
  ks.L("__shared__ uint64_t red_u[32];");
  ks.L("__shared__ double red_d[32];");
  ks.L("__shared__ int64_t red_i[32];");
  auto store = [&](int w, const std::string& val) {
    ks.L("if (threadIdx.x == 0) " + pp + "[(int64_t)" + std::to_string(w) + " * gridDim.x + blockIdx.x] = " + val +
         ";");
  };
  for (size_t j = 0; j < plans.size(); j++) {
    const AggPlan& p = plans[j];
    std::string J = std::to_string(j);
    switch (p.kind) {
      case StateKind::SumF64:
      case StateKind::AvgF64:
        ks.Open("");
        ks.L("double t = kdb_block_reduce(s" + J + ", KdbAddF64(), red_d);");
        store(static_cast<int>(j) * 2, "(uint64_t)__double_as_longlong(t)");
        ks.Close();
        break;
      case StateKind::SumI64:
        ks.Open("");
        ks.L("int64_t t = kdb_block_reduce(s" + J + ", KdbAddI64(), red_i);");
        store(static_cast<int>(j) * 2, "(uint64_t)t");
        ks.Close();
        break;
      case StateKind::MinMaxKey:
        ks.Open("");
        ks.L("uint64_t t = kdb_block_reduce(s" + J + (p.is_min ? ", KdbMinU64(), red_u);" : ", KdbMaxU64(), red_u);"));
        store(static_cast<int>(j) * 2, "t");
        ks.Close();
        break;
      default:
        store(static_cast<int>(j) * 2, "0ULL");
        break;
    }
    ks.Open("");
    ks.L("int64_t t = kdb_block_reduce(c" + J + ", KdbAddI64(), red_i);");
    store(static_cast<int>(j) * 2 + 1, "(uint64_t)t");
    ks.Close();
  }
  ks.Open("");
  ks.L("int64_t t = kdb_block_reduce(rows, KdbAddI64(), red_i);");
  store(nw - 2, "(uint64_t)t");
  ks.Close();
  ks.Open("");
  ks.L("uint64_t t = kdb_block_reduce(first, KdbMinU64(), red_u);");
  store(nw - 1, "t");
  ks.Close();
  // The last CTA can combine the partials itself (KDB_AGG_FUSED_FINALIZE),
  // but measured at 1M rows that kernel's serial tail costs more than the
  // second one-block launch (13.1 us vs 10.6 + 6.6 us; step 50.2 vs 49.1 us)
  fused_finalize = ctx_.OptStr("KDB_AGG_FUSED_FINALIZE") != nullptr;
  if (fused_finalize) {
    // the last CTA to finish combines the partials (same fixed-order
    // reduction as the separate finalize) and writes the result row
    uint32_t* done = arena_.AllocT<uint32_t>(1);
    ctx_.Memset(done, 0, sizeof(uint32_t));
    const std::string dn = ks.Ptr(done, "unsigned");
    ks.L("__shared__ bool kdb_last_block;");
    ks.L("__threadfence();");
    ks.L("__syncthreads();");
    ks.L("if (threadIdx.x == 0) kdb_last_block = atomicAdd(" + dn + ", 1u) == gridDim.x - 1;");
    ks.L("__syncthreads();");
    ks.Open("if (kdb_last_block)");
    ks.L("__threadfence();");
    emit_finalize(ks, eg, pp, "gridDim.x");
    ks.Close();
  }
  {
    // KDB_AGG_MINB: CTAs per SM the register budget must allow (launch
    // bounds); more resident CTAs keep more rows' loads in flight
    const char* mb = ctx_.OptStr("KDB_AGG_MINB");
    std::string src = ks.Kernel("kdb_aggregate", block, mb ? std::max(1, std::atoi(mb)) : 1);
    CUfunction f = ctx_.Kernel(src, "kdb_aggregate");
    ctx_.Launch(f, grid, block, ks.Args(), 0, "aggregate");
  }
  }  // not fused

  if (!fused_finalize) {
    KernelSource fk;
    ExprGen fg(ctx_, fk);
    const std::string fp = fk.Ptr(part, "uint64_t", true);
    emit_finalize(fk, fg, fp, fk.Word(static_cast<uint64_t>(grid)));
    std::string src = fk.Kernel("kdb_aggregate_finalize", 256);
    CUfunction f = ctx_.Kernel(src, "kdb_aggregate_finalize");
    ctx_.Launch(f, 1, 256, fk.Args(), 0, "aggregate finalize");
  }
  ctx_.CheckDeviceError("aggregate");
  out.rows = 1;
  out.pos_is_index = true;
  return out;
}

// ---------------------------------------------------------------------------
// Group-by (group_by_aggregate_translator.cc:36-111 + AggregateHashTable):
// a device open-addressing table updated with atomics, then compaction of the
// occupied slots, a radix sort on each group's first stream position (the
// reference's ForEach emits groups in insertion order,
// compile/proxy/aggregate_hash_table.cc:245-291) and one output kernel.
// ---------------------------------------------------------------------------

KeyLayout PlanKeys(Context& ctx, const std::vector<std::unique_ptr<Expr>>& keys) {
  KeyLayout kl;
  for (const auto& k : keys) {
    int w = 0;
    uint64_t card = 0;
    switch (k->type.id) {
      case TypeId::ENUM: {
        uint64_t n = ctx.Enum(k->type.enum_id).values.size();
        w = 1;
        while ((1ULL << w) < n) w++;
        card = n;
        break;
      }
      case TypeId::BOOLEAN: w = 1; card = 2; break;
      case TypeId::SMALLINT: w = 16; break;
      case TypeId::INT:
      case TypeId::DATE: w = 32; break;
      case TypeId::BIGINT:
      case TypeId::REAL: w = 64; break;
      case TypeId::TEXT: w = 1000; break;
    }
    kl.offset.push_back(kl.bits);
    kl.card.push_back(card);
    kl.width.push_back(w);
    kl.nullable.push_back(k->nullable);
    kl.bits += w + (k->nullable ? 1 : 0);
    if (card == 0) kl.small_domain = false;
    else if (kl.small_domain) kl.domain *= card + (k->nullable ? 1 : 0);
  }
  kl.packed = kl.bits <= 63;
  return kl;
}

// Structural signature of an expression (identical signatures compute the
// same value, so their accumulators can be shared).
std::string ExprSig(const Expr& e) {
  std::ostringstream o;
  o << static_cast<int>(e.kind) << ":" << static_cast<int>(e.type.id) << "." << e.type.enum_id << ":"
    << e.child_idx << "." << e.column_idx << ":" << static_cast<int>(e.bop) << static_cast<int>(e.uop)
    << static_cast<int>(e.agg) << ":" << e.lit_null << "," << e.ival << "," << F64Lit(e.fval) << ","
    << e.sval.size() << "'" << e.sval << "'(";
  for (const auto& k : e.kids) o << ExprSig(*k) << ";";
  for (int32_t v : e.in_values) o << v << ",";
  o << ")" << e.regex.size() << "'" << e.regex << "'";
  return o.str();
}

// Identity of a Skinner child for the serving build cache: the relation
// (and the device arrays it reads), its scan columns, filters and outputs,
// and the columns indexed.
std::string Executor::ChildSig(const Operator& child, const std::set<int>& index_cols) const {
  std::ostringstream o;
  o << static_cast<int>(child.kind) << "|" << child.relation << "|";
  auto it = ctx_.tables.find(child.relation);
  if (it != ctx_.tables.end()) o << it->second.rows << "|";
  for (const auto& sc : child.scan_columns) {
    o << sc.name << ":" << static_cast<int>(sc.type.id) << ":";
    if (it != ctx_.tables.end()) {
      auto c = it->second.cols.find(sc.name);
      if (c != it->second.cols.end()) o << reinterpret_cast<uintptr_t>(c->second.data);
    }
    o << ",";
  }
  o << "|f";
  for (const auto& f : child.filters) o << ExprSig(*f) << ";";
  o << "|o";
  for (const auto& c : child.output) o << ExprSig(*c.expr) << ";";
  o << "|i";
  for (int c : index_cols) o << c << ",";
  return o.str();
}

// Small-domain group-by: every key is ENUM or BOOLEAN, so a group id is the
// mixed-radix number of the key digits (NULL is one extra digit).  Each
// thread keeps all groups' states in registers (selects, no atomics); at the
// end a warp-shuffle + shared-memory reduction gives one partial per CTA and
// a single finalize block combines the partials in a fixed order, orders the
// present groups by their first stream position (the reference's insertion
// order) and evaluates the output schema.  This is the pre-aggregation the
// reference's AggregateHashTable::UpdateOrInsert hot loop
// (compile/proxy/aggregate_hash_table.cc:187-243) turns into on a GPU when the
// group count is tiny.
MatBuffer Executor::RunGroupByDense(const Operator& op, const std::vector<AggPlan>& plans,
                                    const KeyLayout& kl, const Operator* order_by) {
  const int64_t D = static_cast<int64_t>(kl.domain);
  // words per group: per-agg value / count words (shared when identical),
  // then rows and first position
  std::vector<DenseWord> words;
  std::map<std::string, int> word_of;
  std::vector<int> vword(plans.size(), -1), cword(plans.size(), -1);
  auto add_word = [&](const std::string& sig, WordKind k, const std::string& init, const std::string& ct) {
    auto it = word_of.find(sig);
    if (it != word_of.end()) return it->second;
    words.push_back({k, init, ct});
    word_of[sig] = static_cast<int>(words.size()) - 1;
    return static_cast<int>(words.size()) - 1;
  };
  for (size_t j = 0; j < plans.size(); j++) {
    const AggPlan& p = plans[j];
    std::string csig = ExprSig(p.agg->kid(0));
    switch (p.kind) {
      case StateKind::SumF64:
      case StateKind::AvgF64: vword[j] = add_word("fsum|" + csig, WordKind::AddF64, "0.0", "double"); break;
      case StateKind::SumI64: vword[j] = add_word("isum|" + csig, WordKind::AddI64, "0", "int64_t"); break;
      case StateKind::MinMaxKey:
        vword[j] = p.is_min ? add_word("min|" + csig, WordKind::MinU64, "~0ULL", "uint64_t")
                            : add_word("max|" + csig, WordKind::MaxU64, "0ULL", "uint64_t");
        break;
      default: break;
    }
    if (p.child_nullable) cword[j] = add_word("cnt|" + csig, WordKind::AddI64, "0", "int64_t");
  }
  const int rows_w = static_cast<int>(words.size());
  words.push_back({WordKind::AddI64, "0", "int64_t"});
  const int first_w = static_cast<int>(words.size());
  words.push_back({WordKind::MinU64, "~0ULL", "uint64_t"});
  const int W = static_cast<int>(words.size());
  const int64_t K = D * W;
  auto opt_int = [&](const char* name, int dflt) {
    const char* v = ctx_.OptStr(name);
    return v ? std::atoi(v) : dflt;
  };
  // Accumulators in registers (every row updates every group's words under a
  // predicate) while groups x words <= 64: 256-thread CTAs, one per SM, so
  // a thread may hold them all plus two iterations of loads (measured on
  // the Q1 shape, 42 words: 51.5 us and a 97 us query, against 49.6 us and
  // 103 us for 128 x 2 -- twice the partials for the finalize -- 156 us
  // for 512 x 1 and 53.6 us for the shared-memory form).  Beyond that,
  // per-thread shared-memory slots indexed by the group id (a row touches
  // only its own group's words) in 64-thread CTAs, 6 per SM.
  // KDB_DENSE_SMEM=0/1 forces either; KDB_DENSE_BLOCK/MINB/GRID set the
  // shape.
  // KDB_DENSE_TMA: the scan's tiles come into shared memory by TMA bulk
  // copies (persistent CTAs, KDB_TMA_CTAS per SM of KDB_TMA_BLOCK threads,
  // KDB_TMA_STAGES tiles of KDB_TMA_TILE rows in flight), with either kind
  // of accumulator.  Measured on the Q1 shape with shared-memory
  // accumulators it is slower (78-131 us over the shapes tried, against
  // 52 us; 8 warps per SM spend their issue slots on the accumulators'
  // shared-memory read-modify-write chains).
  const bool want_tma = ctx_.OptStr("KDB_DENSE_TMA") != nullptr && Streamable(op.child());
  const char* smem_env = ctx_.OptStr("KDB_DENSE_SMEM");
  const bool want_smem = smem_env ? std::atoi(smem_env) != 0 : K > 64;
  const int block = want_tma ? opt_int("KDB_TMA_BLOCK", 128) : opt_int("KDB_DENSE_BLOCK", want_smem ? 64 : 256);
  const int min_blocks = want_tma ? opt_int("KDB_TMA_CTAS", 2) : opt_int("KDB_DENSE_MINB", want_smem ? 6 : 1);
  const int grid_per_sm = want_tma ? opt_int("KDB_TMA_CTAS", 2) : opt_int("KDB_DENSE_GRID", want_smem ? 6 : 1);
  const bool smem_fits = K * block * 8 <= 48 * 1024;  // static shared memory limit
  const bool in_smem = smem_fits && want_smem;

  auto reg = [&](int64_t g, int w) { return "a" + std::to_string(g) + "_" + std::to_string(w); };
  auto combine = [&](WordKind k, const std::string& a, const std::string& b) -> std::string {
    switch (k) {
      case WordKind::AddF64: return "__dadd_rn(" + a + ", " + b + ")";
      case WordKind::AddI64: return "(int64_t)((uint64_t)" + a + " + (uint64_t)" + b + ")";
      case WordKind::MinU64: return "(" + b + " < " + a + " ? " + b + " : " + a + ")";
      case WordKind::MaxU64: return "(" + b + " > " + a + " ? " + b + " : " + a + ")";
    }
    return a;
  };
  auto to_bits = [&](const DenseWord& w, const std::string& v) {
    return w.ctype == "double" ? "(uint64_t)__double_as_longlong(" + v + ")" : "(uint64_t)" + v;
  };
  auto from_bits = [&](const DenseWord& w, const std::string& v) {
    return w.ctype == "double" ? "__longlong_as_double((long long)" + v + ")" : "(" + w.ctype + ")" + v;
  };

  KernelSource ks;
  ExprGen eg(ctx_, ks);
  auto slot = [&](int w) { return "s" + std::to_string(w); };
  const std::string DB = std::to_string(D * block);
  if (in_smem) {
    for (int w = 0; w < W; w++) {
      ks.L("__shared__ " + words[w].ctype + " " + slot(w) + "[" + DB + "];");
      ks.L("for (int i = threadIdx.x; i < " + DB + "; i += blockDim.x) " + slot(w) + "[i] = " + words[w].init + ";");
    }
  } else {
    for (int64_t g = 0; g < D; g++)
      for (int w = 0; w < W; w++) ks.L(words[w].ctype + " " + reg(g, w) + " = " + words[w].init + ";");
  }
  int64_t src_rows = 0;
  // a streamed child without a join hands each thread its rows in ascending
  // position (grid-stride rows or tiles); a join's matches of one probe row
  // come in table order, and a materialised child's positions in any order
  const bool ascending_rows = Streamable(op.child()) && !StreamHasJoin(op.child()) &&
                              !ctx_.OptStr("KDB_DENSE_FIRST_MIN");
  auto consume = [&](const std::vector<CVal>& in, const std::string& pos) {
    Scope s;
    s.child.push_back(in);
    std::string gid = "0";
    int64_t stride = 1;
    for (size_t k = 0; k < op.group_by.size(); k++) {
      CVal c = eg.Emit(*op.group_by[k], s);
      std::string digit = c.type.id == TypeId::BOOLEAN ? "(" + c.v + " ? 1 : 0)" : "(int64_t)" + c.v;
      if (kl.nullable[k]) digit = "((" + c.n + ") ? " + std::to_string(kl.card[k]) + " : " + digit + ")";
      gid += " + " + digit + " * " + std::to_string(stride);
      stride *= static_cast<int64_t>(kl.card[k] + (kl.nullable[k] ? 1 : 0));
    }
    std::string G = ks.Fresh("gid");
    ks.L("int64_t " + G + " = " + gid + ";");
    // per-row contributions of every word
    std::vector<std::string> contrib(W), active(W, "true");
    std::string fl = "0ULL";
    for (size_t j = 0; j < plans.size(); j++) {
      const AggPlan& p = plans[j];
      CVal c = eg.Emit(p.agg->kid(0), s);
      if (p.count_flag >= 0) fl += " | ((" + c.n + ") ? " + std::to_string(1 << p.count_flag) + "ULL : 0ULL)";
      std::string nn = "!(" + c.n + ")";
      if (vword[j] >= 0 && contrib[vword[j]].empty()) {
        switch (p.kind) {
          case StateKind::SumF64: contrib[vword[j]] = c.v; break;
          case StateKind::AvgF64: contrib[vword[j]] = "(double)" + c.v; break;
          case StateKind::SumI64: contrib[vword[j]] = "(int64_t)" + c.v; break;
          default: contrib[vword[j]] = OKey(eg, c); break;
        }
        active[vword[j]] = nn;
      }
      if (cword[j] >= 0 && contrib[cword[j]].empty()) {
        contrib[cword[j]] = "(int64_t)1";
        active[cword[j]] = nn;
      }
    }
    contrib[rows_w] = "(int64_t)1";
    contrib[first_w] = "(((uint64_t)(" + pos + ") << 8) | (" + fl + "))";
    std::vector<std::string> cv(W);
    for (int w = 0; w < W; w++) {
      cv[w] = ks.Fresh("c");
      ks.L(words[w].ctype + " " + cv[w] + " = " + contrib[w] + ";");
    }
    if (in_smem) {
      // a key outside the domain matches no group (as in the register form)
      ks.Open("if ((uint64_t)" + G + " < " + std::to_string(D) + "ULL)");
      std::string I = ks.Fresh("si");
      ks.L("const int " + I + " = (int)" + G + " * " + std::to_string(block) + " + threadIdx.x;");
      for (int w = 0; w < W; w++) {
        if (w == first_w && ascending_rows) continue;
        if (w == rows_w && ascending_rows) {
          // a thread meets its rows in ascending position: the group's
          // first row for this thread is the one that finds its count at 0
          const std::string old = ks.Fresh("nr");
          ks.L("const int64_t " + old + " = " + slot(w) + "[" + I + "];");
          ks.L(slot(w) + "[" + I + "] = " + old + " + 1;");
          ks.L("if (" + old + " == 0) " + slot(first_w) + "[" + I + "] = " + cv[first_w] + ";");
          continue;
        }
        std::string upd = slot(w) + "[" + I + "] = " + combine(words[w].kind, slot(w) + "[" + I + "]", cv[w]) + ";";
        ks.L(active[w] == "true" ? upd : "if (" + active[w] + ") " + upd);
      }
      ks.Close();
      return;
    }
    if (ctx_.OptStr("KDB_DENSE_SWITCH")) {
      // KDB_DENSE_SWITCH: a branch per group, so that a warp issues only the
      // updates of the groups its rows belong to (four paths of W updates
      // for the Q1 shape) instead of every group's words under a predicate.
      // Measured slower on the Q1 shape (59.9 against 51.7 us): the
      // divergent paths serialise.  A key outside the domain matches no case.
      ks.Open("switch (" + G + ")");
      for (int64_t g = 0; g < D; g++) {
        ks.Open("case " + std::to_string(g) + ":");
        for (int w = 0; w < W; w++) {
          const std::string upd = reg(g, w) + " = " + combine(words[w].kind, reg(g, w), cv[w]) + ";";
          ks.L(active[w] == "true" ? upd : "if (" + active[w] + ") " + upd);
        }
        ks.L("break;");
        ks.Close();
      }
      ks.L("default: break;");
      ks.Close();
      return;
    }
    for (int64_t g = 0; g < D; g++) {
      std::string h = ks.Fresh("h");
      ks.L("bool " + h + " = " + G + " == " + std::to_string(g) + ";");
      for (int w = 0; w < W; w++) {
        std::string cond = active[w] == "true" ? h : "(" + h + " && " + active[w] + ")";
        ks.L(reg(g, w) + " = " + cond + " ? " + combine(words[w].kind, reg(g, w), cv[w]) + " : " + reg(g, w) + ";");
      }
    }
  };
  if (want_tma) {
    tma_tile_ = opt_int("KDB_TMA_TILE", 512);
    tma_stages_ = opt_int("KDB_TMA_STAGES", 3);
  }
  if (Streamable(op.child())) EmitStream(ks, eg, op.child(), consume, src_rows);
  else EmitMatScan(ks, mats_.at(&op.child()), nullptr, consume, src_rows);
  const size_t dsmem = tma_smem_;
  tma_tile_ = tma_stages_ = 0;
  tma_smem_ = 0;

  int grid = static_cast<int>(std::min<int64_t>(ctx_.GridFor(std::max<int64_t>(src_rows, 1), block),
                                                static_cast<int64_t>(ctx_.num_sms) * grid_per_sm));
  uint64_t* part = arena_.AllocT<uint64_t>(static_cast<size_t>(grid) * K);
  std::string PP = ks.Ptr(part, "uint64_t");
  if (in_smem) {
    // per (group, word): fold the block's thread slots in thread order
    ks.L("__syncthreads();");
    ks.Open("for (int k = threadIdx.x; k < " + std::to_string(K) + "; k += blockDim.x)");
    ks.L("const int g = k / " + std::to_string(W) + ", w = k % " + std::to_string(W) + ";");
    ks.L("uint64_t acc = 0;");
    ks.Open("switch (w)");
    for (int w = 0; w < W; w++) {
      const std::string base = "g * " + std::to_string(block);
      ks.Open("case " + std::to_string(w) + ":");
      ks.L(words[w].ctype + " v = " + slot(w) + "[" + base + "];");
      ks.L("for (int i = 1; i < " + std::to_string(block) + "; i++) v = " +
           combine(words[w].kind, "v", slot(w) + "[" + base + " + i]") + ";");
      ks.L("acc = " + to_bits(words[w], "v") + ";");
      ks.L("break;");
      ks.Close();
    }
    ks.Close();
    ks.L(PP + "[(int64_t)k * gridDim.x + blockIdx.x] = acc;");
    ks.Close();
  } else {
  ks.L("__shared__ uint64_t red[" + std::to_string(block / 32) + "][" + std::to_string(K) + "];");
  ks.L("const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;");
  for (int64_t g = 0; g < D; g++)
    for (int w = 0; w < W; w++) {
      std::string r = reg(g, w);
      ks.L("for (int o = 16; o > 0; o >>= 1) { " + words[w].ctype + " y = __shfl_xor_sync(0xffffffffu, " + r +
           ", o); " + r + " = " + combine(words[w].kind, r, "y") + "; }");
      ks.L("if (lane == 0) red[warp][" + std::to_string(g * W + w) + "] = " + to_bits(words[w], r) + ";");
    }
  ks.L("__syncthreads();");
  ks.Open("for (int k = threadIdx.x; k < " + std::to_string(K) + "; k += blockDim.x)");
  ks.L("int w = k % " + std::to_string(W) + ";");
  ks.L("uint64_t acc = red[0][k];");
  ks.Open("for (int wp = 1; wp < " + std::to_string(block / 32) + "; wp++)");
  ks.L("uint64_t y = red[wp][k];");
  ks.Open("switch (w)");
  for (int w = 0; w < W; w++) {
    ks.L("case " + std::to_string(w) + ": acc = " +
         to_bits(words[w], combine(words[w].kind, from_bits(words[w], "acc"), from_bits(words[w], "y"))) + "; break;");
  }
  ks.Close();
  ks.Close();
  ks.L(PP + "[(int64_t)k * gridDim.x + blockIdx.x] = acc;");
  ks.Close();
  }
  {
    std::string src = ks.Kernel("kdb_group_by_dense", block, min_blocks);
    CUfunction f = ctx_.Kernel(src, "kdb_group_by_dense");
    ctx_.Launch(f, grid, block, ks.Args(), dsmem, "group by");
  }

  // finalize: one block combines the per-CTA partials (warp per word, fixed
  // order), orders present groups by first position, evaluates the output
  MatBuffer out = AllocMat(op.output, D);
  uint64_t* ngroups = arena_.AllocT<uint64_t>(1);
  KernelSource fk;
  ExprGen fg(ctx_, fk);
  std::string FP = fk.Ptr(part, "uint64_t", true);
  std::string NG = fk.Ptr(ngroups, "uint64_t");
  std::string GW = "(int64_t)" + fk.Word(static_cast<uint64_t>(grid));
  fk.L("__shared__ int32_t order[" + std::to_string(D) + "];");
  {
    std::vector<WordKind> kinds(K);
    for (int64_t k = 0; k < K; k++) kinds[k] = words[k % W].kind;
    EmitPartialReduce(fk, FP, GW, static_cast<int>(K), kinds);
  }
  // A parent ORDER BY whose keys are all enum GROUP BY keys is done here:
  // the groups, in stream order, are re-ranked by the ORDER BY comparator
  // (enum string order, NULLs after values, ascending or descending) with
  // ties broken by the reference merge sort's tie path of the stream rank --
  // the order the separate ORDER BY would produce.
  std::vector<int> sort_key, sort_asc;
  if (order_by) {
    for (size_t k = 0; k < order_by->sort_keys.size(); k++) {
      const Expr& sk = *order_by->sort_keys[k];
      int key = -1;
      if (sk.kind == ExprKind::ColRef && sk.child_idx == 0 && sk.column_idx < static_cast<int>(op.output.size())) {
        const Expr& oe = *op.output[sk.column_idx].expr;
        if (oe.kind == ExprKind::VirtColRef && oe.column_idx < static_cast<int>(op.group_by.size()) &&
            op.group_by[oe.column_idx]->type.id == TypeId::ENUM)
          key = oe.column_idx;
      }
      if (key < 0) {
        sort_key.clear();
        break;
      }
      sort_key.push_back(key);
      sort_asc.push_back(order_by->asc[k] ? 1 : 0);
    }
  }
  const bool fuse_order_pre = !sort_key.empty();
  // the sort keys' enum string ranks, staged in shared memory by all
  // threads (thread 0's comparisons below then wait on no global load)
  std::vector<std::string> rank_smem(op.group_by.size());
  if (fuse_order_pre) {
    for (int k : sort_key) {
      if (!rank_smem[k].empty()) continue;
      const std::string name = "kdb_rk" + std::to_string(k);
      const int64_t card = static_cast<int64_t>(kl.card[k]);
      fk.L("__shared__ int32_t " + name + "[" + std::to_string(std::max<int64_t>(card, 1)) + "];");
      fk.L("for (int i = threadIdx.x; i < " + std::to_string(card) + "; i += blockDim.x) " + name + "[i] = " +
           fg.EnumRank(op.group_by[k]->type, "i") + ";");
      rank_smem[k] = name;
    }
    fk.L("__syncthreads();");
  }
  // thread 0 orders the present groups (shared memory only); all threads
  // then write one output row each
  fk.L("__shared__ int32_t kdb_ng;");
  fk.L("__shared__ int32_t kdb_fin[" + std::to_string(D) + "];");
  fk.Open("if (threadIdx.x == 0)");
  fk.L("int32_t ng = 0;");
  fk.Open("for (int32_t g = 0; g < " + std::to_string(D) + "; g++)");
  fk.Open("if ((int64_t)tot[g * " + std::to_string(W) + " + " + std::to_string(rows_w) + "] > 0)");
  // insertion by first position
  fk.L("int32_t j = ng++;");
  fk.L("uint64_t fg = tot[g * " + std::to_string(W) + " + " + std::to_string(first_w) + "];");
  fk.L("while (j > 0 && tot[order[j - 1] * " + std::to_string(W) + " + " + std::to_string(first_w) +
       "] > fg) { order[j] = order[j - 1]; j--; }");
  fk.L("order[j] = g;");
  fk.Close();
  fk.Close();
  fk.L("*" + NG + " = (uint64_t)ng;");
  const bool fuse_order = !sort_key.empty();
  if (fuse_order) {
    // digit of key k of group g, and its enum string rank (NULL: -1)
    auto key_rank = [&](int k, const std::string& g) {
      int64_t stride = 1;
      for (int j = 0; j < k; j++) stride *= static_cast<int64_t>(kl.card[j] + (kl.nullable[j] ? 1 : 0));
      const int64_t base = static_cast<int64_t>(kl.card[k] + (kl.nullable[k] ? 1 : 0));
      const std::string digit = "((" + g + " / " + std::to_string(stride) + ") % " + std::to_string(base) + ")";
      const std::string rank = "(int64_t)" + rank_smem[k] + "[(int32_t)" + digit + "]";
      if (!kl.nullable[k]) return rank;
      return "(" + digit + " == " + std::to_string(kl.card[k]) + " ? (int64_t)-1 : " + rank + ")";
    };
    fk.Open("auto kless = [&](int32_t ra, int32_t rb) -> bool");
    fk.L("const int64_t ga = order[ra], gb = order[rb];");
    for (size_t k = 0; k < sort_key.size(); k++) {
      const std::string K = std::to_string(k);
      fk.L("{ const int64_t xa = " + key_rank(sort_key[k], "ga") + ", xb = " + key_rank(sort_key[k], "gb") + ";");
      // proxy::LessThan: a NULL (-1) sorts after every value
      fk.L("  const bool ab = xa >= 0 && (xb < 0 || xa < xb), ba = xb >= 0 && (xa < 0 || xb < xa);");
      fk.L(std::string("  if (ab) return ") + (sort_asc[k] ? "true" : "false") + "; if (ba) return " +
           (sort_asc[k] ? "false" : "true") + "; }");
    }
    fk.L("return kdb_tie_path((uint64_t)ra, (uint64_t)ng) < kdb_tie_path((uint64_t)rb, (uint64_t)ng);");
    fk.indent--;
    fk.L("};");
    fk.L("int32_t* fin = kdb_fin;");
    fk.Open("for (int32_t r = 0; r < ng; r++)");
    fk.L("int32_t j = r;");
    fk.L("while (j > 0 && kless(r, fin[j - 1])) { fin[j] = fin[j - 1]; j--; }");
    fk.L("fin[j] = r;");
    fk.Close();
  }
  fk.L("kdb_ng = ng;");
  fk.Close();
  fk.L("__syncthreads();");
  std::vector<std::string> optr, onull;
  for (const auto& c : out.cols) {
    optr.push_back(fk.Ptr(c.data, StoreType(c.type.id)));
    onull.push_back(c.nullable ? fk.Ptr(c.nulls, "int8_t") : "");
  }
  std::string posp = fk.Ptr(out.pos, "uint64_t");
  fk.L("const int32_t ng = kdb_ng;");
  fk.Open("for (int32_t r = threadIdx.x; r < ng; r += blockDim.x)");
  fk.L(fuse_order ? "int64_t g = order[kdb_fin[r]];" : "int64_t g = order[r];");
  fk.L("const uint64_t* t = tot + g * " + std::to_string(W) + ";");
  fk.L("int64_t rows = (int64_t)t[" + std::to_string(rows_w) + "];");
  fk.L("uint64_t fst = t[" + std::to_string(first_w) + "];");
  std::vector<CVal> virt;
  int64_t stride = 1;
  for (size_t k = 0; k < op.group_by.size(); k++) {
    const Type& ty = op.group_by[k]->type;
    int64_t base = static_cast<int64_t>(kl.card[k] + (kl.nullable[k] ? 1 : 0));
    std::string digit = "((g / " + std::to_string(stride) + ") % " + std::to_string(base) + ")";
    std::string v = ty.id == TypeId::BOOLEAN ? "(" + digit + " != 0)" : "(" + CType(ty.id) + ")" + digit;
    std::string n = kl.nullable[k] ? "(" + digit + " == " + std::to_string(kl.card[k]) + ")" : "false";
    virt.push_back(fg.Bind(ty, v, n));
    stride *= base;
  }
  for (size_t j = 0; j < plans.size(); j++) {
    const AggPlan& p = plans[j];
    const Type& rt = p.agg->type;
    const Type& ct = p.agg->kid(0).type;
    std::string cnt = cword[j] >= 0 ? "(int64_t)t[" + std::to_string(cword[j]) + "]" : "rows";
    std::string v = vword[j] >= 0 ? from_bits(words[vword[j]], "t[" + std::to_string(vword[j]) + "]") : "";
    switch (p.kind) {
      case StateKind::SumF64: virt.push_back(fg.Bind(rt, v, cnt + " == 0")); break;
      case StateKind::SumI64: virt.push_back(fg.Bind(rt, "(" + CType(rt.id) + ")" + v, cnt + " == 0")); break;
      case StateKind::AvgF64: virt.push_back(fg.Bind(rt, "__ddiv_rn(" + v + ", (double)" + cnt + ")", cnt + " == 0")); break;
      case StateKind::Count: {
        std::string val = cnt;
        if (p.count_flag >= 0) val = "(" + cnt + " + (int64_t)((fst >> " + std::to_string(p.count_flag) + ") & 1ULL))";
        virt.push_back(fg.Bind(rt, val, "false"));
        break;
      }
      case StateKind::MinMaxKey: virt.push_back(fg.Bind(rt, OKeyInv(ct, v), cnt + " == 0")); break;
      default: throw Error(-5, "dense group-by cannot hold TEXT MIN/MAX");
    }
  }
  Scope sc;
  sc.virt = virt;
  for (size_t c = 0; c < op.output.size(); c++) {
    CVal v = fg.Emit(*op.output[c].expr, sc);
    std::string val = v.type.id == TypeId::BOOLEAN ? "(int8_t)(" + v.v + " ? 1 : 0)" : v.v;
    fk.L(optr[c] + "[r] = " + val + ";");
    if (!onull[c].empty()) fk.L(onull[c] + "[r] = (" + v.n + ") ? 1 : 0;");
  }
  fk.L(posp + "[r] = (uint64_t)r;");
  fk.Close();
  {
    std::string src = fk.Kernel("kdb_group_by_finalize", 1024);
    CUfunction f = ctx_.Kernel(src, "kdb_group_by_finalize");
    ctx_.Launch(f, 1, 1024, fk.Args(), 0, "group by finalize");
  }
  out.rows = ReadU64(ngroups);
  ctx_.CheckDeviceError("group by");
  out.pos_is_index = true;
  group_sorted_ = fuse_order;
  return out;
}

// GROUP BY over a hash join whose keys are all build-side columns and
// include the build key, with that key unique among the build rows (checked
// on the device): each build row then is its own group, so the matched build
// row's index is the group id and no group table is probed.  (The reference
// still hashes every joined row into its AggregateHashTable,
// compile/proxy/aggregate_hash_table.cc:187-243; the groups, their values
// and their first-insertion order are the same.)
bool Executor::BuildRowGroups(const Operator& op, std::vector<int>* key_cols) {
  const Operator& join = op.child();
  if (join.kind != OpKind::HASH_JOIN || op.group_by.empty() || !joins_.count(&join)) return false;
  const JoinTable& jt = joins_.at(&join);
  if (jt.build.rows <= 0 || jt.build.rows >= (int64_t(1) << 31)) return false;
  // first positions keep the probe row in 24 bits (see the group ordering)
  if (RowBound(join.child(1)) >= (int64_t(1) << 24)) return false;
  key_cols->clear();
  for (const auto& g : op.group_by) {
    if (g->kind != ExprKind::ColRef || g->child_idx != 0) return false;
    const Expr& src = *join.output.at(g->column_idx).expr;
    if (src.kind != ExprKind::ColRef || src.child_idx != 0) return false;
    key_cols->push_back(src.column_idx);
  }
  std::vector<int> bkeys;
  for (const auto& k : join.left_keys) {
    if (std::find(key_cols->begin(), key_cols->end(), k->column_idx) == key_cols->end()) return false;
    bkeys.push_back(k->column_idx);
  }
  // uniqueness of the build key: a key-in-slot table found duplicates while
  // it was built
  if (jt.key_in_slot && jt.dup && bkeys.size() == 1 && bkeys[0] == jt.key_col && !ctx_.OptStr("KDB_KEY_CHECK_PASS"))
    return ReadU64(jt.dup) == 0 || ctx_.dry;
  // otherwise every non-NULL build row must find itself only (rows with a
  // NULL key never join)
  uint64_t* dup = arena_.AllocT<uint64_t>(1);
  ctx_.Memset(dup, 0, sizeof(uint64_t));
  {
    KernelSource ks;
    ExprGen eg(ctx_, ks);
    std::string N = ks.Word(static_cast<uint64_t>(jt.build.rows)), D = ks.Ptr(dup, "unsigned long long");
    ks.Open("for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < (int64_t)" + N +
            "; r += (int64_t)gridDim.x * blockDim.x)");
    auto vals = LoadMatRow(ks, eg, jt.build, "r", nullptr);
    std::vector<CVal> keys;
    for (int c : bkeys) keys.push_back(vals.at(c));
    ks.L("int matches = 0;");
    EmitProbe(ks, eg, jt, bkeys, keys, [&](const std::vector<CVal>&, const std::string&) { ks.L("matches++;"); });
    ks.L("if (matches > 1) atomicOr(" + D + ", 1ULL);");
    ks.Close();
    LaunchPipeline(ks, jt.build.rows, "join key check");
  }
  return ReadU64(dup) == 0 || ctx_.dry;
}

MatBuffer Executor::RunGroupByBuildRows(const Operator& op, const std::vector<AggPlan>& plans,
                                        const std::vector<int>& key_cols, bool any_order) {
  const Operator& join = op.child();
  const JoinTable& jt = joins_.at(&join);
  const int64_t nb = jt.build.rows;
  const size_t nk = op.group_by.size();
  std::vector<char> counted(plans.size(), 1);  // per aggregate: NeedsCount, decided at emission
  uint64_t* first = arena_.AllocT<uint64_t>(nb);
  std::vector<uint64_t*> sv(plans.size()), sc(plans.size());
  for (size_t j = 0; j < plans.size(); j++) {
    sv[j] = arena_.AllocT<uint64_t>(nb);
    sc[j] = arena_.AllocT<uint64_t>(nb);
  }
  // initial states are byte patterns (all ones, or zero): memsets
  ctx_.Memset(first, 0xff, sizeof(uint64_t) * nb);
  for (size_t j = 0; j < plans.size(); j++) {
    const bool min_init = plans[j].kind == StateKind::MinMaxKey && plans[j].is_min;
    ctx_.Memset(sv[j], min_init ? 0xff : 0, sizeof(uint64_t) * nb);
    ctx_.Memset(sc[j], 0, sizeof(uint64_t) * nb);
  }
  // probe pipeline: aggregate into the matched build row
  std::vector<int> bkeys;
  for (const auto& k : join.left_keys) bkeys.push_back(k->column_idx);
  struct GroupPtrs {
    std::string F;
    std::vector<std::string> SV, SC;
  };
  auto group_ptrs = [&](KernelSource& ks) {
    GroupPtrs gp;
    gp.F = ks.Ptr(first, "uint64_t");
    for (size_t j = 0; j < plans.size(); j++) {
      gp.SV.push_back(ks.Ptr(sv[j], "uint64_t"));
      gp.SC.push_back(ks.Ptr(sc[j], "uint64_t"));
    }
    return gp;
  };
  // one joined row folded into the state of build row g
  auto fold = [&](KernelSource& ks, ExprGen& eg, const GroupPtrs& gp, const std::vector<CVal>& left,
                  const std::vector<CVal>& right, const std::string& pos, const std::string& g) {
    Scope s2;
    s2.child.push_back(left);
    s2.child.push_back(right);
    std::vector<CVal> joined;
    for (const auto& c : join.output) joined.push_back(eg.Emit(*c.expr, s2));
    Scope s3;
    s3.child.push_back(joined);
    std::string fl = "0ULL";
    for (size_t j = 0; j < plans.size(); j++) {
      CVal c = eg.Emit(plans[j].agg->kid(0), s3);
      if (plans[j].count_flag >= 0)
        fl += " | ((" + c.n + ") ? " + std::to_string(1 << plans[j].count_flag) + "ULL : 0ULL)";
      counted[j] = NeedsCount(plans[j], c);
      EmitGroupUpdate(ks, eg, plans[j], c, gp.SV[j], gp.SC[j], g, counted[j]);
    }
    // every row of the group matches the same build row: the first
    // position is the probe position alone (bits 40 and up)
    ks.L("kdb_atomic_min_u64(&" + gp.F + "[" + g + "], ((uint64_t)(" + pos + ") << 40) | (" + fl + "));");
  };
  const Operator& probe_op = join.child(1);
  const bool split = (probe_op.kind == OpKind::SCAN || probe_op.kind == OpKind::SCAN_SELECT) &&
                     ctx_.OptStr("KDB_SPLIT_PROBE_GROUPS") && !ctx_.OptStr("KDB_VECTOR_PROBE_SCAN") &&
                     !ctx_.OptStr("KDB_PROBE_AHEAD") && !ctx_.OptStr("KDB_PROBE_VEC") &&
                     !ctx_.OptStr("KDB_LAZY_PROBE_COLUMNS");
  if (split) {
    // KDB_SPLIT_PROBE_GROUPS: two kernels.  Measured on the Q3 shape it is
    // slower than the one fused kernel (probe 43 + aggregation 19 us against
    // 52 us): the probe stays bound by its dependent table accesses however
    // few bytes it streams.  The probe reads only the probe keys (and filter
    // columns), probes the table and writes each match as a (build row,
    // probe row) pair into its CTA's region of a pair buffer (a probe row
    // matches at most one build row: the build key is unique, so a CTA's
    // matches fit in the rows it scans); the aggregation then loads the
    // measure columns for the matched rows only and folds them into the
    // build rows.  Non-matching rows cost their key bytes alone.
    const int block = 256;
    const int64_t prow = std::max<int64_t>(ctx_.tables.at(probe_op.relation).rows, 1);
    const int G = ctx_.GridFor(prow, block);
    const int64_t per_cta = (prow + static_cast<int64_t>(G) * block - 1) / (static_cast<int64_t>(G) * block) * block;
    uint64_t* pairs = arena_.AllocT<uint64_t>(static_cast<int64_t>(G) * per_cta);
    uint32_t* pcount = arena_.AllocT<uint32_t>(G);
    // scan columns the probe needs: its filters' and its keys'
    std::set<int> key_cols_scan;
    std::function<void(const Expr&)> scan_refs = [&](const Expr& e) {
      if (e.kind == ExprKind::VirtColRef || e.kind == ExprKind::ColRef) key_cols_scan.insert(e.column_idx);
      for (const auto& k : e.kids) scan_refs(*k);
    };
    for (const auto& f : probe_op.filters) scan_refs(*f);
    std::function<void(const Expr&)> key_refs = [&](const Expr& e) {
      if (e.kind == ExprKind::ColRef && e.child_idx == 1) scan_refs(*probe_op.output.at(e.column_idx).expr);
      for (const auto& k : e.kids) key_refs(*k);
    };
    for (const auto& k : join.right_keys) key_refs(*k);
    {
      KernelSource ks;
      ExprGen eg(ctx_, ks);
      ks.pre << "  __shared__ unsigned kdb_block_rows;\n"
                "  if (threadIdx.x == 0) kdb_block_rows = 0;\n"
                "  __syncthreads();\n";
      const std::string P = ks.Ptr(pairs, "uint64_t"), PC = ks.Ptr(pcount, "uint32_t");
      const std::string RW = ks.Word(static_cast<uint64_t>(per_cta));
      const std::string ERR = ks.Ptr(ctx_.d_err, "int");
      int64_t src_rows = 0;
      auto body = [&](const std::vector<CVal>& right, const std::string& pos) {
        Scope s;
        s.child.resize(2);
        s.child[1] = right;
        std::vector<CVal> pk;
        for (const auto& k : join.right_keys) pk.push_back(eg.Emit(*k, s));
        EmitProbe(ks, eg, jt, bkeys, pk, [&](const std::vector<CVal>&, const std::string&) {
          ks.L("const uint32_t kdb_s = kdb_alloc_block_slot(&kdb_block_rows);");
          ks.L("if (kdb_s < (uint32_t)" + RW + ") " + P + "[(int64_t)blockIdx.x * (int64_t)" + RW +
               " + kdb_s] = ((uint64_t)(uint32_t)" + probe_br_ + " << 32) | (uint64_t)(uint32_t)(" + pos + ");");
          ks.L("else kdb_set_error(" + ERR + ", 1);");
        });
      };
      probe_side_scan_ = true;
      prefetch_only_ = &key_cols_scan;
      EmitStream(ks, eg, probe_op, body, src_rows);
      probe_side_scan_ = false;
      prefetch_only_ = nullptr;
      ks.L("__syncthreads();");
      ks.L("if (threadIdx.x == 0) " + PC + "[blockIdx.x] = kdb_block_rows < (unsigned)" + RW +
           " ? kdb_block_rows : (unsigned)" + RW + ";");
      LaunchPipeline(ks, src_rows, "join probe", block);
    }
    {
      KernelSource ks;
      ExprGen eg(ctx_, ks);
      GroupPtrs gp = group_ptrs(ks);
      const std::string P = ks.Ptr(pairs, "uint64_t", true), PC = ks.Ptr(pcount, "uint32_t", true);
      const std::string RW = ks.Word(static_cast<uint64_t>(per_cta)), GW = ks.Word(static_cast<uint64_t>(G));
      ks.Open("for (int64_t kdb_b = blockIdx.x; kdb_b < (int64_t)" + GW + "; kdb_b += gridDim.x)");
      ks.L("const uint32_t kdb_n = " + PC + "[kdb_b];");
      ks.Open("for (uint32_t kdb_i = threadIdx.x; kdb_i < kdb_n; kdb_i += blockDim.x)");
      ks.L("const uint64_t kdb_pr = " + P + "[kdb_b * (int64_t)" + RW + " + kdb_i];");
      ks.L("const int64_t r = (int64_t)(uint32_t)kdb_pr;");
      ks.L("const int64_t kdb_br = (int64_t)(kdb_pr >> 32);");
      std::vector<CVal> right = EmitScanRowAt(ks, eg, probe_op, "r");
      std::vector<CVal> left = LoadMatRow(ks, eg, jt.build, "kdb_br", nullptr);
      fold(ks, eg, gp, left, right, "(uint64_t)r", "kdb_br");
      ks.Close();
      ks.Close();
      LaunchPipeline(ks, static_cast<int64_t>(G) * block, "group by", block);
    }
  } else {
    KernelSource ks;
    ExprGen eg(ctx_, ks);
    GroupPtrs gp = group_ptrs(ks);
    int64_t src_rows = 0;
    auto body = [&](const std::vector<CVal>& right, const std::string& pos) {
      Scope s;
      s.child.resize(2);
      s.child[1] = right;
      std::vector<CVal> pk;
      for (const auto& k : join.right_keys) pk.push_back(eg.Emit(*k, s));
      EmitProbe(ks, eg, jt, bkeys, pk, [&](const std::vector<CVal>& left, const std::string&) {
        fold(ks, eg, gp, left, right, pos, probe_br_);
      });
    };
    // KDB_SMEM_BLOOM: every CTA (1024 threads, one per SM) first copies the
    // join filter (at most 2^20 bits) into shared memory, so a probe row the
    // filter rejects costs no L1/L2 access
    size_t sbloom = 0;
    if (ctx_.OptStr("KDB_SMEM_BLOOM") && jt.bloom && jt.bloom_log2 <= 20 && !ctx_.OptStr("KDB_PROBE_AHEAD") &&
        !ctx_.OptStr("KDB_PROBE_VEC")) {
      const size_t words = (size_t(1) << jt.bloom_log2) / 32;
      sbloom = words * sizeof(uint32_t);
      const std::string gb = ks.Ptr(jt.bloom, "uint4", true);
      ks.pre << "  extern __shared__ __align__(16) uint32_t kdb_sbloom[];\n"
             << "  for (int i = threadIdx.x; i < " << words / 4 << "; i += blockDim.x) reinterpret_cast<uint4*>(kdb_sbloom)[i] = "
             << gb << "[i];\n"
             << "  __syncthreads();\n";
      smem_bloom_ = "kdb_sbloom";
    }
    probe_side_scan_ = !ctx_.OptStr("KDB_VECTOR_PROBE_SCAN");
    if (probe_side_scan_) SetProbeAhead(join, jt);
    if (Streamable(join.child(1))) EmitStream(ks, eg, join.child(1), body, src_rows);
    else EmitMatScan(ks, mats_.at(&join.child(1)), nullptr, body, src_rows);
    probe_side_scan_ = false;
    ahead_jt_ = nullptr;
    ahead_probe_jt_ = nullptr;
    smem_bloom_.clear();
    if (sbloom) {
      const std::string src = ks.Kernel("kdb_group_by", 1024, 1);
      CUfunction f = ctx_.Kernel(src, "kdb_group_by");
      ctx_.Launch(f, ctx_.num_sms, 1024, ks.Args(), sbloom, "group by");
    } else {
      LaunchPipeline(ks, src_rows, "group by");
    }
  }
  ctx_.CheckDeviceError("group by");
  // groups = touched build rows, in first-insertion order
  uint64_t* keys = arena_.AllocT<uint64_t>(nb);
  uint32_t* vals = arena_.AllocT<uint32_t>(nb);
  uint64_t* ngroups = arena_.AllocT<uint64_t>(1);
  ctx_.Memset(ngroups, 0, sizeof(uint64_t));
  {
    KernelSource ks;
    std::string F = ks.Ptr(first, "uint64_t", true);
    std::string K = ks.Ptr(keys, "uint64_t"), V = ks.Ptr(vals, "uint32_t");
    std::string NG = ks.Ptr(ngroups, "unsigned long long");
    std::string C = ks.Word(static_cast<uint64_t>(nb));
    ks.Open("for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)" + C +
            "; i += (int64_t)gridDim.x * blockDim.x)");
    ks.L("const uint64_t f = " + F + "[i];");
    ks.Open("if (f != ~0ULL)");
    ks.L("uint64_t o = kdb_alloc_slot(" + NG + ");");
    // a probe row matches at most one (unique) build row, so groups'
    // first positions differ in their probe part: sort on it alone
    ks.L(K + "[o] = f >> 40; " + V + "[o] = (uint32_t)i;");
    ks.Close();
    ks.Close();
    LaunchPipeline(ks, nb, "group compact");
  }
  int64_t ng = ReadU64(ngroups);
  if (!any_order) ctx_.RadixSortPairs(keys, vals, ng, arena_, 24);
  MatBuffer out = AllocMat(op.output, ng);
  if (ng > 0) {
    KernelSource ks;
    ExprGen eg(ctx_, ks);
    std::string F = ks.Ptr(first, "uint64_t", true), V = ks.Ptr(vals, "uint32_t", true);
    std::string FK = any_order ? ks.Ptr(keys, "uint64_t", true) : "";
    std::string NGW = ks.Word(static_cast<uint64_t>(ng));
    std::vector<std::string> SV(plans.size()), SC(plans.size());
    for (size_t j = 0; j < plans.size(); j++) {
      SV[j] = ks.Ptr(sv[j], "uint64_t", true);
      SC[j] = ks.Ptr(sc[j], "uint64_t", true);
    }
    std::vector<std::string> optr, onull;
    for (const auto& c : out.cols) {
      optr.push_back(ks.Ptr(c.data, StoreType(c.type.id)));
      onull.push_back(c.nullable ? ks.Ptr(c.nulls, "int8_t") : "");
    }
    std::string posp = ks.Ptr(out.pos, "uint64_t");
    ks.Open("for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < (int64_t)" + NGW +
            "; r += (int64_t)gridDim.x * blockDim.x)");
    ks.L("uint64_t i = " + V + "[r];");
    ks.L("uint64_t fst = " + F + "[i];");
    auto bv = LoadMatRow(ks, eg, jt.build, "i", nullptr);
    std::vector<CVal> virt;
    for (size_t k = 0; k < nk; k++) {
      const CVal& c = bv.at(key_cols[k]);
      virt.push_back(eg.Bind(op.group_by[k]->type, c.v, c.n));
    }
    for (size_t j = 0; j < plans.size(); j++)
      virt.push_back(GroupResult(eg, plans[j], SV[j], SC[j], "i", "fst", counted[j] != 0));
    Scope sc;
    sc.virt = virt;
    for (size_t c = 0; c < op.output.size(); c++) {
      CVal v = eg.Emit(*op.output[c].expr, sc);
      std::string val = v.type.id == TypeId::BOOLEAN ? "(int8_t)(" + v.v + " ? 1 : 0)" : v.v;
      ks.L(optr[c] + "[r] = " + val + ";");
      if (!onull[c].empty()) ks.L(onull[c] + "[r] = (" + v.n + ") ? 1 : 0;");
    }
    ks.L(posp + "[r] = " + (any_order ? FK + "[r]" : std::string("(uint64_t)r")) + ";");
    ks.Close();
    LaunchPipeline(ks, ng, "group output");
  }
  out.rows = ng;
  out.pos_is_index = !any_order;
  return out;
}

MatBuffer Executor::RunGroupBy(const Operator& op, bool any_order, const Operator* order_by) {
  PrepareInput(op.child());
  int flags = 0;
  std::vector<AggPlan> plans;
  for (const auto& a : op.aggs) plans.push_back(PlanAgg(*a, flags));
  KeyLayout kl = PlanKeys(ctx_, op.group_by);
  const size_t nk = op.group_by.size();
  std::vector<char> counted(plans.size(), 1);  // per aggregate: NeedsCount, decided at emission
  {
    // small key domain: register pre-aggregation (no atomics) when the
    // per-thread state (groups x distinct accumulator words) stays small
    bool dense = kl.small_domain && kl.domain <= 32 && !op.group_by.empty();
    std::set<std::string> distinct;
    for (const auto& p : plans) {
      if (p.kind == StateKind::MinMaxText) dense = false;
      std::string csig = ExprSig(p.agg->kid(0));
      if (p.kind == StateKind::SumF64 || p.kind == StateKind::AvgF64) distinct.insert("f|" + csig);
      else if (p.kind == StateKind::SumI64) distinct.insert("i|" + csig);
      else if (p.kind == StateKind::MinMaxKey) distinct.insert((p.is_min ? "n|" : "x|") + csig);
      if (p.child_nullable) distinct.insert("c|" + csig);
    }
    int64_t words = static_cast<int64_t>(distinct.size()) + 2;
    if (dense && static_cast<int64_t>(kl.domain) * words <= 64 && !ctx_.OptStr("KDB_NO_DENSE_GROUPBY"))
      return RunGroupByDense(op, plans, kl, order_by);
  }

  {
    std::vector<int> key_cols;
    if (!ctx_.OptStr("KDB_NO_BUILD_ROW_GROUPS") && BuildRowGroups(op, &key_cols))
      return RunGroupByBuildRows(op, plans, key_cols, any_order);
  }

  // capacity: exact for small key domains; otherwise twice the input-row
  // bound capped at 2^20 slots (regrown on overflow)
  uint64_t cap = 1024;
  if (kl.small_domain) {
    while (cap < 2 * kl.domain) cap <<= 1;
  } else {
    uint64_t want = std::min<uint64_t>(2 * static_cast<uint64_t>(std::max<int64_t>(RowBound(op.child()), 1)),
                                       1ULL << 20);
    while (cap < want) cap <<= 1;
  }
  for (int attempt = 0; attempt < 8; attempt++) {
    const auto mark = ctx_.RecordMark();
    uint64_t mask = cap - 1;
    uint64_t* slots = arena_.AllocT<uint64_t>(cap);
    uint64_t* first = arena_.AllocT<uint64_t>(cap);
    std::vector<uint64_t*> kw(nk), sv(plans.size()), sc(plans.size());
    std::vector<int32_t*> klen(nk);
    std::vector<int8_t*> kn(nk);
    if (!kl.packed)
      for (size_t k = 0; k < nk; k++) {
        kw[k] = arena_.AllocT<uint64_t>(cap);
        klen[k] = arena_.AllocT<int32_t>(cap);
        kn[k] = arena_.AllocT<int8_t>(cap);
      }
    for (size_t j = 0; j < plans.size(); j++) {
      sv[j] = arena_.AllocT<uint64_t>(cap);
      sc[j] = arena_.AllocT<uint64_t>(cap);
    }
    // init kernel
    {
      KernelSource ks;
      std::string S = ks.Ptr(slots, "uint64_t"), F = ks.Ptr(first, "uint64_t");
      std::string C = ks.Word(cap);
      ks.Open("for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)" + C +
              "; i += (int64_t)gridDim.x * blockDim.x)");
      ks.L(S + "[i] = 0; " + F + "[i] = ~0ULL;");
      for (size_t j = 0; j < plans.size(); j++) {
        std::string V = ks.Ptr(sv[j], "uint64_t"), N = ks.Ptr(sc[j], "uint64_t");
        bool min_init = plans[j].kind == StateKind::MinMaxKey && plans[j].is_min;
        ks.L(V + "[i] = " + (min_init ? "~0ULL" : "0ULL") + "; " + N + "[i] = 0;");
      }
      ks.Close();
      LaunchPipeline(ks, static_cast<int64_t>(cap), "group init");
    }
    // aggregation pipeline
    {
      KernelSource ks;
      ExprGen eg(ctx_, ks);
      std::string S = ks.Ptr(slots, "uint64_t"), F = ks.Ptr(first, "uint64_t");
      std::string M = "(uint64_t)" + ks.Word(mask);
      std::string ERR = ks.Ptr(ctx_.d_err, "int");
      std::vector<std::string> KW(nk), KL(nk), KN(nk), SV(plans.size()), SC(plans.size());
      if (!kl.packed)
        for (size_t k = 0; k < nk; k++) {
          KW[k] = ks.Ptr(kw[k], "uint64_t");
          KL[k] = ks.Ptr(klen[k], "int32_t");
          KN[k] = ks.Ptr(kn[k], "int8_t");
        }
      for (size_t j = 0; j < plans.size(); j++) {
        SV[j] = ks.Ptr(sv[j], "uint64_t");
        SC[j] = ks.Ptr(sc[j], "uint64_t");
      }
      int64_t src_rows = 0;
      auto consume = [&](const std::vector<CVal>& in, const std::string& pos) {
        Scope s;
        s.child.push_back(in);
        std::vector<CVal> keys;
        for (const auto& g : op.group_by) keys.push_back(eg.Emit(*g, s));
        std::string g = ks.Fresh("g");
        if (kl.packed) {
          std::string pk = "0x8000000000000000ULL";
          for (size_t k = 0; k < nk; k++) {
            const CVal& c = keys[k];
            std::string bits;
            switch (c.type.id) {
              case TypeId::REAL: bits = "kdb_dbits(" + c.v + ")"; break;
              case TypeId::BOOLEAN: bits = "(uint64_t)(" + c.v + " ? 1 : 0)"; break;
              case TypeId::SMALLINT: bits = "(uint64_t)(uint16_t)" + c.v; break;
              case TypeId::BIGINT: bits = "(uint64_t)" + c.v; break;
              default: bits = "(uint64_t)(uint32_t)" + c.v; break;
            }
            uint64_t m = kl.width[k] >= 64 ? ~0ULL : ((1ULL << kl.width[k]) - 1);
            std::string field = "((" + c.n + ") ? 0ULL : ((" + bits + ") & " + std::to_string(m) + "ULL))";
            pk += " | (" + field + " << " + std::to_string(kl.offset[k]) + ")";
            if (kl.nullable[k])
              pk += " | ((" + c.n + ") ? (1ULL << " + std::to_string(kl.offset[k] + kl.width[k]) + ") : 0ULL)";
          }
          ks.L("int64_t " + g + " = kdb_group_find_packed(" + S + ", " + M + ", " + pk + ", " + ERR + ");");
        } else {
          std::string h = "0x2545f4914f6cdd1dULL";
          for (size_t k = 0; k < nk; k++)
            h = "kdb_hash_combine(" + h + ", (" + keys[k].n + ") ? 0x9e3779b97f4a7c15ULL : " + eg.HashOf(keys[k]) + ")";
          std::string eq = "true", init;
          for (size_t k = 0; k < nk; k++) {
            const CVal& c = keys[k];
            std::string stored_null = "(__ldcg(&" + KN[k] + "[i]) != 0)";
            std::string w = "__ldcg((const unsigned long long*)&" + KW[k] + "[i])";
            std::string veq;
            switch (c.type.id) {
              case TypeId::TEXT:
                veq = "kdb_str_eq(kdb_mkstr((const char*)" + w + ", __ldcg(&" + KL[k] + "[i])), " + c.v + ")";
                init += KW[k] + "[i] = (uint64_t)" + c.v + ".p; " + KL[k] + "[i] = " + c.v + ".len; ";
                break;
              case TypeId::REAL:
                veq = "(__longlong_as_double((long long)" + w + ") == " + c.v + ")";
                init += KW[k] + "[i] = (uint64_t)__double_as_longlong(" + c.v + "); ";
                break;
              case TypeId::BOOLEAN:
                veq = "((" + w + " != 0) == " + c.v + ")";
                init += KW[k] + "[i] = " + c.v + " ? 1ULL : 0ULL; ";
                break;
              default:
                veq = "((int64_t)" + w + " == (int64_t)" + c.v + ")";
                init += KW[k] + "[i] = (uint64_t)(int64_t)" + c.v + "; ";
                break;
            }
            init += KN[k] + "[i] = (" + c.n + ") ? 1 : 0; ";
            eq += " && (" + stored_null + " == (" + c.n + ")) && ((" + c.n + ") || " + veq + ")";
          }
          ks.L("int64_t " + g + " = kdb_group_find(" + S + ", " + M + ", (" + h +
               ") | 0x8000000000000000ULL, [&](uint64_t i) { return " + eq + "; }, [&](uint64_t i) { " + init +
               "}, " + ERR + ");");
        }
        ks.Open("if (" + g + " >= 0)");
        std::string fl = "0ULL";
        for (size_t j = 0; j < plans.size(); j++) {
          CVal c = eg.Emit(plans[j].agg->kid(0), s);
          if (plans[j].count_flag >= 0)
            fl += " | ((" + c.n + ") ? " + std::to_string(1 << plans[j].count_flag) + "ULL : 0ULL)";
          counted[j] = NeedsCount(plans[j], c);
          EmitGroupUpdate(ks, eg, plans[j], c, SV[j], SC[j], g, counted[j]);
        }
        ks.L("kdb_atomic_min_u64(&" + F + "[" + g + "], ((uint64_t)(" + pos + ") << 8) | (" + fl + "));");
        ks.Close();
      };
      if (Streamable(op.child())) EmitStream(ks, eg, op.child(), consume, src_rows);
      else EmitMatScan(ks, mats_.at(&op.child()), nullptr, consume, src_rows);
      LaunchPipeline(ks, src_rows, "group by");
    }
    try {
      ctx_.CheckDeviceError("group by");
    } catch (const Error& e) {
      if (e.code == -4 && !kl.small_domain) {
        cap <<= 3;
        ctx_.RecordTruncate(mark);
        continue;
      }
      throw;
    }
    // compact occupied slots: (first position, slot)
    uint64_t* keys = arena_.AllocT<uint64_t>(cap);
    uint32_t* vals = arena_.AllocT<uint32_t>(cap);
    uint64_t* ngroups = arena_.AllocT<uint64_t>(1);
    ctx_.Memset(ngroups, 0, sizeof(uint64_t));
    {
      KernelSource ks;
      std::string S = ks.Ptr(slots, "uint64_t", true), F = ks.Ptr(first, "uint64_t", true);
      std::string K = ks.Ptr(keys, "uint64_t"), V = ks.Ptr(vals, "uint32_t");
      std::string NG = ks.Ptr(ngroups, "unsigned long long");
      std::string C = ks.Word(cap);
      ks.Open("for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)" + C +
              "; i += (int64_t)gridDim.x * blockDim.x)");
      ks.Open("if (" + S + "[i] >= 2)");
      ks.L("uint64_t o = kdb_alloc_slot(" + NG + ");");
      ks.L(K + "[o] = " + F + "[i]; " + V + "[o] = (uint32_t)i;");
      ks.Close();
      ks.Close();
      LaunchPipeline(ks, static_cast<int64_t>(cap), "group compact");
    }
    int64_t ng = ReadU64(ngroups);
    if (!any_order) ctx_.RadixSortPairs(keys, vals, ng, arena_, 64);
    // output kernel
    MatBuffer out = AllocMat(op.output, ng);
    if (ng > 0) {
      KernelSource ks;
      ExprGen eg(ctx_, ks);
      std::string S = ks.Ptr(slots, "uint64_t", true), F = ks.Ptr(first, "uint64_t", true);
      std::string V = ks.Ptr(vals, "uint32_t", true);
      std::string FK = any_order ? ks.Ptr(keys, "uint64_t", true) : "";
      std::string NGW = ks.Word(static_cast<uint64_t>(ng));
      std::vector<std::string> KW(nk), KL(nk), KN(nk), SV(plans.size()), SC(plans.size());
      if (!kl.packed)
        for (size_t k = 0; k < nk; k++) {
          KW[k] = ks.Ptr(kw[k], "uint64_t", true);
          KL[k] = ks.Ptr(klen[k], "int32_t", true);
          KN[k] = ks.Ptr(kn[k], "int8_t", true);
        }
      for (size_t j = 0; j < plans.size(); j++) {
        SV[j] = ks.Ptr(sv[j], "uint64_t", true);
        SC[j] = ks.Ptr(sc[j], "uint64_t", true);
      }
      std::vector<std::string> optr, onull;
      for (const auto& c : out.cols) {
        optr.push_back(ks.Ptr(c.data, StoreType(c.type.id)));
        onull.push_back(c.nullable ? ks.Ptr(c.nulls, "int8_t") : "");
      }
      std::string posp = ks.Ptr(out.pos, "uint64_t");
      ks.Open("for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < (int64_t)" + NGW +
              "; r += (int64_t)gridDim.x * blockDim.x)");
      ks.L("uint64_t i = " + V + "[r];");
      ks.L("uint64_t fst = " + F + "[i];");
      std::vector<CVal> virt;
      for (size_t k = 0; k < nk; k++) {
        const Type& t = op.group_by[k]->type;
        if (kl.packed) {
          uint64_t m = kl.width[k] >= 64 ? ~0ULL : ((1ULL << kl.width[k]) - 1);
          std::string bits = "((" + S + "[i] >> " + std::to_string(kl.offset[k]) + ") & " + std::to_string(m) + "ULL)";
          std::string v;
          switch (t.id) {
            case TypeId::REAL: v = "__longlong_as_double((long long)" + bits + ")"; break;
            case TypeId::BOOLEAN: v = "(" + bits + " != 0)"; break;
            case TypeId::SMALLINT: v = "(int16_t)(uint16_t)" + bits; break;
            case TypeId::BIGINT: v = "(int64_t)" + bits; break;
            default: v = "(int32_t)(uint32_t)" + bits; break;
          }
          std::string n = kl.nullable[k]
                              ? "(((" + S + "[i] >> " + std::to_string(kl.offset[k] + kl.width[k]) + ") & 1ULL) != 0)"
                              : "false";
          virt.push_back(eg.Bind(t, v, n));
        } else {
          std::string w = KW[k] + "[i]";
          std::string v;
          switch (t.id) {
            case TypeId::TEXT: v = "kdb_mkstr((const char*)" + w + ", " + KL[k] + "[i])"; break;
            case TypeId::REAL: v = "__longlong_as_double((long long)" + w + ")"; break;
            case TypeId::BOOLEAN: v = "(" + w + " != 0)"; break;
            default: v = "(" + CType(t.id) + ")(int64_t)" + w; break;
          }
          virt.push_back(eg.Bind(t, v, "(" + KN[k] + "[i] != 0)"));
        }
      }
      for (size_t j = 0; j < plans.size(); j++)
        virt.push_back(GroupResult(eg, plans[j], SV[j], SC[j], "i", "fst", counted[j] != 0));
      Scope s;
      s.virt = virt;
      for (size_t c = 0; c < op.output.size(); c++) {
        CVal v = eg.Emit(*op.output[c].expr, s);
        std::string val = v.type.id == TypeId::BOOLEAN ? "(int8_t)(" + v.v + " ? 1 : 0)" : v.v;
        ks.L(optr[c] + "[r] = " + val + ";");
        if (!onull[c].empty()) ks.L(onull[c] + "[r] = (" + v.n + ") ? 1 : 0;");
      }
      ks.L(posp + "[r] = " + (any_order ? FK + "[r]" : std::string("(uint64_t)r")) + ";");
      ks.Close();
      LaunchPipeline(ks, ng, "group output");
    }
    ctx_.CheckDeviceError("group output");
    out.rows = ng;
    out.pos_is_index = !any_order;
    return out;
  }
  throw Error(-4, "group table did not fit");
}

// ---------------------------------------------------------------------------
// Order-by (order_by_translator.cc:35-110): materialise the child, then
// stable radix passes -- stream order, the reference merge sort's tie key,
// then every sort key from the least significant (NULL flag after value so
// NULL sorts last ascending, LessThan in evaluate.cc:339-402).
// ---------------------------------------------------------------------------

MatBuffer Executor::RunOrderBy(const Operator& op) {
  // every ORDER BY path below orders rows that are not in stream order by
  // their stream position, so a GROUP BY child need not sort its groups
  group_sorted_ = false;
  MatBuffer m = op.child().kind == OpKind::GROUP_BY_AGGREGATE && !ctx_.OptStr("KDB_GROUP_ORDER_SORT")
                    ? RunGroupBy(op.child(), true, ctx_.OptStr("KDB_NO_GROUP_ORDER_FUSE") ? nullptr : &op)
                    : Materialize(op.child());
  if (group_sorted_) {
    // the dense GROUP BY wrote its groups in this ORDER BY's order; an
    // output schema that passes every column through in place needs no
    // further work
    group_sorted_ = false;
    bool identity = op.output.size() == m.cols.size();
    for (size_t c = 0; identity && c < op.output.size(); c++) {
      const Expr& e = *op.output[c].expr;
      identity = e.kind == ExprKind::ColRef && e.child_idx == 0 && e.column_idx == static_cast<int>(c);
    }
    if (identity) return m;
    uint32_t* idx = arena_.AllocT<uint32_t>(std::max<int64_t>(m.rows, 1));
    if (m.rows > 0) {
      KernelSource ks;
      std::string I = ks.Ptr(idx, "uint32_t");
      std::string N = ks.Word(static_cast<uint64_t>(m.rows));
      ks.Open("for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)" + N +
              "; i += (int64_t)gridDim.x * blockDim.x)");
      ks.L(I + "[i] = (uint32_t)i;");
      ks.Close();
      LaunchPipeline(ks, m.rows, "order rows");
    }
    return MaterializeStream(op, idx, &m);
  }
  int64_t n = m.rows;
  if (n <= kSmallOrder) return SmallOrderBy(op, m);
  return LargeOrderBy(op, m);
}

// ORDER BY of at most kSmallOrder rows in one block: every row's final rank
// is the number of rows that compare before it under the generated
// comparator (sort keys, then the reference merge sort's tie key of the
// row's stream index), so one launch replaces the radix passes.
MatBuffer Executor::SmallOrderBy(const Operator& op, MatBuffer& m) {
  int64_t n = m.rows;
  uint32_t* idx = arena_.AllocT<uint32_t>(std::max<int64_t>(n, 1));
  if (n > 0) {
    KernelSource ks;
    ExprGen eg(ctx_, ks);
    std::string P = ks.Ptr(m.pos, "uint64_t", true);
    std::string I = ks.Ptr(idx, "uint32_t");
    std::string N = "nrows";
    ks.L("__shared__ uint32_t sidx[" + std::to_string(kSmallOrder) + "];");
    ks.L("const int64_t nrows = (int64_t)" + ks.Word(static_cast<uint64_t>(n)) + ";");
    ks.Open("for (int64_t i = threadIdx.x; i < " + N + "; i += blockDim.x)");
    ks.L("uint64_t p = " + P + "[i]; uint32_t c = 0;");
    ks.L("for (int64_t j = 0; j < " + N + "; j++) c += " + P + "[j] < p;");
    ks.L("sidx[i] = c;");
    ks.Close();
    ks.L("__syncthreads();");
    // comparator over the materialised key columns
    std::string less = "auto less = [&](int64_t ra, int64_t rb) -> bool {\n";
    for (size_t k = 0; k < op.sort_keys.size(); k++) {
      const MatCol& mc = m.cols.at(op.sort_keys[k]->column_idx);
      if (mc.type.id == TypeId::BOOLEAN) throw Error(-1, "Can't be less than.");
      std::string D = ks.Ptr(mc.data, StoreType(mc.type.id), true);
      std::string NP = mc.nullable ? ks.Ptr(mc.nulls, "int8_t", true) : "";
      std::string na = NP.empty() ? "false" : "(" + NP + "[ra] != 0)";
      std::string nb = NP.empty() ? "false" : "(" + NP + "[rb] != 0)";
      std::string ab, ba;
      switch (mc.type.id) {
        case TypeId::TEXT:
          ab = "(kdb_str_cmp(" + D + "[ra], " + D + "[rb]) < 0)";
          ba = "(kdb_str_cmp(" + D + "[rb], " + D + "[ra]) < 0)";
          break;
        case TypeId::ENUM:
          ab = "(" + eg.EnumRank(mc.type, D + "[ra]") + " < " + eg.EnumRank(mc.type, D + "[rb]") + ")";
          ba = "(" + eg.EnumRank(mc.type, D + "[rb]") + " < " + eg.EnumRank(mc.type, D + "[ra]") + ")";
          break;
        default:
          ab = "(" + D + "[ra] < " + D + "[rb])";
          ba = "(" + D + "[rb] < " + D + "[ra])";
          break;
      }
      // proxy::LessThan: NULL sorts after every value
      std::string lt_ab = "(!" + na + " && (" + nb + " || " + ab + "))";
      std::string lt_ba = "(!" + nb + " && (" + na + " || " + ba + "))";
      bool asc = op.asc[k];
      less += "    if " + lt_ab + " return " + (asc ? "true" : "false") + ";\n";
      less += "    if " + lt_ba + " return " + (asc ? "false" : "true") + ";\n";
    }
    less += "    return kdb_tie_path(sidx[ra], " + N + ") < kdb_tie_path(sidx[rb], " + N + ");\n  };";
    ks.L(less);
    ks.Open("for (int64_t i = threadIdx.x; i < " + N + "; i += blockDim.x)");
    ks.L("uint32_t r = 0;");
    ks.L("for (int64_t j = 0; j < " + N + "; j++) r += (j != i) && less(j, i);");
    ks.L(I + "[r] = (uint32_t)i;");
    ks.Close();
    std::string src = ks.Kernel("kdb_order_by_small", 1024);
    CUfunction f = ctx_.Kernel(src, "kdb_order_by_small");
    ctx_.Launch(f, 1, 1024, ks.Args(), 0, "order by small");
  }
  return MaterializeStream(op, idx, &m);
}

// (key, tie) order of 16-byte items: the range-bucket sort (16384
// equal-width key buckets, each item ranked within its bucket), falling
// back to the block sort plus merge passes when a bucket holds more than
// 1024 items (many equal keys); KDB_ORDER_MERGE forces the merge passes and
// KDB_ORDER_SAMPLE a sample sort (splitters from a sorted sample).  On the
// 134k-item ORDER BY of the Q3-shape query the query steps at 228 us with
// the range sort against 241 us with the merge passes (198 / 211 us with
// Zipf keys); the sample sort was slower than both.
bool Executor::SortItems(uint64_t* items, int64_t n, unsigned long long* ties, uint32_t tie_mask,
                         const unsigned long long* key_range) {
  if (ctx_.OptStr("KDB_ORDER_SAMPLE") && ctx_.SampleSortItems(items, n, arena_)) return false;
  if (!ctx_.OptStr("KDB_ORDER_MERGE") && !ctx_.OptStr("KDB_ORDER_SAMPLE") &&
      ctx_.RangeSortItems(items, n, arena_, ctx_.OptStr("KDB_ORDER_TIE_PASS") ? nullptr : ties, tie_mask,
                          KeyRangeWanted() ? key_range : nullptr))
    return ties != nullptr && !ctx_.OptStr("KDB_ORDER_TIE_PASS");
  ctx_.MergeSortItems(items, n, arena_);
  return false;
}

MatBuffer Executor::LargeOrderBy(const Operator& op, MatBuffer& m) {
  int64_t n = m.rows;
  uint64_t* keys = arena_.AllocT<uint64_t>(std::max<int64_t>(n, 1));
  uint32_t* idx = arena_.AllocT<uint32_t>(std::max<int64_t>(n, 1));
  auto keygen = [&](const std::function<std::string(KernelSource&, ExprGen&, const std::string&)>& body) {
    KernelSource ks;
    ExprGen eg(ctx_, ks);
    std::string K = ks.Ptr(keys, "uint64_t");
    std::string I = ks.Ptr(idx, "uint32_t");
    std::string N = ks.Word(static_cast<uint64_t>(n));
    ks.Open("for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)" + N +
            "; i += (int64_t)gridDim.x * blockDim.x)");
    std::string expr = body(ks, eg, I);
    ks.L(K + "[i] = " + expr + ";");
    ks.Close();
    LaunchPipeline(ks, n, "order key");
  };
  if (n > 1) {
    // stream order (skipped when the rows already are in it)
    auto stream_order = [&]() {
      if (m.pos_is_index) {
        keygen([&](KernelSource& ks, ExprGen&, const std::string& I) {
          ks.L(I + "[i] = (uint32_t)i;");
          return std::string("0ULL");
        });
      } else {
        keygen([&](KernelSource& ks, ExprGen&, const std::string& I) {
          std::string P = ks.Ptr(m.pos, "uint64_t", true);
          ks.L(I + "[i] = (uint32_t)i;");
          return P + "[i]";
        });
        ctx_.RadixSortPairs(keys, idx, n, arena_, 64);
      }
    };
    // the tie key uses at most depth = ceil(log2 n) + 1 leading bits
    int depth = 1;
    while ((1LL << (depth - 1)) < n) depth++;
    // One numeric key: (key, tie rank) pairs are unique, so a block sort
    // plus merge-path passes over 16-byte items orders them in a few
    // launches (the radix path needs two launches per 8-bit digit).  A
    // nullable key folds its NULL flag in as the most significant bit: the
    // key's low bit moves to the top of the tie word, which then holds the
    // tie rank in 31 bits.
    const MatCol* mk = op.sort_keys.size() == 1 ? &m.cols.at(op.sort_keys[0]->column_idx) : nullptr;
    const bool merge_ok = mk && depth <= 32 && !ctx_.OptStr("KDB_ORDER_RADIX") && mk->type.id != TypeId::TEXT &&
                          mk->type.id != TypeId::BOOLEAN && (!mk->nullable || depth <= 31);
    if (merge_ok) {
      const MatCol& mc = *mk;
      const TypeId t = mc.type.id;
      uint64_t* items = arena_.AllocT<uint64_t>(2 * n);
      // stream_ties: rows in stream order (idx) with the reference merge
      // sort's tie rank; otherwise rows in buffer order with the row index
      // as a provisional (unique) tie
      // the items' key range, reduced while they are made (the range-bucket
      // sort then needs no pass of its own for it)
      unsigned long long* key_range = KeyRangeWanted() ? arena_.AllocT<unsigned long long>(2) : nullptr;
      auto make_items = [&](bool stream_ties) {
        KernelSource ks;
        ExprGen eg(ctx_, ks);
        std::string IT = ks.Ptr(items, "uint64_t"), I = ks.Ptr(idx, "uint32_t", true);
        std::string D = ks.Ptr(mc.data, StoreType(t), true);
        std::string N = ks.Word(static_cast<uint64_t>(n));
        std::string KR;
        if (key_range) {
          ctx_.Memset(key_range, 0xff, sizeof(unsigned long long));
          ctx_.Memset(key_range + 1, 0, sizeof(unsigned long long));
          KR = ks.Ptr(key_range, "unsigned long long");
          ks.L("unsigned long long kdb_klo = ~0ULL, kdb_khi = 0ULL;");
        }
        ks.Open("for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)" + N +
                "; i += (int64_t)gridDim.x * blockDim.x)");
        ks.L(std::string("const uint32_t row = ") + (m.pos_is_index || !stream_ties ? "(uint32_t)i" : I + "[i]") +
             ";");
        std::string v = D + "[row]", norm;
        switch (t) {
          case TypeId::REAL: norm = "kdb_dord(" + v + ")"; break;
          case TypeId::ENUM: norm = "(uint64_t)(uint32_t)" + eg.EnumRank(mc.type, v); break;
          default: norm = "((uint64_t)(int64_t)" + v + " ^ 0x8000000000000000ULL)"; break;
        }
        const std::string tie = stream_ties ? "(kdb_tie_path((uint64_t)i, " + std::to_string(n) + "ULL) >> " +
                                                  std::to_string(64 - depth) + ")"
                                            : std::string("(uint64_t)row");
        if (!mc.nullable) {
          ks.L(IT + "[2 * i] = " + (op.asc[0] ? "" : "~") + "(" + norm + ");");
          ks.L(IT + "[2 * i + 1] = " + tie + " | ((uint64_t)row << 32);");
        } else {
          // NULLs sort after every value ascending, before them descending
          // (proxy::LessThan), and tie among themselves
          std::string NP = ks.Ptr(mc.nulls, "int8_t", true);
          ks.L("const bool isnull = " + NP + "[row] != 0;");
          ks.L("const uint64_t k = isnull ? 0ULL : " + std::string(op.asc[0] ? "" : "~") + "(" + norm + ");");
          ks.L(std::string("const uint64_t flag = ") + (op.asc[0] ? "isnull" : "!isnull") + " ? 1ULL : 0ULL;");
          ks.L(IT + "[2 * i] = (flag << 63) | (k >> 1);");
          ks.L(IT + "[2 * i + 1] = ((k & 1ULL) << 31) | " + tie + " | ((uint64_t)row << 32);");
        }
        if (key_range) {
          ks.L("{ const unsigned long long kk = " + IT + "[2 * i]; kdb_klo = kk < kdb_klo ? kk : kdb_klo; "
               "kdb_khi = kk > kdb_khi ? kk : kdb_khi; }");
        }
        ks.Close();
        if (key_range) {
          ks.L("for (int o = 16; o > 0; o >>= 1) { const unsigned long long a = __shfl_xor_sync(0xffffffffu, kdb_klo, o), "
               "b = __shfl_xor_sync(0xffffffffu, kdb_khi, o); kdb_klo = a < kdb_klo ? a : kdb_klo; "
               "kdb_khi = b > kdb_khi ? b : kdb_khi; }");
          ks.L("if ((threadIdx.x & 31) == 0 && kdb_klo <= kdb_khi) { atomicMin(&" + KR + "[0], kdb_klo); atomicMax(&" + KR +
               "[1], kdb_khi); }");
        }
        LaunchPipeline(ks, n, "order key");
      };
      auto order_rows = [&]() {
        KernelSource ks;
        std::string IT = ks.Ptr(items, "uint64_t", true), I = ks.Ptr(idx, "uint32_t");
        std::string N = ks.Word(static_cast<uint64_t>(n));
        ks.Open("for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)" + N +
                "; i += (int64_t)gridDim.x * blockDim.x)");
        ks.L(I + "[i] = (uint32_t)(" + IT + "[2 * i + 1] >> 32);");
        ks.Close();
        LaunchPipeline(ks, n, "order rows");
      };
      // the output in sorted order, its rows read from the items' high words
      // (KDB_ORDER_ROWS_PASS: through a separate row-index array)
      auto sorted_output = [&]() {
        if (ctx_.OptStr("KDB_ORDER_ROWS_PASS")) {
          order_rows();
          return MaterializeStream(op, idx, &m);
        }
        order_items_ = items;
        MatBuffer out = MaterializeStream(op, idx, &m);
        order_items_ = nullptr;
        return out;
      };
      if (!m.pos_is_index && !ctx_.OptStr("KDB_ORDER_TIE_SORT")) {
        // Rows not in stream order (groups in table order): sort by the key
        // alone and look for equal neighbours.  Without ties the tie rank
        // never decides, and the stream-order sort is not needed.
        make_items(false);
        uint64_t* ties = arena_.AllocT<uint64_t>(1);
        ctx_.Memset(ties, 0, sizeof(uint64_t));
        // the range sort counts ties while it ranks (equal keys share a
        // bucket); after the other sorts a pass compares neighbours
        if (!SortItems(items, n, reinterpret_cast<unsigned long long*>(ties), mc.nullable ? 0x80000000u : 0u,
                       key_range)) {
          KernelSource ks;
          std::string IT = ks.Ptr(items, "uint64_t", true), T = ks.Ptr(ties, "unsigned long long");
          std::string N = ks.Word(static_cast<uint64_t>(n));
          ks.Open("for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i + 1 < (int64_t)" + N +
                  "; i += (int64_t)gridDim.x * blockDim.x)");
          std::string eq = IT + "[2 * i] == " + IT + "[2 * i + 2]";
          if (mc.nullable) eq += " && ((" + IT + "[2 * i + 1] ^ " + IT + "[2 * i + 3]) & 0x80000000ULL) == 0";
          ks.L("if (" + eq + ") atomicAdd(" + T + ", 1ULL);");
          ks.Close();
          LaunchPipeline(ks, n, "order ties");
        }
        if (ReadU64(ties) == 0 && !ctx_.dry) return sorted_output();
      }
      stream_order();
      make_items(true);
      SortItems(items, n, nullptr, 0, key_range);
      return sorted_output();
    }
    stream_order();
    auto tie_sort = [&]() {
      keygen([&](KernelSource&, ExprGen&, const std::string&) {
        return "(kdb_tie_path((uint64_t)i, " + std::to_string(n) + "ULL) >> " + std::to_string(64 - depth) + ")";
      });
      ctx_.RadixSortPairs(keys, idx, n, arena_, depth);
    };
    auto key_sorts = [&]() {
      const auto& child_schema = SchemaOf(op.child());
      for (int k = static_cast<int>(op.sort_keys.size()) - 1; k >= 0; k--) {
        int col = op.sort_keys[k]->column_idx;
        const MatCol& mc = m.cols.at(col);
        bool asc = op.asc[k];
        (void)child_schema;
        const std::string inv = asc ? "" : "~";
        auto load = [&](KernelSource& ks, ExprGen& eg, const std::string& I) {
          std::string D = ks.Ptr(mc.data, StoreType(mc.type.id), true);
          return std::make_pair(D + "[" + I + "[i]]", std::string());
        };
        // NULLs compare equal among themselves: their key is a constant (the
        // NULL pass below then moves them last), so they keep tie order
        auto guard = [&](KernelSource& ks, const std::string& I, const std::string& key) {
          if (!mc.nullable) return key;
          return "((" + ks.Ptr(mc.nulls, "int8_t", true) + "[" + I + "[i]] != 0) ? 0ULL : (uint64_t)(" + key + "))";
        };
        if (mc.type.id == TypeId::BOOLEAN) throw Error(-1, "Can't be less than.");
        if (mc.type.id == TypeId::TEXT) {
          // max length over the rows decides the number of 8-byte chunks
          uint64_t* mx = arena_.AllocT<uint64_t>(1);
          ctx_.Memset(mx, 0, sizeof(uint64_t));
          {
            KernelSource ks;
            std::string D = ks.Ptr(mc.data, "kdb_str", true), MX = ks.Ptr(mx, "unsigned long long");
            std::string N = ks.Word(static_cast<uint64_t>(n));
            ks.Open("for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)" + N +
                    "; i += (int64_t)gridDim.x * blockDim.x)");
            ks.L("atomicMax(" + MX + ", (unsigned long long)" + D + "[i].len);");
            ks.Close();
            LaunchPipeline(ks, n, "text max len");
          }
          int64_t maxlen = ReadU64(mx);
          keygen([&](KernelSource& ks, ExprGen& eg, const std::string& I) {
            return guard(ks, I, inv + "(uint64_t)" + load(ks, eg, I).first + ".len");
          });
          ctx_.RadixSortPairs(keys, idx, n, arena_, 64);
          for (int64_t c = (maxlen + 7) / 8 - 1; c >= 0; c--) {
            keygen([&](KernelSource& ks, ExprGen& eg, const std::string& I) {
              return guard(ks, I, inv + "kdb_str_chunk(" + load(ks, eg, I).first + ", " + std::to_string(c) + ")");
            });
            ctx_.RadixSortPairs(keys, idx, n, arena_, 64);
          }
        } else {
          keygen([&](KernelSource& ks, ExprGen& eg, const std::string& I) {
            std::string v = load(ks, eg, I).first;
            std::string norm;
            switch (mc.type.id) {
              case TypeId::REAL: norm = "kdb_dord(" + v + ")"; break;
              case TypeId::ENUM: norm = "(uint64_t)(uint32_t)" + eg.EnumRank(mc.type, v); break;
              default: norm = "((uint64_t)(int64_t)" + v + " ^ 0x8000000000000000ULL)"; break;
            }
            return guard(ks, I, inv + "(" + norm + ")");
          });
          ctx_.RadixSortPairs(keys, idx, n, arena_, 64);
        }
        if (mc.nullable) {
          keygen([&](KernelSource& ks, ExprGen&, const std::string& I) {
            std::string NP = ks.Ptr(mc.nulls, "int8_t", true);
            std::string isnull = "(uint64_t)(" + NP + "[" + I + "[i]] != 0)";
            return asc ? isnull : "(1ULL - " + isnull + ")";
          });
          ctx_.RadixSortPairs(keys, idx, n, arena_, 8);
        }
      }
    };
    // Float sort keys rarely tie: sort the stream-ordered rows by the keys
    // alone and check adjacent rows for ties; only if two rows tie is the
    // merge sort's tie order (the tie-path key) needed, and the sort is
    // redone with it from the stream order.
    bool floats_only = !ctx_.OptStr("KDB_ORDER_TIE_SORT");
    for (const auto& sk : op.sort_keys)
      if (m.cols.at(sk->column_idx).type.id != TypeId::REAL) floats_only = false;
    bool done = false;
    if (floats_only) {
      uint32_t* stream_rows = nullptr;  // the stream order, when it is not the identity
      if (!m.pos_is_index) {
        stream_rows = arena_.AllocT<uint32_t>(n);
        KernelSource ks;
        std::string I = ks.Ptr(idx, "uint32_t", true), SR = ks.Ptr(stream_rows, "uint32_t");
        std::string N = ks.Word(static_cast<uint64_t>(n));
        ks.Open("for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)" + N +
                "; i += (int64_t)gridDim.x * blockDim.x)");
        ks.L(SR + "[i] = " + I + "[i];");
        ks.Close();
        LaunchPipeline(ks, n, "order stream copy");
      }
      key_sorts();
      uint64_t* ties = arena_.AllocT<uint64_t>(1);
      ctx_.Memset(ties, 0, sizeof(uint64_t));
      {
        KernelSource ks;
        std::string I = ks.Ptr(idx, "uint32_t", true), T = ks.Ptr(ties, "unsigned long long");
        std::string N = ks.Word(static_cast<uint64_t>(n));
        ks.Open("for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i + 1 < (int64_t)" + N +
                "; i += (int64_t)gridDim.x * blockDim.x)");
        ks.L("const uint32_t ra = " + I + "[i], rb = " + I + "[i + 1];");
        ks.L("bool eq = true;");
        for (const auto& sk : op.sort_keys) {
          const MatCol& mc = m.cols.at(sk->column_idx);
          std::string D = ks.Ptr(mc.data, "double", true);
          if (mc.nullable) {
            std::string NP = ks.Ptr(mc.nulls, "int8_t", true);
            ks.L("{ const bool na = " + NP + "[ra] != 0, nb = " + NP + "[rb] != 0; eq = eq && na == nb && (na || kdb_dord(" +
                 D + "[ra]) == kdb_dord(" + D + "[rb])); }");
          } else {
            ks.L("eq = eq && kdb_dord(" + D + "[ra]) == kdb_dord(" + D + "[rb]);");
          }
        }
        ks.L("if (eq) atomicAdd(" + T + ", 1ULL);");
        ks.Close();
        LaunchPipeline(ks, n, "order ties");
      }
      if (ReadU64(ties) == 0 && !ctx_.dry) {
        done = true;
      } else {
        keygen([&](KernelSource& ks, ExprGen&, const std::string& I) {  // back to stream order
          if (stream_rows) ks.L(I + "[i] = " + ks.Ptr(stream_rows, "uint32_t", true) + "[i];");
          else ks.L(I + "[i] = (uint32_t)i;");
          return std::string("0ULL");
        });
      }
    }
    if (!done) {
      tie_sort();
      key_sorts();
    }
  } else if (n == 1) {
    ctx_.Memset(idx, 0, sizeof(uint32_t));
  }
  return MaterializeStream(op, idx, &m);
}

// ---------------------------------------------------------------------------
// Result download (runtime/printer.cc formats it on the host)
// ---------------------------------------------------------------------------


// ---------------------------------------------------------------------------
// Skinner join: adaptive join ordering by UCT over budgeted episodes
// (permutable_skinner_join_translator.cc:82-994,
//  runtime/skinner_join_executor.cc:34-879).
//
// Reference: each table gets a generated "table function"; the executor's
// UCT agent picks a join order per episode, runs it for a fixed step budget
// and resumes it later from a progress tree, deduplicating result tuples in a
// TupleIdxTable.  Here: one generated kernel whose join order is a runtime
// argument (like the reference's permutable variant, no recompilation per
// order) runs an episode as an index-nested-loop over a slice of the leftmost
// table; the slice is sized so the episode's work (tuples examined) matches
// the budget.  Exactly-once emission without a dedup table: every table t
// keeps an offset (tuples of t fully processed while t was leftmost), and
// every later episode skips those tuples of t in any position, so each result
// combination is produced by the first episode whose leftmost slice covers
// one of its tuples.  The join is complete when one table's offset reaches its
// cardinality.  The UCT search below restates UctNode/UctJoinAgent
// (skinner_join_executor.cc:559-838): exploration weight 1e-5, untried
// actions first, connected-table heuristic below the root, random connected
// playout; reward = 0.5 * progress + 0.5 * results / budget
// (JoinEnvironment::Reward, :252-274).
// ---------------------------------------------------------------------------

class JoinEnv {
 public:
  virtual ~JoinEnv() = default;
  virtual bool IsConnected(const std::set<int>& joined, int table) = 0;
  virtual bool IsComplete() = 0;
  virtual double Execute(const std::vector<int>& order) = 0;
  // Learned prior: predicted episode reward of appending each of `cands`
  // to the tables in `joined` (a bit mask).
  virtual bool HasPrior() const { return false; }
  virtual void PriorValues(uint64_t joined, const std::vector<int>& cands, std::vector<double>& out) {
    out.assign(cands.size(), 0.0);
  }
};

class UctNode {
 public:
  UctNode(int round, int num_tables, JoinEnv& env, const std::vector<int>& already_joined, uint32_t seed)
      : env_(env), created_in_(round), num_tables_(num_tables),
        num_actions_(num_tables - static_cast<int>(already_joined.size())), children_(num_actions_),
        tries_(num_actions_, 0), reward_(num_actions_, 0.0), table_of_action_(num_actions_), rng_(seed) {
    for (int a = 0; a < num_actions_; a++) {
      priority_.push_back(a);
      recommended_.insert(a);
    }
    joined_.insert(already_joined.begin(), already_joined.end());
    int a = 0;
    for (int t = 0; t < num_tables_; t++)
      if (!joined_.count(t)) {
        unjoined_.push_back(t);
        table_of_action_[a++] = t;
      }
    InitPrior();
  }

  UctNode(int round, UctNode& parent, int joined_table, uint32_t seed)
      : env_(parent.env_), created_in_(round), num_tables_(parent.num_tables_),
        num_actions_(parent.num_actions_ - 1), children_(num_actions_), tries_(num_actions_, 0),
        reward_(num_actions_, 0.0), joined_(parent.joined_), unjoined_(parent.unjoined_),
        table_of_action_(num_actions_), rng_(seed) {
    joined_.insert(joined_table);
    unjoined_.erase(std::find(unjoined_.begin(), unjoined_.end(), joined_table));
    for (int a = 0; a < num_actions_; a++) table_of_action_[a] = unjoined_[a];
    // connected-table heuristic (skinner_join_executor.cc:617-630)
    for (int a = 0; a < num_actions_; a++)
      if (env_.IsConnected(joined_, table_of_action_[a])) recommended_.insert(a);
    if (recommended_.empty())
      for (int a = 0; a < num_actions_; a++) recommended_.insert(a);
    for (int a = 0; a < num_actions_; a++)
      if (recommended_.count(a)) priority_.push_back(a);
    InitPrior();
  }

  // One episode of the search (select, expand, playout, back-propagate).
  // With `trail`, every (node, action) whose statistics the sample updated
  // is recorded: an episode that runs later in a batch reports its reward
  // as a placeholder, and Correct() adds the difference to the true reward
  // along exactly that path once the batch has run, leaving the statistics
  // as if the true reward had been back-propagated.
  double Sample(int round, std::vector<int>& order, std::vector<std::pair<UctNode*, int>>* trail = nullptr) {
    if (num_actions_ == 0) return env_.Execute(order);
    int action = SelectAction();
    int table = table_of_action_[action];
    order[joined_.size()] = table;
    if (created_in_ != round && !children_[action])
      children_[action] = std::make_unique<UctNode>(round, *this, table, static_cast<uint32_t>(rng_()));
    UctNode* child = children_[action].get();
    double reward = child ? child->Sample(round, order, trail) : Playout(order);
    visits_++;
    tries_[action]++;
    reward_[action] += reward;
    if (trail) trail->emplace_back(this, action);
    return reward;
  }

  static void Correct(const std::vector<std::pair<UctNode*, int>>& trail, double delta) {
    for (const auto& [node, action] : trail) node->reward_[action] += delta;
  }

 private:
  // With a learned prior every action starts as tried once with the
  // predicted reward: the search begins at the prior's choice and the
  // observed rewards overrule it (UCT has the last word).
  void InitPrior() {
    if (!env_.HasPrior() || num_actions_ == 0) return;
    std::vector<double> v;
    env_.PriorValues(Mask(joined_), table_of_action_, v);
    priority_.clear();
    for (int a = 0; a < num_actions_; a++) {
      tries_[a] = 1;
      reward_[a] = v[a];
    }
    visits_ = num_actions_;
  }

  static uint64_t Mask(const std::set<int>& s) {
    uint64_t m = 0;
    for (int t : s) m |= 1ULL << t;
    return m;
  }

  double Playout(std::vector<int>& order) {
    int last = order[joined_.size()];
    std::set<int> cur(joined_.begin(), joined_.end());
    cur.insert(last);
    std::vector<int> rest;
    for (int t = 0; t < num_tables_; t++)
      if (!joined_.count(t) && t != last) rest.push_back(t);
    if (env_.HasPrior()) {  // greedy continuation by the prior among connected tables
      for (int pos = static_cast<int>(joined_.size()) + 1; pos < num_tables_; pos++) {
        std::vector<int> cands;
        for (int t : rest)
          if (!cur.count(t)) cands.push_back(t);
        std::vector<double> v;
        env_.PriorValues(Mask(cur), cands, v);
        int pick = -1;
        double best = -1e300;
        for (int pass = 0; pass < 2 && pick < 0; pass++)
          for (size_t i = 0; i < cands.size(); i++)
            if ((pass == 1 || env_.IsConnected(cur, cands[i])) && v[i] > best) {
              best = v[i];
              pick = cands[i];
            }
        order[pos] = pick;
        cur.insert(pick);
      }
      return env_.Execute(order);
    }
    std::shuffle(rest.begin(), rest.end(), rng_);
    for (int pos = static_cast<int>(joined_.size()) + 1; pos < num_tables_; pos++) {
      int pick = -1;
      for (int t : rest)
        if (!cur.count(t) && env_.IsConnected(cur, t)) {
          pick = t;
          break;
        }
      if (pick < 0)
        for (int t : rest)
          if (!cur.count(t)) {
            pick = t;
            break;
          }
      order[pos] = pick;
      cur.insert(pick);
    }
    return env_.Execute(order);
  }

  int SelectAction() {
    if (!priority_.empty()) {
      int idx = static_cast<int>(rng_() % priority_.size());
      int action = priority_[idx];
      priority_.erase(priority_.begin() + idx);
      return action;
    }
    int offset = static_cast<int>(rng_() % num_actions_);
    int best = -1;
    double best_q = -1;
    for (int i = 0; i < num_actions_; i++) {
      int a = (offset + i) % num_actions_;
      if (!recommended_.count(a)) continue;
      double q = reward_[a] / tries_[a] + kExploration * std::sqrt(std::log(visits_) / tries_[a]);
      if (q > best_q) {
        best = a;
        best_q = q;
      }
    }
    return best;
  }

  static constexpr double kExploration = 1e-5;
  JoinEnv& env_;
  int created_in_, num_tables_, num_actions_;
  std::vector<int> priority_;
  std::vector<std::unique_ptr<UctNode>> children_;
  int visits_ = 0;
  std::vector<int> tries_;
  std::vector<double> reward_;
  std::set<int> joined_;
  std::set<int> recommended_;
  std::vector<int> unjoined_;
  std::vector<int> table_of_action_;
  std::default_random_engine rng_;
};

struct SkinnerPred {  // equality between two children's columns
  int cond;
  int ta, ca, tb, cb;
};

class SkinnerEngine : public JoinEnv {
 public:
  SkinnerEngine(Context& ctx, Arena& arena, const Operator& op, std::vector<const MatBuffer*> mats,
                std::vector<std::vector<JoinTable>> index_for, const std::vector<SkinnerPred>& preds,
                std::function<MatBuffer(int64_t)> alloc_out, int64_t budget, uint32_t seed,
                const SkinnerAgg* agg = nullptr)
      : ctx_(ctx), arena_(arena), op_(op), mats_(std::move(mats)), preds_(preds),
        alloc_out_(std::move(alloc_out)), budget_(budget), seed_(seed), agg_(agg) {
    T_ = static_cast<int>(mats_.size());
    for (const MatBuffer* m : mats_) cards_.push_back(m->rows);
    offsets_.assign(T_, 0);
    // first slice of each leftmost table: a share of the budget (later
    // slices are sized from the measured work per leftmost tuple)
    slice_est_.assign(T_, std::max<int64_t>(1, std::min<int64_t>(budget_ / 64, 65536)));
    // tables each condition references
    std::function<void(const Expr&, uint64_t&)> collect = [&](const Expr& e, uint64_t& m) {
      if (e.kind == ExprKind::ColRef) m |= 1ULL << e.child_idx;
      for (const auto& k : e.kids) collect(*k, m);
    };
    for (const auto& c : op_.conditions) {
      uint64_t m = 0;
      collect(*c, m);
      cond_tables_.push_back(m);
    }
    adj_.assign(T_, 0);
    for (const auto& pr : preds_) {
      connected_.insert({pr.ta, pr.tb});
      connected_.insert({pr.tb, pr.ta});
      adj_[pr.ta] |= 1ULL << pr.tb;
      adj_[pr.tb] |= 1ULL << pr.ta;
    }
    index_for_ = std::move(index_for);
  }

  bool HasPrior() const override {
    return ctx_.skinner_policy == 1 && ctx_.join_prior != nullptr && T_ <= kPriorTables;
  }

  // The prior's value of every (joined set, next table) pair of the join,
  // in one forward pass (at most 8 tables: 2^7 * 8 = 1024 rows), so the
  // search never waits on a forward pass of its own.
  void PrecomputePrior() {
    if (!HasPrior() || ctx_.dry) return;
    std::vector<uint64_t> masks;
    std::vector<int> cand;
    const uint64_t full = (T_ >= 64) ? ~0ULL : ((1ULL << T_) - 1);
    for (uint64_t m = 0; m < full; m++)
      for (int t = 0; t < T_; t++)
        if (!(m >> t & 1ULL)) {
          masks.push_back(m);
          cand.push_back(t);
        }
    std::vector<float> x(masks.size() * JoinPrior::kIn), y(masks.size());
    for (size_t i = 0; i < masks.size(); i++) Features(masks[i], cand[i], &x[i * JoinPrior::kIn]);
    constexpr int64_t kChunk = 4096;  // rows per forward call
    for (size_t b = 0; b < masks.size(); b += kChunk) {
      const int64_t rows = std::min<int64_t>(kChunk, static_cast<int64_t>(masks.size() - b));
      ctx_.join_prior->Forward(x.data() + b * JoinPrior::kIn, rows, y.data() + b);
    }
    for (size_t i = 0; i < masks.size(); i++) {
      auto& v = prior_cache_[masks[i]];
      if (v.empty()) v.assign(T_, 0.0);
      v[cand[i]] = y[i];
    }
  }

  void PriorValues(uint64_t joined, const std::vector<int>& cands, std::vector<double>& out) override {
    auto it = prior_cache_.find(joined);
    if (it == prior_cache_.end()) {
      // one forward pass for every table not yet joined
      std::vector<int> all;
      for (int t = 0; t < T_; t++)
        if (!(joined >> t & 1ULL)) all.push_back(t);
      std::vector<float> x(all.size() * JoinPrior::kIn), y(all.size());
      for (size_t i = 0; i < all.size(); i++) Features(joined, all[i], &x[i * JoinPrior::kIn]);
      if (!all.empty() && !ctx_.dry) ctx_.join_prior->Forward(x.data(), static_cast<int64_t>(all.size()), y.data());
      std::vector<double> v(T_, 0.0);
      for (size_t i = 0; i < all.size(); i++) v[all[i]] = y[i];
      it = prior_cache_.emplace(joined, std::move(v)).first;
    }
    out.resize(cands.size());
    for (size_t i = 0; i < cands.size(); i++) out[i] = it->second[cands[i]];
  }

  // Features of appending table `cand` to the tables in `joined`: per table
  // slot (6 each, 8 slots) presence, log cardinality after the table's
  // filters, joined, candidate, linked to the joined set, linked to the
  // candidate; then candidate-centred summaries.  Only the join graph and
  // the cardinalities enter, so a (joined set, candidate) pair always maps
  // to the same vector.
  void Features(uint64_t joined, int cand, float* f) const {
    std::fill(f, f + JoinPrior::kIn, 0.f);
    auto lrows = [&](int t) { return static_cast<float>(std::log2(1.0 + static_cast<double>(cards_[t])) / 24.0); };
    auto linked = [&](int t, uint64_t set) { return (adj_[t] & set) != 0; };
    const uint64_t cand_bit = 1ULL << cand;
    int njoined = 0;
    for (int t = 0; t < T_ && t < kPriorTables; t++) {
      float* g = f + 6 * t;
      const bool in = joined >> t & 1ULL;
      njoined += in;
      g[0] = 1.f;
      g[1] = lrows(t);
      g[2] = in ? 1.f : 0.f;
      g[3] = t == cand ? 1.f : 0.f;
      g[4] = linked(t, joined) ? 1.f : 0.f;
      g[5] = linked(t, cand_bit) ? 1.f : 0.f;
    }
    float min_other = 0.f, max_other = 0.f, min_joined = 0.f;
    int smaller = 0, nb_unjoined = 0, nb_joined = 0;
    bool any_other = false, any_joined = false;
    for (int t = 0; t < T_; t++) {
      if (t == cand) continue;
      const float l = lrows(t);
      if (joined >> t & 1ULL) {
        min_joined = any_joined ? std::min(min_joined, l) : l;
        any_joined = true;
        nb_joined += (adj_[cand] >> t) & 1ULL;
      } else {
        min_other = any_other ? std::min(min_other, l) : l;
        max_other = any_other ? std::max(max_other, l) : l;
        any_other = true;
        smaller += cards_[t] < cards_[cand];
        nb_unjoined += (adj_[cand] >> t) & 1ULL;
      }
    }
    f[48] = njoined / 8.f;
    f[49] = T_ / 8.f;
    f[50] = lrows(cand);
    f[51] = linked(cand, joined) ? 1.f : 0.f;
    f[52] = min_other;
    f[53] = smaller / 8.f;
    f[54] = nb_unjoined / 8.f;
    f[55] = nb_joined / 8.f;
    f[56] = max_other;
    f[57] = min_joined;
  }

  int64_t work() const { return total_work_; }

  bool IsConnected(const std::set<int>& joined, int table) override {
    for (int t : joined)
      if (connected_.count({t, table})) return true;
    return false;
  }
  bool IsComplete() override {
    for (int t = 0; t < T_; t++)
      if (offsets_[t] >= cards_[t]) return true;
    return false;
  }

  MatBuffer Run(const std::vector<int>& prefix) {
    if (agg_) {
      out_ = MatBuffer();
      out_.cap = std::numeric_limits<int64_t>::max();
    } else {
      out_ = alloc_out_(1 << 12);
    }
    // result count, work, the two task queues' counts, then per episode of
    // a batch its results and its work (all read back together)
    stats_ = arena_.AllocT<uint64_t>(4 + 2 * kMaxBatch);
    ctx_.Memset(stats_, 0, (4 + 2 * kMaxBatch) * sizeof(uint64_t));
    count_ = stats_;
    work_ = stats_ + 1;
    tcount_ = stats_ + 2;
    eres_ = stats_ + 4;
    ework_ = stats_ + 4 + kMaxBatch;
    ep_ = arena_.AllocT<uint64_t>(static_cast<size_t>(kMaxBatch) * EpWords());
    // episodes per batch: the next join orders are chosen before the
    // current ones' rewards are known (their placeholders corrected after),
    // so a batch's episodes share each launch and host round trip
    batch_ = 8;
    if (const char* b = ctx_.OptStr("KDB_SKINNER_BATCH")) batch_ = std::atoi(b);
    batch_ = std::max(1, std::min(batch_, kMaxBatch));
    produced_ = 0;
    bool empty = false;
    for (int64_t c : cards_) empty |= c == 0;
    if (!empty) {
      beg_ = arena_.AllocT<uint64_t>(kMaxSlice);
      offs_ = arena_.AllocT<uint64_t>(kMaxSlice + 1);
      deep_ = T_ > 2 && !ctx_.OptStr("KDB_SKINNER_DEPTH1");
      if (deep_) {
        beg2_ = arena_.AllocT<uint64_t>(kMaxItems2);
        offs2_ = arena_.AllocT<uint64_t>(kMaxItems2 + 1);
      }
      split_ = T_ > 2 && !ctx_.OptStr("KDB_SKINNER_NO_SPLIT");
      if (const char* r = ctx_.OptStr("KDB_SKINNER_SPLIT")) split_run_ = std::max<int64_t>(1, std::atoll(r));
      if (const char* c = ctx_.OptStr("KDB_SKINNER_TASKS")) task_cap_ = std::max<int64_t>(1, std::atoll(c));
      if (split_)
        for (int q = 0; q < 2; q++) tasks_[q] = arena_.AllocT<uint64_t>(task_cap_ * (4 + T_));
      Generate();
      std::vector<int> order(T_);
      for (size_t i = 0; i < prefix.size(); i++) order[i] = prefix[i];
      const int64_t max_episodes = ctx_.dry ? 1 : (1 << 24);
      // a batch fills until it holds batch_ episodes, the join completes
      // (an offset reaches its table's end) or its slices fill kMaxSlice
      auto batch_open = [&]() {
        return static_cast<int>(pending_.size()) < batch_ && !IsComplete() &&
               episodes_ + static_cast<int64_t>(pending_.size()) < max_episodes && batch_items_ < kMaxSlice;
      };
      if (ctx_.skinner_policy == 2) {
        // uniformly random connected orders (training data for the prior)
        std::mt19937_64 rng(seed_);
        batching_ = true;
        while (!IsComplete() && episodes_ < max_episodes) {
         while (batch_open()) {
          uint64_t in = 0;
          for (size_t i = 0; i < prefix.size(); i++) in |= 1ULL << prefix[i];
          for (int pos = static_cast<int>(prefix.size()); pos < T_; pos++) {
            std::vector<int> linked, any;
            for (int t = 0; t < T_; t++)
              if (!(in >> t & 1ULL)) {
                any.push_back(t);
                if (adj_[t] & in) linked.push_back(t);
              }
            const std::vector<int>& from = linked.empty() ? any : linked;
            order[pos] = from[rng() % from.size()];
            in |= 1ULL << order[pos];
          }
          Execute(order);
         }
         RunBatch();
        }
        batching_ = false;
      } else {
        PrecomputePrior();
        UctNode root(0, T_, *this, prefix, seed_);
        int round = 0;
        std::vector<std::vector<std::pair<UctNode*, int>>> trails;
        std::vector<double> placeholders;
        batching_ = true;
        while (!IsComplete() && episodes_ < max_episodes) {
          trails.clear();
          placeholders.clear();
          while (batch_open()) {
            round++;
            trails.emplace_back();
            root.Sample(round, order, &trails.back());
            placeholders.push_back(pending_.back().placeholder);
          }
          RunBatch();
          for (size_t k = 0; k < trails.size(); k++)
            UctNode::Correct(trails[k], last_rewards_[k] - placeholders[k]);
        }
        batching_ = false;
      }
      LogSamples(prefix.size());
    }
    out_.rows = produced_;
    return out_;
  }

  // (features, reward) of every choice of every episode, for training the
  // prior
  void LogSamples(size_t prefix_len) {
    ctx_.skinner_features.clear();
    ctx_.skinner_rewards.clear();
    if (!ctx_.skinner_log || T_ > kPriorTables) return;
    constexpr size_t kMaxSamples = 1 << 16;
    for (const auto& [order, reward] : log_) {
      uint64_t in = 0;
      for (size_t d = 0; d < prefix_len; d++) in |= 1ULL << order[d];
      for (int d = static_cast<int>(prefix_len); d + 1 < T_; d++) {
        if (ctx_.skinner_rewards.size() >= kMaxSamples) return;
        const size_t base = ctx_.skinner_features.size();
        ctx_.skinner_features.resize(base + JoinPrior::kIn);
        Features(in, order[d], &ctx_.skinner_features[base]);
        ctx_.skinner_rewards.push_back(static_cast<float>(reward));
        in |= 1ULL << order[d];
      }
    }
  }

  int64_t episodes() const { return episodes_; }

  // An episode's join order and slice, decided when it is chosen: its
  // leftmost table's slice starts at that table's offset, which moves past
  // the slice at once, so the episodes of one batch take consecutive slices
  // and each sees the offsets the earlier ones leave -- exactly the state a
  // one-at-a-time run would give it.  Results therefore stay exactly-once
  // however many episodes run together.
  struct Pending {
    std::vector<int> order;
    int L = 0;
    int64_t s0 = 0, s1 = 0, remaining = 0;
    std::vector<int64_t> off;
    double placeholder = 0;
  };

  double Execute(const std::vector<int>& order) override {
    Pending p;
    p.order = order;
    p.L = order[0];
    p.remaining = cards_[p.L] - offsets_[p.L];
    const int64_t room = std::max<int64_t>(1, kMaxSlice - batch_items_);
    const int64_t len = std::max<int64_t>(1, std::min<int64_t>({slice_est_[p.L], p.remaining, room}));
    p.s0 = offsets_[p.L];
    p.s1 = p.s0 + len;
    p.off = offsets_;
    offsets_[p.L] = p.s1;
    batch_items_ += len;
    p.placeholder = rewards_seen_ ? reward_sum_ / rewards_seen_ : 0.0;
    pending_.push_back(std::move(p));
    if (batching_) return pending_.back().placeholder;
    RunBatch();
    return last_rewards_[0];
  }

  // Runs the pending episodes together: one set of launches for the whole
  // batch, each item finding its episode's parameters in a small block the
  // host writes first.
  void RunBatch() {
    const int nb = static_cast<int>(pending_.size());
    if (nb == 0) return;
    const int W = EpWords();
    std::vector<uint64_t> ep(static_cast<size_t>(nb) * W, 0);
    int64_t start = 0;
    for (int e = 0; e < nb; e++) {
      const Pending& pe = pending_[e];
      uint64_t* q = ep.data() + static_cast<size_t>(e) * W;
      std::vector<int> pos_of(T_);
      for (int p = 0; p < T_; p++) pos_of[pe.order[p]] = p;
      uint64_t bound = 0;
      for (int p = 0; p < T_; p++) {
        int t = pe.order[p];
        int lk = -1;
        int used_pred = -1;
        if (p > 0)
          for (size_t j = 0; j < preds_.size() && lk < 0; j++) {
            const SkinnerPred& pr = preds_[j];
            if (pr.tb == t && (bound >> pr.ta & 1ULL)) {
              lk = static_cast<int>(j) * 2;
              used_pred = pr.cond;
            } else if (pr.ta == t && (bound >> pr.tb & 1ULL)) {
              lk = static_cast<int>(j) * 2 + 1;
              used_pred = pr.cond;
            }
          }
        uint64_t after = bound | (1ULL << t);
        uint64_t sched = 0;
        for (size_t c = 0; c < cond_tables_.size(); c++) {
          uint64_t m = cond_tables_[c];
          bool ready_now = (m & ~after) == 0 && (p == 0 ? true : (m & ~bound) != 0);
          if (p == 0 && m == 0) ready_now = true;  // constant conditions at the first table
          if (ready_now && static_cast<int>(c) != used_pred) sched |= 1ULL << c;
        }
        bound = after;
        q[p] = static_cast<uint64_t>(t);
        q[T_ + p] = static_cast<uint64_t>(static_cast<int64_t>(lk));
        q[2 * T_ + p] = sched;
      }
      for (int t = 0; t < T_; t++) q[3 * T_ + t] = static_cast<uint64_t>(pe.off[t]);
      q[4 * T_] = static_cast<uint64_t>(pe.s0);
      q[4 * T_ + 1] = static_cast<uint64_t>(pe.s1);
      q[4 * T_ + 2] = static_cast<uint64_t>(start);
      start += pe.s1 - pe.s0;
    }
    const int64_t S = start;
    ctx_.H2D(ep_, ep.data(), sizeof(uint64_t) * ep.size());
    KArgs a = args_;
    a.w[w_nep_] = static_cast<uint64_t>(nb);
    a.w[w_total_] = static_cast<uint64_t>(S);
    const int K = kMaxBatch;
    std::vector<uint64_t> st(4 + 2 * K, 0);
    for (int attempt = 0; attempt < 8; attempt++) {
      a.w[w_cap_] = static_cast<uint64_t>(out_.cap);
      PatchOut(a);
      a.w[w_phase_] = 0;
      ctx_.Launch(fn_, ctx_.GridFor(S, 128), 128, a, 0, T_ > 1 ? "skinner expand" : "skinner episode");
      if (T_ > 1) {
        ctx_.ScanU64(offs_, S);
        if (deep_) {
          // position-1 items expand their position-2 runs (or, past
          // kMaxItems2 items, run depth-first as below); then every
          // position-2 candidate is an item of its own
          a.w[w_phase_] = 2;
          ctx_.Launch(fn_, ctx_.num_sms * 8, 128, a, 0, "skinner expand2");
          ctx_.ScanU64Bounded(offs2_, offs_ + S, kMaxItems2);
          a.w[w_phase_] = 3;
          ctx_.Launch(fn_, ctx_.num_sms * 8, 128, a, 0, "skinner episode");
        } else {
          a.w[w_phase_] = 1;
          ctx_.Launch(fn_, ctx_.num_sms * 8, 128, a, 0, "skinner episode");
        }
      }
      ctx_.D2H(st.data(), stats_, sizeof(uint64_t) * st.size());
      if (split_ && st[2] > 0 && !ctx_.dry) {
        // queued hot runs: each round's tasks sit one position deeper than
        // the previous round's, so at most T rounds
        int qi = 0;
        uint64_t pending = st[2];
        for (int round = 0; pending > 0; round++) {
          if (round > T_) throw Error(-5, "skinner task rounds did not converge");
          a.w[w_phase_] = 4;
          a.w[w_qin_] = static_cast<uint64_t>(qi);
          ctx_.Launch(fn_, ctx_.num_sms * 8, 128, a, 0, "skinner tasks");
          ctx_.Memset(tcount_ + qi, 0, sizeof(uint64_t));
          qi = 1 - qi;
          ctx_.D2H(&pending, tcount_ + qi, sizeof(uint64_t));
        }
        ctx_.D2H(st.data(), stats_, sizeof(uint64_t) * st.size());
      }
      ctx_.CheckDeviceError("skinner episode");
      int64_t total = static_cast<int64_t>(st[0]);
      if (total <= out_.cap || ctx_.dry) {
        produced_ = ctx_.dry ? 0 : total;
        break;
      }
      Grow(total);  // the batch reruns into the larger buffer
      uint64_t keep = static_cast<uint64_t>(produced_);
      ctx_.H2D(count_, &keep, sizeof(uint64_t));
      ctx_.Memset(work_, 0, sizeof(uint64_t));
      ctx_.Memset(eres_, 0, sizeof(uint64_t) * 2 * K);
    }
    ctx_.Memset(work_, 0, sizeof(uint64_t));
    ctx_.Memset(eres_, 0, sizeof(uint64_t) * 2 * K);
    // per episode: reward, and the next slice size of its leftmost table
    // so its work matches the budget
    last_rewards_.assign(nb, 0.0);
    std::vector<int64_t> lwork(T_, 0), llen(T_, 0);
    for (int e = 0; e < nb; e++) {
      const Pending& pe = pending_[e];
      const int64_t len = pe.s1 - pe.s0;
      const int64_t results = static_cast<int64_t>(st[4 + e]);
      const int64_t work = static_cast<int64_t>(st[4 + K + e]);
      lwork[pe.L] += work;
      llen[pe.L] += len;
      const double progress = static_cast<double>(len) / static_cast<double>(pe.remaining);
      const double reward = 0.5 * progress + 0.5 * static_cast<double>(results) / static_cast<double>(budget_);
      last_rewards_[e] = reward;
      reward_sum_ += reward;
      rewards_seen_++;
      total_work_ += work;
      if (ctx_.skinner_log && log_.size() < (1u << 16)) log_.emplace_back(pe.order, reward);
    }
    for (int t = 0; t < T_; t++)
      if (llen[t]) {
        const double per_row = static_cast<double>(std::max<int64_t>(lwork[t], 1)) / llen[t];
        slice_est_[t] = std::max<int64_t>(1, std::min<int64_t>(int64_t(budget_ / per_row), 1LL << 26));
      }
    episodes_ += nb;
    batches_++;
    pending_.clear();
    batch_items_ = 0;
  }

  int64_t batches() const { return batches_; }

 private:
  // Generates the episode kernel once; per-episode values are patched into
  // reserved argument words.
  void Generate() {
    KernelSource ks;
    ExprGen eg(ctx_, ks);
    const int T = T_;
    // per-episode parameters of the batch (host-written block, EPW words
    // per episode): order, lookup, condition schedule, offsets, s0, s1,
    // first item index
    const std::string EP = ks.Ptr(ep_, "uint64_t", true);
    const std::string EPW = std::to_string(EpWords());
    w_nep_ = ks.Arg(0);
    w_total_ = ks.Arg(0);
    w_cap_ = ks.Arg(0);
    std::string TS = std::to_string(T);
    const std::string KB = std::to_string(kMaxBatch);
    ks.L("int32_t ord[" + TS + "]; int32_t lk[" + TS + "]; uint64_t sched[" + TS + "]; int64_t off[" + TS + "];");
    ks.L("int64_t card[" + TS + "];");
    for (int t = 0; t < T; t++) ks.L("card[" + std::to_string(t) + "] = (int64_t)" + ks.Word(static_cast<uint64_t>(cards_[t])) + ";");
    ks.L("const int nep = (int)a.w[" + std::to_string(w_nep_) + "];");
    ks.L("const int64_t S = (int64_t)a.w[" + std::to_string(w_total_) + "];");
    ks.L("int cur_e = -1; int64_t s0 = 0, e_start = 0;");
    ks.Open("auto use_ep = [&](int e)");
    ks.L("if (e == cur_e) return;");
    ks.L("cur_e = e;");
    ks.L("const uint64_t* q = " + EP + " + (int64_t)e * " + EPW + ";");
    ks.L("for (int p = 0; p < " + TS + "; p++) { ord[p] = (int32_t)q[p]; lk[p] = (int32_t)(int64_t)q[" + TS +
         " + p]; sched[p] = q[2 * " + TS + " + p]; off[p] = (int64_t)q[3 * " + TS + " + p]; }");
    ks.L("s0 = (int64_t)q[4 * " + TS + "]; e_start = (int64_t)q[4 * " + TS + " + 2];");
    ks.indent--;
    ks.L("};");
    // the episode whose slice holds batch item x (items numbered episode
    // after episode)
    ks.Open("auto ep_of = [&](int64_t x) -> int");
    ks.L("int e = 0;");
    ks.L("while (e + 1 < nep && (int64_t)" + EP + "[(int64_t)(e + 1) * " + EPW + " + 4 * " + TS + " + 2] <= x) e++;");
    ks.L("return e;");
    ks.indent--;
    ks.L("};");
    // tuples examined and results, per episode of the batch
    ks.L("unsigned long long wk[" + KB + "]; unsigned long long nres[" + KB + "];");
    ks.L("for (int e = 0; e < " + KB + "; e++) { wk[e] = 0; nres[e] = 0; }");
    w_phase_ = ks.Arg(0);
    w_qin_ = ks.Arg(0);
    ks.L("int64_t rows[" + TS + "]; int64_t iti[" + TS + "]; int64_t ite[" + TS + "];");
    if (agg_) {
      ks.L("unsigned long long fa_nres = 0; int64_t fa_rows = 0;");
      for (size_t j = 0; j < agg_->plans->size(); j++) {
        const AggPlan& p = (*agg_->plans)[j];
        const std::string J = std::to_string(j);
        const bool mn = p.kind == StateKind::MinMaxKey && p.is_min;
        ks.L("uint64_t fa_v" + J + " = " + (mn ? "~0ULL" : "0ULL") + "; int64_t fa_c" + J + " = 0;");
      }
    }
    std::vector<std::vector<std::string>> cache(T);
    auto load = [&](int t, std::vector<CVal>& out) {
      out = LoadMat(ks, eg, *mats_[t], "rows[" + std::to_string(t) + "]", &cache[t]);
    };
    // conditions
    ks.Open("auto cond = [&](int c) -> bool");
    ks.Open("switch (c)");
    for (size_t c = 0; c < op_.conditions.size(); c++) {
      ks.Open("case " + std::to_string(c) + ":");
      Scope sc;
      sc.child.resize(T);
      for (int t = 0; t < T; t++)
        if (cond_tables_[c] >> t & 1ULL) load(t, sc.child[t]);
      CVal v = eg.Emit(*op_.conditions[c], sc);
      ks.L("return !(" + v.n + ") && " + v.v + ";");
      ks.Close();
    }
    ks.Close();
    ks.L("return false;");
    ks.indent--;
    ks.L("};");
    ks.L("auto conds_ok = [&](uint64_t m) -> bool { while (m) { int c = __ffsll((long long)m) - 1; m &= m - 1; if (!cond(c)) return false; } return true; };");
    // lookups: case 2j probes table tb with the key of ta; 2j+1 the reverse.
    // init(p) sets [iti, ite) to the candidate run of position p: the whole
    // table for a scan, the run of the probe key's hash in the grouped index
    ks.Open("auto init = [&](int p)");
    ks.Open("switch (lk[p])");
    ks.L("case -1: iti[p] = 0; ite[p] = card[ord[p]]; break;");
    for (size_t j = 0; j < preds_.size(); j++)
      for (int side = 0; side < 2; side++) {
        const SkinnerPred& pr = preds_[j];
        int from = side == 0 ? pr.ta : pr.tb, fcol = side == 0 ? pr.ca : pr.cb;
        int to = side == 0 ? pr.tb : pr.ta;
        const JoinTable& jt = index_for_[to][side == 0 ? pr.cb : pr.ca];
        ks.Open("case " + std::to_string(j * 2 + side) + ":");
        std::vector<CVal> fv;
        load(from, fv);
        const CVal& key = fv.at(fcol);
        ks.L("iti[p] = 0; ite[p] = 0;");
        ks.Open("if (!(" + key.n + "))");
        std::string SL = ks.Ptr(jt.slots, "uint64_t", true), LN = ks.Ptr(jt.lens, "uint32_t", true);
        std::string M = ks.Word(jt.mask);
        ks.L("const uint32_t h = " + JoinHash(eg, {key}) + ";");
        ks.L("uint32_t s = h & (uint32_t)" + M + ";");
        ks.Open("for (uint32_t k = 0; k <= (uint32_t)" + M + "; k++, s = (s + 1) & (uint32_t)" + M + ")");
        ks.L("const uint64_t e = " + SL + "[s];");
        ks.L("if (e == 0) break;");
        ks.Open("if ((uint32_t)(e >> 32) == h)");
        ks.L("iti[p] = (int64_t)(uint32_t)e - 1; ite[p] = iti[p] + (int64_t)" + LN + "[s];");
        ks.L("break;");
        ks.Close();
        ks.Close();
        ks.Close();
        ks.L("break;");
        ks.Close();
      }
    ks.Close();
    ks.indent--;
    ks.L("};");
    // cand(p, c): the row of candidate c of position p's run, or -1 when its
    // key differs from the probe key (another key with the same hash)
    ks.Open("auto cand = [&](int p, int64_t c) -> int64_t");
    ks.Open("switch (lk[p])");
    ks.L("case -1: return c;");
    for (size_t j = 0; j < preds_.size(); j++)
      for (int side = 0; side < 2; side++) {
        const SkinnerPred& pr = preds_[j];
        int from = side == 0 ? pr.ta : pr.tb, fcol = side == 0 ? pr.ca : pr.cb;
        int to = side == 0 ? pr.tb : pr.ta, tcol = side == 0 ? pr.cb : pr.ca;
        const JoinTable& jt = index_for_[to][tcol];
        ks.Open("case " + std::to_string(j * 2 + side) + ":");
        std::string SR = ks.Ptr(jt.srow, "uint32_t", true);
        ks.L("int64_t br = (int64_t)" + SR + "[c];");
        std::vector<CVal> fv;
        load(from, fv);
        auto tv = LoadMat(ks, eg, *mats_[to], "br", &cache[to]);
        ks.L("return (" + eg.EqOf(tv.at(tcol), fv.at(fcol)) + ") ? br : (int64_t)-1;");
        ks.Close();
      }
    ks.Close();
    ks.L("return -1;");
    ks.indent--;
    ks.L("};");
    ks.Open("auto next = [&](int p) -> int64_t");
    ks.Open("while (iti[p] < ite[p])");
    ks.L("const int64_t r = cand(p, iti[p]++);");
    ks.L("if (r >= 0) return r;");
    ks.Close();
    ks.L("return -1;");
    ks.indent--;
    ks.L("};");
    // emission of one result row (output schema over the bound children)
    out_ptr_words_.clear();
    ks.Open("auto emit = [&]()");
    if (agg_) {
      Scope sc;
      sc.child.resize(T);
      for (int t = 0; t < T; t++) load(t, sc.child[t]);
      std::vector<CVal> vals;
      for (const auto& c : op_.output) vals.push_back(eg.Emit(*c.expr, sc));
      Scope s2;
      s2.child.push_back(vals);
      for (size_t j = 0; j < agg_->plans->size(); j++) {
        const AggPlan& p = (*agg_->plans)[j];
        const std::string J = std::to_string(j);
        CVal c = eg.Emit(p.agg->kid(0), s2);
        switch (p.kind) {
          case StateKind::MinMaxKey:
            ks.L("{ uint64_t k = " + OKey(eg, c) + "; fa_v" + J + " = (k " + (p.is_min ? "<" : ">") + " fa_v" + J +
                 ") ? k : fa_v" + J + "; }");
            break;
          case StateKind::SumI64: ks.L("fa_v" + J + " += (uint64_t)(int64_t)" + c.v + ";"); break;
          default: break;
        }
        ks.L("fa_c" + J + "++;");
      }
      ks.L("fa_rows++; fa_nres++; nres[cur_e]++;");
      w_count_ = ks.Arg(0);
    } else {
      Scope sc;
      sc.child.resize(T);
      for (int t = 0; t < T; t++) load(t, sc.child[t]);
      std::vector<CVal> vals;
      for (const auto& c : op_.output) vals.push_back(eg.Emit(*c.expr, sc));
      int wc = ks.Arg(0);
      w_count_ = wc;
      ks.L("nres[cur_e]++;");
      ks.L("uint64_t slot = kdb_alloc_slot((unsigned long long*)a.w[" + std::to_string(wc) + "]);");
      ks.Open("if (slot < a.w[" + std::to_string(w_cap_) + "])");
      for (size_t c = 0; c < vals.size(); c++) {
        const MatCol& mc = out_.cols[c];
        int wd = ks.Arg(0);
        out_ptr_words_.push_back(wd);
        std::string val = vals[c].type.id == TypeId::BOOLEAN ? "(int8_t)(" + vals[c].v + " ? 1 : 0)" : vals[c].v;
        ks.L("((" + StoreType(mc.type.id) + "*)a.w[" + std::to_string(wd) + "])[slot] = " + val + ";");
        int wn = ks.Arg(0);
        out_ptr_words_.push_back(wn);
        if (mc.nullable) ks.L("((int8_t*)a.w[" + std::to_string(wn) + "])[slot] = (" + vals[c].n + ") ? 1 : 0;");
      }
      w_pos_ = ks.Arg(0);
      ks.L("((uint64_t*)a.w[" + std::to_string(w_pos_) + "])[slot] = slot;");
      ks.Close();
    }
    ks.indent--;
    ks.L("};");
    // push(p, q): queue the candidate run of position p (rows of the earlier
    // positions bound) as tasks of split_run_ candidates on queue q; false
    // when the queue is full (the caller walks the run itself; the slots it
    // reserved past the capacity that are in range hold empty tasks)
    std::string TQ0, TQ1, TC, RUN, TCAP;
    const std::string TW = std::to_string(4 + T);  // position, begin, end, rows, episode
    if (split_) {
      TQ0 = ks.Ptr(tasks_[0], "uint64_t");
      TQ1 = ks.Ptr(tasks_[1], "uint64_t");
      TC = ks.Ptr(tcount_, "unsigned long long");
      RUN = "(int64_t)" + ks.Word(static_cast<uint64_t>(split_run_));
      TCAP = "(uint64_t)" + ks.Word(static_cast<uint64_t>(task_cap_));
      ks.Open("auto push = [&](int p, int q) -> bool");
      ks.L("const int64_t len = ite[p] - iti[p];");
      ks.L("const uint64_t n = (uint64_t)((len + " + RUN + " - 1) / " + RUN + ");");
      ks.L("const uint64_t base = atomicAdd(&" + TC + "[q], (unsigned long long)n);");
      ks.L("uint64_t* tq = q ? " + TQ1 + " : " + TQ0 + ";");
      ks.L("const bool ok = base + n <= " + TCAP + ";");
      ks.L("const uint64_t lim = ok ? base + n : (base < " + TCAP + " ? " + TCAP + " : base);");
      ks.Open("for (uint64_t i = base; i < lim; i++)");
      ks.L("uint64_t* t = tq + i * " + TW + ";");
      ks.L("const int64_t b = ok ? iti[p] + (int64_t)(i - base) * " + RUN + " : 0;");
      ks.L("const int64_t e = ok ? (b + " + RUN + " < ite[p] ? b + " + RUN + " : ite[p]) : 0;");
      ks.L("t[0] = (uint64_t)p; t[1] = (uint64_t)b; t[2] = (uint64_t)e;");
      ks.L("for (int k = 0; k < " + TS + "; k++) t[3 + k] = (uint64_t)rows[k];");
      ks.L("t[3 + " + TS + "] = (uint64_t)cur_e;");
      ks.Close();
      ks.L("return ok;");
      ks.indent--;
      ks.L("};");
    }
    // Phase 0 (expand): each leftmost tuple of the slice that passes its
    // conditions records its position-1 candidate run [beg, beg + len).
    // Phase 1 (episode), after an exclusive scan of the lengths: every
    // (leftmost tuple, position-1 candidate) pair is a work item spread over
    // all threads, so a tuple with a huge fan-out (skewed keys) is shared by
    // the whole grid; each item continues depth-first from position 2.
    std::string BG = ks.Ptr(beg_, "uint64_t"), OF = ks.Ptr(offs_, "uint64_t");
    ks.L("const int phase = (int)a.w[" + std::to_string(w_phase_) + "];");
    ks.Open("if (phase == 0)");
    ks.Open("for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < S; x += (int64_t)gridDim.x * blockDim.x)");
    ks.L("use_ep(ep_of(x)); rows[ord[0]] = s0 + (x - e_start); wk[cur_e]++;");
    if (T == 1) {
      ks.L("if (conds_ok(sched[0])) emit();");
    } else {
      ks.L("uint64_t len = 0;");
      ks.Open("if (conds_ok(sched[0]))");
      ks.L("init(1);");
      ks.L(BG + "[x] = (uint64_t)iti[1];");
      ks.L("len = (uint64_t)(ite[1] - iti[1]);");
      ks.Close();
      ks.L(OF + "[x] = len;");
    }
    ks.Close();
    ks.Close();
    if (T > 1) {
      ks.Open("else if (phase == 1)");
      ks.L("const int64_t m = S;");
      ks.L("const uint64_t total = " + OF + "[m];");
      ks.Open("for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x)");
      ks.L("int64_t lo = 0, hi = m - 1;");
      ks.Open("while (lo < hi)");
      ks.L("const int64_t mid = (lo + hi + 1) >> 1;");
      ks.L("if (" + OF + "[mid] <= w) lo = mid; else hi = mid - 1;");
      ks.Close();
      ks.L("use_ep(ep_of(lo)); rows[ord[0]] = s0 + (lo - e_start);");
      ks.L("const int64_t c1 = cand(1, (int64_t)(" + BG + "[lo] + (w - " + OF + "[lo])));");
      ks.L("if (c1 < 0 || c1 < off[ord[1]]) continue;");
      ks.L("rows[ord[1]] = c1; wk[cur_e]++;");
      ks.L("if (!conds_ok(sched[1])) continue;");
      // depth-first over positions from..T-1, the earlier ones bound; with
      // `preset` position `from`'s run is already in [iti, ite) (a task);
      // hot runs at position 3 and deeper go to queue `q`
      auto depth_first = [&](const std::string& from, bool preset, const std::string& q) {
        auto split = [&]() {
          if (split_)
            ks.L("if (p >= 3 && ite[p] - iti[p] > " + RUN + " && push(p, " + q + ")) iti[p] = ite[p];");
        };
        ks.L("int p = " + from + ";");
        ks.L("const int pmin = p;");
        if (!preset) {
          ks.L("init(p);");
          split();
        }
        ks.Open("while (p >= pmin)");
        ks.L("int64_t c = next(p);");
        ks.Open("if (c < 0)");
        ks.L("p--;");
        ks.L("continue;");
        ks.Close();
        ks.L("int t = ord[p];");
        ks.L("if (c < off[t]) continue;");
        ks.L("rows[t] = c; wk[cur_e]++;");
        ks.L("if (!conds_ok(sched[p])) continue;");
        ks.Open("if (p == " + std::to_string(T - 1) + ")");
        ks.L("emit();");
        ks.Close();
        ks.Open("else");
        ks.L("p++;");
        ks.L("init(p);");
        split();
        ks.Close();
        ks.Close();
      };
      if (T == 2) {
        ks.L("emit();");
      } else {
        depth_first("2", false, "0");
      }
      ks.Close();
      ks.Close();
      if (T > 2 && deep_) {
        // Phase 2: every position-1 item records its position-2 run (when
        // the items fit kMaxItems2; otherwise it finishes depth-first here).
        // Phase 3, after a scan of those lengths: every position-2
        // candidate is a work item, so a position-1 item whose key is hot
        // at position 2 is shared by the grid instead of one thread.
        std::string B2 = ks.Ptr(beg2_, "uint64_t"), O2 = ks.Ptr(offs2_, "uint64_t");
        std::string CAP2 = "(uint64_t)" + ks.Word(static_cast<uint64_t>(kMaxItems2));
        ks.Open("else if (phase == 2)");
        ks.L("const int64_t m = S;");
        ks.L("const uint64_t total = " + OF + "[m];");
        ks.L("const bool fits = total <= " + CAP2 + ";");
        ks.Open("for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x)");
        ks.L("uint64_t len2 = 0;");
        ks.Open("");
        ks.L("int64_t lo = 0, hi = m - 1;");
        ks.Open("while (lo < hi)");
        ks.L("const int64_t mid = (lo + hi + 1) >> 1;");
        ks.L("if (" + OF + "[mid] <= w) lo = mid; else hi = mid - 1;");
        ks.Close();
        ks.L("use_ep(ep_of(lo)); rows[ord[0]] = s0 + (lo - e_start);");
        ks.L("const int64_t c1 = cand(1, (int64_t)(" + BG + "[lo] + (w - " + OF + "[lo])));");
        ks.Open("if (c1 >= 0 && c1 >= off[ord[1]])");
        ks.L("rows[ord[1]] = c1; wk[cur_e]++;");
        ks.Open("if (conds_ok(sched[1]))");
        ks.Open("if (fits)");
        ks.L("init(2);");
        ks.L(B2 + "[w] = (uint64_t)iti[2];");
        ks.L("len2 = (uint64_t)(ite[2] - iti[2]);");
        ks.Close();
        ks.Open("else");
        depth_first("2", false, "0");
        ks.Close();
        ks.Close();
        ks.Close();
        ks.Close();
        ks.L("if (fits) " + O2 + "[w] = len2;");
        ks.Close();
        ks.Close();
        ks.Open("else if (phase == 3)");
        ks.L("const int64_t m = S;");
        ks.L("const uint64_t total = " + OF + "[m];");
        ks.Open("if (total <= " + CAP2 + " && total > 0)");
        ks.L("const uint64_t total2 = " + O2 + "[total];");
        ks.Open("for (uint64_t w2 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w2 < total2; w2 += (uint64_t)gridDim.x * blockDim.x)");
        ks.L("int64_t lo1 = 0, hi1 = (int64_t)total - 1;");
        ks.Open("while (lo1 < hi1)");
        ks.L("const int64_t mid = (lo1 + hi1 + 1) >> 1;");
        ks.L("if (" + O2 + "[mid] <= w2) lo1 = mid; else hi1 = mid - 1;");
        ks.Close();
        ks.L("const uint64_t w = (uint64_t)lo1;");
        ks.L("int64_t lo = 0, hi = m - 1;");
        ks.Open("while (lo < hi)");
        ks.L("const int64_t mid = (lo + hi + 1) >> 1;");
        ks.L("if (" + OF + "[mid] <= w) lo = mid; else hi = mid - 1;");
        ks.Close();
        ks.L("use_ep(ep_of(lo)); rows[ord[0]] = s0 + (lo - e_start);");
        // the item had a non-empty run: its position-1 candidate is valid
        ks.L("rows[ord[1]] = cand(1, (int64_t)(" + BG + "[lo] + (w - " + OF + "[lo])));");
        ks.L("const int64_t c2 = cand(2, (int64_t)(" + B2 + "[w] + (w2 - " + O2 + "[w])));");
        ks.L("if (c2 < 0 || c2 < off[ord[2]]) continue;");
        ks.L("rows[ord[2]] = c2; wk[cur_e]++;");
        ks.L("if (!conds_ok(sched[2])) continue;");
        if (T == 3) ks.L("emit();");
        else depth_first("3", false, "0");
        ks.Close();
        ks.Close();
        ks.Close();
      }
      if (split_) {
        // Phase 4: the queued tasks of queue qin, one per thread, each
        // continuing depth-first from its position; their hot runs go to
        // the other queue
        ks.Open("else if (phase == 4)");
        ks.L("const int qi = (int)a.w[" + std::to_string(w_qin_) + "];");
        ks.L("const uint64_t nq = " + TC + "[qi];");
        ks.L("const uint64_t nt = nq < " + TCAP + " ? nq : " + TCAP + ";");
        ks.L("const uint64_t* tq = qi ? " + TQ1 + " : " + TQ0 + ";");
        ks.Open("for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nt; w += (uint64_t)gridDim.x * blockDim.x)");
        ks.L("const uint64_t* t = tq + w * " + TW + ";");
        ks.L("use_ep((int)t[3 + " + TS + "]);");
        ks.L("const int tp = (int)t[0];");
        ks.L("iti[tp] = (int64_t)t[1]; ite[tp] = (int64_t)t[2];");
        ks.L("for (int k = 0; k < " + TS + "; k++) rows[k] = (int64_t)t[3 + k];");
        depth_first("tp", true, "1 - qi");
        ks.Close();
        ks.Close();
      }
    }
    {
      const std::string WT = ks.Ptr(work_, "unsigned long long");
      const std::string ER = ks.Ptr(eres_, "unsigned long long"), EW = ks.Ptr(ework_, "unsigned long long");
      ks.Open("for (int e = 0; e < nep; e++)");
      ks.L("if (wk[e]) { atomicAdd(&" + EW + "[e], wk[e]); atomicAdd(" + WT + ", wk[e]); }");
      ks.L("if (nres[e]) atomicAdd(&" + ER + "[e], nres[e]);");
      ks.Close();
    }
    if (agg_) {
      std::string ST = ks.Ptr(agg_->state, "unsigned long long");
      ks.Open("if (fa_rows)");
      for (size_t j = 0; j < agg_->plans->size(); j++) {
        const AggPlan& p = (*agg_->plans)[j];
        const std::string J = std::to_string(j), V = std::to_string(2 * j), C = std::to_string(2 * j + 1);
        if (p.kind == StateKind::MinMaxKey)
          ks.L(std::string(p.is_min ? "atomicMin" : "atomicMax") + "(&" + ST + "[" + V + "], (unsigned long long)fa_v" +
               J + ");");
        else if (p.kind == StateKind::SumI64)
          ks.L("atomicAdd(&" + ST + "[" + V + "], (unsigned long long)fa_v" + J + ");");
        ks.L("atomicAdd(&" + ST + "[" + C + "], (unsigned long long)fa_c" + J + ");");
      }
      ks.L("atomicAdd(&" + ST + "[" + std::to_string(agg_->nw - 2) + "], (unsigned long long)fa_rows);");
      ks.L("atomicAdd((unsigned long long*)a.w[" + std::to_string(w_count_) + "], fa_nres);");
      ks.Close();
    }
    std::string src = ks.Kernel("kdb_skinner_episode", 128);
    fn_ = ctx_.Kernel(src, "kdb_skinner_episode");
    args_ = ks.Args();
  }

  void PatchOut(KArgs& a) {
    a.w[w_count_] = reinterpret_cast<uint64_t>(count_);
    if (agg_) return;
    for (size_t c = 0; c < out_.cols.size(); c++) {
      a.w[out_ptr_words_[2 * c]] = reinterpret_cast<uint64_t>(out_.cols[c].data);
      a.w[out_ptr_words_[2 * c + 1]] = reinterpret_cast<uint64_t>(out_.cols[c].nulls);
    }
    a.w[w_pos_] = reinterpret_cast<uint64_t>(out_.pos);
  }

  void Grow(int64_t need) {
    MatBuffer bigger = alloc_out_(std::max<int64_t>(need, 2 * out_.cap));
    for (size_t c = 0; c < out_.cols.size(); c++) {
      size_t w = StoreWidth(out_.cols[c].type.id);
      if (produced_ && !ctx_.dry)
        KDB_CUDA(cudaMemcpyAsync(bigger.cols[c].data, out_.cols[c].data, w * produced_, cudaMemcpyDeviceToDevice,
                                 ctx_.stream));
      if (out_.cols[c].nulls && produced_ && !ctx_.dry)
        KDB_CUDA(cudaMemcpyAsync(bigger.cols[c].nulls, out_.cols[c].nulls, produced_, cudaMemcpyDeviceToDevice,
                                 ctx_.stream));
    }
    if (produced_ && !ctx_.dry)
      KDB_CUDA(cudaMemcpyAsync(bigger.pos, out_.pos, 8 * produced_, cudaMemcpyDeviceToDevice, ctx_.stream));
    out_ = bigger;
  }

  std::vector<CVal> LoadMat(KernelSource& ks, ExprGen& eg, const MatBuffer& m, const std::string& row,
                            std::vector<std::string>* cache) {
    std::vector<CVal> vals;
    for (size_t c = 0; c < m.cols.size(); c++) {
      const MatCol& mc = m.cols[c];
      if (cache->size() < 2 * m.cols.size()) cache->resize(2 * m.cols.size());
      if ((*cache)[2 * c].empty()) {
        (*cache)[2 * c] = ks.Ptr(mc.data, StoreType(mc.type.id), true);
        (*cache)[2 * c + 1] = mc.nullable ? ks.Ptr(mc.nulls, "int8_t", true) : "";
      }
      std::string dp = (*cache)[2 * c], np = (*cache)[2 * c + 1];
      std::string v = dp + "[" + row + "]";
      if (mc.type.id == TypeId::BOOLEAN) v = "(" + v + " != 0)";
      vals.push_back(eg.Bind(mc.type, v, mc.nullable ? "(" + np + "[" + row + "] != 0)" : "false"));
    }
    return vals;
  }

  std::string JoinHash(ExprGen& eg, const std::vector<CVal>& keys) {
    std::string h;
    for (const auto& k : keys) h = h.empty() ? eg.KeyHash32(k) : "kdb_hash_combine32(" + h + ", " + eg.KeyHash32(k) + ")";
    return h;
  }

  Context& ctx_;
  Arena& arena_;
  const Operator& op_;
  std::vector<const MatBuffer*> mats_;
  std::vector<SkinnerPred> preds_;
  std::function<MatBuffer(int64_t)> alloc_out_;
  int64_t budget_;
  uint32_t seed_;
  int T_ = 0;
  std::vector<int64_t> cards_, offsets_, slice_est_;
  std::vector<uint64_t> cond_tables_;
  std::set<std::pair<int, int>> connected_;
  const SkinnerAgg* agg_ = nullptr;  // fused aggregate, or null: materialise the results
  std::vector<uint64_t> adj_;  // join-graph neighbours of each table
  static constexpr int kPriorTables = 8;
  std::map<uint64_t, std::vector<double>> prior_cache_;  // joined set -> value per table
  std::vector<std::pair<std::vector<int>, double>> log_;   // (order, reward) per episode
  int64_t total_work_ = 0;
  std::vector<std::vector<JoinTable>> index_for_;
  MatBuffer out_;
  uint64_t* stats_ = nullptr;
  uint64_t* count_ = nullptr;
  uint64_t* work_ = nullptr;
  // Hot runs: a depth-first walk that meets a candidate run longer than
  // split_run_ at position 3 or deeper pushes it, in chunks of split_run_,
  // as tasks {position, begin, end, bound rows} to a queue instead of
  // walking it alone; the host then runs the queued tasks grid-wide (their
  // own hot runs go to the other queue) until both are empty.  A full queue
  // leaves the run to the thread that met it.
  bool split_ = false;
  int64_t split_run_ = 1024;
  int64_t task_cap_ = 1 << 16;
  uint64_t* tasks_[2] = {nullptr, nullptr};
  uint64_t* tcount_ = nullptr;
  int w_qin_ = 0;
  int64_t produced_ = 0;
  int64_t episodes_ = 0;
  CUfunction fn_ = nullptr;
  KArgs args_;
  int w_nep_ = 0, w_total_ = 0, w_cap_ = 0, w_count_ = 0, w_pos_ = 0, w_phase_ = 0;
  // batched episodes
  static constexpr int kMaxBatch = 16;
  int EpWords() const { return 4 * T_ + 4; }  // order, lookup, schedule, offsets (T each), s0, s1, start, pad
  int batch_ = 8;
  bool batching_ = false;  // Execute queues the episode instead of running it
  std::vector<Pending> pending_;
  int64_t batch_items_ = 0;  // leftmost tuples of the pending episodes
  std::vector<double> last_rewards_;
  double reward_sum_ = 0;
  int64_t rewards_seen_ = 0;
  int64_t batches_ = 0;
  uint64_t* ep_ = nullptr;     // device: per-episode parameters
  uint64_t* eres_ = nullptr;   // device: per-episode results (in stats_)
  uint64_t* ework_ = nullptr;  // device: per-episode work (in stats_)
  static constexpr int64_t kMaxSlice = 1 << 20;  // leftmost tuples per episode
  // position-1 items of an episode that can be expanded to position 2
  static constexpr int64_t kMaxItems2 = 1 << 20;
  bool deep_ = false;
  uint64_t* beg2_ = nullptr;   // per position-1 item: first position-2 candidate
  uint64_t* offs2_ = nullptr;  // per position-1 item: candidate count, then its exclusive prefix
  uint64_t* beg_ = nullptr;   // per slice tuple: first position-1 candidate
  uint64_t* offs_ = nullptr;  // per slice tuple: candidate count, then its exclusive prefix
  std::vector<int> out_ptr_words_;
};

MatBuffer Executor::RunSkinner(const Operator& op, const SkinnerAgg* agg) {
  ctx_.NotReplayable();  // episode decisions follow the host's UCT search
  const int T = static_cast<int>(op.children.size());
  if (T > 16) throw Error(-5, "Skinner join of more than 16 tables");
  if (op.conditions.size() > 64) throw Error(-5, "Skinner join with more than 64 conditions");
  // equality predicates between two children: the join graph and indexes
  std::vector<SkinnerPred> preds;
  for (size_t c = 0; c < op.conditions.size(); c++) {
    const Expr& e = *op.conditions[c];
    if (e.kind != ExprKind::Binary || e.bop != BinOp::EQ) continue;
    const Expr& x = e.kid(0);
    const Expr& y = e.kid(1);
    if (x.kind != ExprKind::ColRef || y.kind != ExprKind::ColRef || x.child_idx == y.child_idx) continue;
    preds.push_back({static_cast<int>(c), x.child_idx, x.column_idx, y.child_idx, y.column_idx});
  }
  // the join columns each child needs an index on
  std::vector<std::set<int>> index_cols(T);
  for (const auto& pr : preds) {
    index_cols[pr.tb].insert(pr.cb);
    index_cols[pr.ta].insert(pr.ca);
  }
  std::vector<std::vector<JoinTable>> index_for(T);
  for (int t = 0; t < T; t++) {
    const Operator& child = op.child(t);
    // A serving slot reuses a child's rows and indexes built by an earlier
    // request (the build cache waits on the event that follows their
    // construction); a plain query builds them itself.
    std::shared_ptr<BuildEntry> cached;
    std::string key;
    if (ctx_.build_cache && !ctx_.dry && !mats_.count(&child) &&
        (child.kind == OpKind::SCAN || child.kind == OpKind::SCAN_SELECT)) {
      key = ChildSig(child, index_cols[t]);
      cached = ctx_.build_cache->Find(key);
      if (cached) {
        KDB_CUDA(cudaStreamWaitEvent(ctx_.stream, cached->ready, 0));
      } else {
        cached = std::make_shared<BuildEntry>(ctx_);
        arena_.RedirectTo(&cached->arena);
        try {
          cached->mat = Materialize(child);
          cached->index.resize(cached->mat.cols.size());
          for (int c : index_cols[t]) cached->index[c] = BuildGroupedIndex(cached->mat, c);
        } catch (...) {
          arena_.RedirectTo(nullptr);
          throw;
        }
        arena_.RedirectTo(nullptr);
        KDB_CUDA(cudaEventRecord(cached->ready, ctx_.stream));
        cached = ctx_.build_cache->Insert(key, cached);
      }
      held_.push_back(cached);  // until this query is done with it
      mats_[&child] = cached->mat;
      index_for[t] = cached->index;
      continue;
    }
    if (!mats_.count(&child)) mats_[&child] = Materialize(child);
    index_for[t].resize(mats_.at(&child).cols.size());
  }
  std::vector<const MatBuffer*> mats;
  for (int t = 0; t < T; t++) mats.push_back(&mats_.at(&op.child(t)));
  for (const auto& pr : preds) {
    if (!index_for[pr.tb][pr.cb].slots) index_for[pr.tb][pr.cb] = BuildGroupedIndex(*mats[pr.tb], pr.cb);
    if (!index_for[pr.ta][pr.ca].slots) index_for[pr.ta][pr.ca] = BuildGroupedIndex(*mats[pr.ta], pr.ca);
  }
  auto alloc = [&](int64_t cap) { return AllocMat(op.output, cap); };
  SkinnerEngine eng(ctx_, arena_, op, mats, index_for, preds, alloc, ctx_.skinner_budget, ctx_.skinner_seed, agg);
  MatBuffer out = eng.Run(op.prefix_order);
  ctx_.last_skinner_episodes = eng.episodes();
  ctx_.last_skinner_batches = eng.batches();
  ctx_.last_skinner_work = eng.work();
  return out;
}

HostResult Executor::Run(const Operator& root) {
  MatBuffer m = Materialize(root);
  return Download(m, root);
}

HostResult Executor::Download(const MatBuffer& m, const Operator& root, bool check_error) {
  const auto& schema = SchemaOf(root);
  HostResult res;
  res.rows = m.rows;
  // one batch of device->host copies into the context's pinned staging
  // buffer and a single synchronisation (not one per column); with
  // `check_error` the device error word travels in the same batch
  std::vector<size_t> data_off(m.cols.size()), null_off(m.cols.size());
  size_t total = 0;
  for (size_t c = 0; c < m.cols.size(); c++) {
    data_off[c] = total;
    total += (StoreWidth(m.cols[c].type.id) * m.rows + 15) & ~size_t(15);
    null_off[c] = total;
    if (m.cols[c].nulls) total += (static_cast<size_t>(m.rows) + 15) & ~size_t(15);
  }
  const size_t err_off = total;
  std::shared_ptr<char> pinned = ctx_.AcquireHostBlock(total + 16);
  char* stage = pinned.get();
  if (!ctx_.dry && (m.rows > 0 || check_error)) {
    // several small segments: gather on the device, one copy to the host
    PackSegs segs;
    auto add = [&](const void* src, size_t bytes, size_t off) {
      if (segs.n < kMaxPackSegs) segs.seg[segs.n] = PackSeg{static_cast<const char*>(src), bytes, off};
      segs.n++;
    };
    if (m.rows > 0)
      for (size_t c = 0; c < m.cols.size(); c++) {
        const MatCol& mc = m.cols[c];
        add(mc.data, StoreWidth(mc.type.id) * m.rows, data_off[c]);
        if (mc.nulls) add(mc.nulls, m.rows, null_off[c]);
      }
    if (check_error) add(ctx_.d_err, 16, err_off);
    if (segs.n > 2 && segs.n <= kMaxPackSegs && total + 16 <= (size_t(64) << 20)) {
      ctx_.PackToHost(segs, err_off + (check_error ? 16 : 0), stage);
    } else {
      for (int i = 0; i < std::min(segs.n, kMaxPackSegs); i++)
        KDB_CUDA(cudaMemcpyAsync(stage + segs.seg[i].off, segs.seg[i].src, segs.seg[i].bytes, cudaMemcpyDeviceToHost,
                                 ctx_.stream));
      if (segs.n > kMaxPackSegs) {  // wide results: the remaining segments one by one
        int i = 0;
        for (size_t c = 0; c < m.cols.size() && m.rows > 0; c++) {
          const MatCol& mc = m.cols[c];
          for (int part = 0; part < (mc.nulls ? 2 : 1); part++, i++) {
            if (i < kMaxPackSegs) continue;
            if (part == 0)
              KDB_CUDA(cudaMemcpyAsync(stage + data_off[c], mc.data, StoreWidth(mc.type.id) * m.rows,
                                       cudaMemcpyDeviceToHost, ctx_.stream));
            else
              KDB_CUDA(cudaMemcpyAsync(stage + null_off[c], mc.nulls, m.rows, cudaMemcpyDeviceToHost, ctx_.stream));
          }
        }
        if (check_error && i >= kMaxPackSegs)
          KDB_CUDA(cudaMemcpyAsync(stage + err_off, ctx_.d_err, 16, cudaMemcpyDeviceToHost, ctx_.stream));
      }
    }
    KDB_CUDA(cudaStreamSynchronize(ctx_.stream));
    if (check_error) {
      int err[4];
      std::memcpy(err, stage + err_off, sizeof(err));
      if (err[0]) {
        KDB_CUDA(cudaMemsetAsync(ctx_.d_err, 0, sizeof(int) * 4, ctx_.stream));
        throw Error(-4, "replayed query raised a device error");
      }
    }
    if (m.rows == 0 && total) std::memset(stage, 0, total);
  } else if (total) {
    std::memset(stage, 0, total);
  }
  // A small result is copied out of the pinned block, which goes straight
  // back to the pool: callers that hold many results (a server's finished
  // tickets) would otherwise make every further result allocate pinned
  // memory, and pinned allocation and release stall the whole device.
  constexpr size_t kSmallResult = size_t(64) << 10;
  if (total + 16 <= kSmallResult) {
    res.block = std::shared_ptr<char>(new char[total + 16], std::default_delete<char[]>());
    std::memcpy(res.block.get(), stage, total + 16);
    stage = res.block.get();
  } else {
    res.block = pinned;
  }
  for (size_t c = 0; c < m.cols.size(); c++) {
    const MatCol& mc = m.cols[c];
    HostColumn hc;
    hc.name = schema[c].name;
    hc.type = mc.type;
    const char* raw = stage + data_off[c];
    if (mc.type.id != TypeId::TEXT) {
      // the column stays in the result's block as downloaded
      hc.packed = true;
      hc.data = raw;
      hc.nulls = mc.nulls ? reinterpret_cast<const int8_t*>(stage + null_off[c]) : nullptr;
      hc.width = static_cast<int>(StoreWidth(mc.type.id));
      res.cols.push_back(std::move(hc));
      continue;
    }
    if (mc.nulls) hc.null.assign(stage + null_off[c], stage + null_off[c] + m.rows);
    else hc.null.assign(m.rows, 0);
    // TEXT: the strings' bytes are gathered on the device and copied once
    const DevStr* ds = reinterpret_cast<const DevStr*>(raw);
    std::vector<int64_t> off(m.rows + 1, 0);
    for (int64_t r = 0; r < m.rows; r++) off[r + 1] = off[r] + (hc.null[r] ? 0 : ds[r].len);
    int64_t nbytes = off[m.rows];
    hc.s.resize(m.rows);
    if (nbytes > 0) {
      int64_t* d_off = arena_.AllocT<int64_t>(m.rows + 1);
      char* d_chars = arena_.AllocT<char>(nbytes);
      ctx_.H2D(d_off, off.data(), sizeof(int64_t) * (m.rows + 1));
      KernelSource ks;
      std::string D = ks.Ptr(mc.data, "kdb_str", true), O = ks.Ptr(d_off, "int64_t", true);
      std::string CH = ks.Ptr(d_chars, "char");
      std::string N = ks.Word(static_cast<uint64_t>(m.rows));
      ks.Open("for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < (int64_t)" + N +
              "; r += (int64_t)gridDim.x * blockDim.x)");
      ks.L("int64_t len = " + O + "[r + 1] - " + O + "[r];");
      ks.L("for (int64_t b = 0; b < len; b++) " + CH + "[" + O + "[r] + b] = " + D + "[r].p[b];");
      ks.Close();
      LaunchPipeline(ks, m.rows, "text download");
      std::vector<char> chars(nbytes);
      ctx_.D2H(chars.data(), d_chars, nbytes);
      for (int64_t r = 0; r < m.rows; r++) hc.s[r].assign(chars.data() + off[r], off[r + 1] - off[r]);
    }
    res.cols.push_back(std::move(hc));
  }
  return res;
}

}  // namespace

PreparedQuery::~PreparedQuery() {
  if (exec) cudaGraphExecDestroy(exec);
}

void PreparedQuery::Replay(cudaStream_t s) const {
  if (direct) {
    for (const auto& op : ops) op(s);
    KDB_CUDA(cudaGetLastError());
  } else {
    KDB_CUDA(cudaGraphLaunch(exec, s));
  }
}

namespace {

constexpr size_t kMaxPreparedBytes = size_t(1) << 30;  // device memory a prepared query may keep

// CUDA-event timing of one query's pipelines on the context's stream (the
// context's two timing events, made once).  Mark() follows the pipelines'
// work and precedes the result download, whose own synchronisation then
// completes the end event: Done() adds no round trip to the device.
class QueryTimer {
 public:
  explicit QueryTimer(Context& ctx) : ctx_(ctx) {
    ctx.BeginQueryProfile();
    ctx.QueryEvents(&e0_, &e1_);
    KDB_CUDA(cudaEventRecord(e0_, ctx.stream));
  }
  void Mark() {
    if (marked_) return;
    KDB_CUDA(cudaEventRecord(e1_, ctx_.stream));
    marked_ = true;
  }
  void Done() {
    Mark();
    KDB_CUDA(cudaEventSynchronize(e1_));
    float ms = 0;
    KDB_CUDA(cudaEventElapsedTime(&ms, e0_, e1_));
    ctx_.last_device_ms = ms;
    ctx_.EndQueryProfile();
  }

 private:
  Context& ctx_;
  cudaEvent_t e0_ = nullptr, e1_ = nullptr;
  bool marked_ = false;
};

}  // namespace

// Graph launch or launches one by one: a graph costs a fixed latency before
// its first kernel starts, separate launches cost host time per launch that
// the GPU may overtake.  Both are timed on the device (alternating, median
// of three) for queries of a few launches that run under a few
// milliseconds; the replays recompute the same result in place.
void ChooseReplay(Context& ctx, PreparedQuery& pq) {
  constexpr size_t kMaxDirectOps = 48;
  if (pq.ops.size() > kMaxDirectOps || ctx.OptStr("KDB_REPLAY_GRAPH")) return;
  cudaEvent_t e0, e1;
  KDB_CUDA(cudaEventCreate(&e0));
  KDB_CUDA(cudaEventCreate(&e1));
  auto time = [&](bool direct) {
    pq.direct = direct;
    KDB_CUDA(cudaStreamSynchronize(ctx.stream));
    KDB_CUDA(cudaEventRecord(e0, ctx.stream));
    pq.Replay(ctx.stream);
    KDB_CUDA(cudaEventRecord(e1, ctx.stream));
    KDB_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    KDB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    return ms;
  };
  std::vector<float> g, d;
  g.push_back(time(false));
  if (g[0] < 2.0f) {
    g.clear();
    for (int i = 0; i < 3; i++) {
      g.push_back(time(false));
      d.push_back(time(true));
    }
    std::sort(g.begin(), g.end());
    std::sort(d.begin(), d.end());
  }
  pq.direct = !d.empty() && d[1] < g[1];
  if (ctx.OptStr("KDB_REPLAY_DIRECT")) pq.direct = true;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
}

HostResult ExecutePlan(Context& ctx, const plan::Operator& root, std::unique_ptr<PreparedQuery>* prepared) {
  if (ctx.dry) {
    Arena arena(ctx);
    Executor ex(ctx, arena);
    return ex.Run(root);
  }
  // Profiling a prepared query: its recorded launches replayed with an event
  // pair around every kernel, queued behind a short delay so that the
  // kernels run back to back as in the query's replay (a fresh execution
  // leaves the GPU waiting for the host between a kernel's start event and
  // its launch, and charges that wait to the kernel).
  if (ctx.profile && prepared && *prepared && (*prepared)->catalog_version == ctx.catalog_version &&
      (*prepared)->tags.size() == (*prepared)->ops.size() && !ctx.OptStr("KDB_PROFILE_FRESH")) {
    PreparedQuery& pq = **prepared;
    // a fixed delay first: the host queues every launch and event behind
    // it, so the kernels then run back to back
    ctx.DelayStream(std::min(2000.0, 20.0 + 10.0 * static_cast<double>(pq.ops.size())));
    QueryTimer timer(ctx);
    for (size_t i = 0; i < pq.ops.size(); i++) {
      if (pq.tags[i].empty()) {
        pq.ops[i](ctx.stream);
        continue;
      }
      Context::LaunchTiming t;
      t.tag = pq.tags[i];
      KDB_CUDA(cudaEventCreate(&t.start));
      KDB_CUDA(cudaEventCreate(&t.stop));
      ctx.timings.push_back(t);
      KDB_CUDA(cudaEventRecord(t.start, ctx.stream));
      pq.ops[i](ctx.stream);
      KDB_CUDA(cudaEventRecord(t.stop, ctx.stream));
    }
    KDB_CUDA(cudaGetLastError());
    timer.Mark();
    ctx.kernel_launches += pq.launches;
    HostResult r;
    try {
      Arena arena(ctx);
      Executor ex(ctx, arena);
      r = ex.Download(pq.result, root, true);
    } catch (...) {
      cudaStreamSynchronize(ctx.stream);
      throw;
    }
    timer.Done();
    return r;
  }
  const bool prepare = prepared != nullptr && !ctx.profile;
  if (prepare && *prepared) {
    PreparedQuery& pq = **prepared;
    if (pq.catalog_version == ctx.catalog_version && !pq.exec && !pq.direct) {
      // first replay: capture the recorded launches as a graph and choose
      // between the graph and the launches themselves
      cudaGraph_t g = nullptr;
      KDB_CUDA(cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeThreadLocal));
      for (auto& op : pq.ops) op(ctx.stream);
      KDB_CUDA(cudaStreamEndCapture(ctx.stream, &g));
      cudaError_t ie = cudaGraphInstantiate(&pq.exec, g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) {
        cudaGetLastError();
        pq.exec = nullptr;
        pq.direct = true;
      } else {
        ChooseReplay(ctx, pq);
      }
    }
    if (pq.catalog_version == ctx.catalog_version) {
      // replay: one graph launch (or the recorded launches), then the
      // result download
      QueryTimer timer(ctx);
      pq.Replay(ctx.stream);
      timer.Mark();
      ctx.kernel_launches += pq.launches;
      bool ok = true;
      HostResult r;
      try {
        Arena arena(ctx);
        Executor ex(ctx, arena);
        r = ex.Download(pq.result, root, true);
      } catch (const Error&) {
        ok = false;  // run it afresh below
      }
      if (ok) {
        timer.Done();
        return r;
      }
    }
    prepared->reset();
  }
  QueryTimer timer(ctx);
  auto pq = std::make_unique<PreparedQuery>();
  pq->arena = std::make_unique<Arena>(ctx);
  Recorder rec;
  if (prepare) ctx.rec = &rec;
  HostResult r;
  MatBuffer m;
  try {
    Executor ex(ctx, *pq->arena);
    m = ex.MaterializeRoot(root);
    ctx.rec = nullptr;
    timer.Mark();
    r = ex.Download(m, root);
  } catch (...) {
    ctx.rec = nullptr;
    cudaStreamSynchronize(ctx.stream);
    throw;
  }
  timer.Done();
  if (prepare && rec.replayable && pq->arena->bytes() <= kMaxPreparedBytes) {
    // the graph is built on the first replay: a plan that never repeats
    // over the same tables (tables re-uploaded before every run) pays only
    // for recording the launches
    pq->result = m;
    pq->catalog_version = ctx.catalog_version;
    pq->launches = rec.launches;
    pq->ops = std::move(rec.ops);
    pq->tags = std::move(rec.tags);
    *prepared = std::move(pq);
  }
  return r;
}


// ---------------------------------------------------------------------------
// Per-operator scan-select (kernel a; scan_select_translator.cc:92-156 with
// the filter semantics of expression_translator.cc): the filter is compiled
// into a kernel that evaluates 4 consecutive rows per thread from 128-bit
// loads and compacts the qualifying row ids of each 1024-row tile in row
// order (per-thread counts, warp shuffle scan, block scan of the warp
// totals) into a tile-sized region of a scratch buffer; a scan of the tile
// counts and one gather then produce the selection vector in ascending row
// order.
// ---------------------------------------------------------------------------
std::unique_ptr<ops::SelVec> ScanSelectRows(Context& ctx, const std::string& table,
                                            const std::vector<std::string>& colnames, const plan::Expr& filter) {
  auto it = ctx.tables.find(table);
  if (it == ctx.tables.end()) throw Error(-1, "unknown table " + table);
  if (ctx.dry) throw Error(-5, "operators need a device context");
  const int64_t n = std::max<int64_t>(it->second.rows, 0);
  if (n >= (int64_t(1) << 31)) throw Error(-4, "selection vectors hold row ids below 2^31");
  auto sv = std::make_unique<ops::SelVec>();
  sv->table = table;
  KernelSource ks;
  ExprGen eg(ctx, ks);
  std::vector<const DevColumn*> cols;
  std::vector<std::string> dp, np, tp;
  for (const auto& name : colnames) {
    const DevColumn& c = ctx.Column(table, name);
    cols.push_back(&c);
    if (c.type.id == TypeId::TEXT) {
      dp.push_back(ks.Ptr(c.toff, "int64_t", true));
      tp.push_back(ks.Ptr(c.tchars, "char", true));
    } else {
      dp.push_back(ks.Ptr(c.data, StoreType(c.type.id), true));
      tp.push_back("");
    }
    np.push_back(c.nulls ? ks.Ptr(c.nulls, "int8_t", true) : "");
  }
  const int64_t ntiles = (n + 1023) / 1024;
  Arena arena(ctx);
  int32_t* scratch = arena.AllocT<int32_t>(std::max<int64_t>(ntiles * 1024, 1));
  uint64_t* counts = arena.AllocT<uint64_t>(ntiles + 1);
  const std::string sp = ks.Ptr(scratch, "int32_t");
  const std::string cp = ks.Ptr(counts, "uint64_t");
  ks.pre << "  __shared__ unsigned kdb_wsum[8];\n";
  ks.L("const int64_t nrows = (int64_t)" + ks.Word(static_cast<uint64_t>(n)) + ";");
  ks.L("const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;");
  ks.Open("for (int64_t tile = blockIdx.x; tile * 1024 < nrows; tile += gridDim.x)");
  ks.L("const int64_t base = tile * 1024 + threadIdx.x * 4;");
  ks.L("const bool full = base + 4 <= nrows;");
  std::vector<std::string> arr(cols.size()), narr(cols.size());
  for (size_t k = 0; k < cols.size(); k++) {
    if (cols[k]->type.id == TypeId::TEXT) continue;
    const std::string st = StoreType(cols[k]->type.id);
    arr[k] = ks.Fresh("L");
    ks.L(st + " " + arr[k] + "[4];");
    ks.L("if (full) kdb_ld4(" + dp[k] + ", base, " + arr[k] + "); else for (int u = 0; u < 4; u++) " + arr[k] +
         "[u] = base + u < nrows ? " + dp[k] + "[base + u] : (" + st + ")0;");
    if (!np[k].empty()) {
      narr[k] = ks.Fresh("N");
      ks.L("int8_t " + narr[k] + "[4];");
      ks.L("if (full) kdb_ld4(" + np[k] + ", base, " + narr[k] + "); else for (int u = 0; u < 4; u++) " + narr[k] +
           "[u] = base + u < nrows ? " + np[k] + "[base + u] : (int8_t)0;");
    }
  }
  ks.L("bool f[4];");
  ks.L("#pragma unroll");
  ks.Open("for (int u = 0; u < 4; u++)");
  ks.L("const int64_t r = base + u;");
  ks.L("f[u] = false;");
  ks.Open("if (r < nrows)");
  std::vector<CVal> bound;
  for (size_t k = 0; k < cols.size(); k++) {
    const DevColumn& c = *cols[k];
    std::string v;
    std::string nul = "false";
    if (c.type.id == TypeId::TEXT) {
      v = "kdb_text_at(" + dp[k] + ", " + tp[k] + ", r)";
      if (!np[k].empty()) nul = "(" + np[k] + "[r] != 0)";
    } else {
      v = c.type.id == TypeId::BOOLEAN ? "(" + arr[k] + "[u] != 0)" : arr[k] + "[u]";
      if (!narr[k].empty()) nul = "(" + narr[k] + "[u] != 0)";
    }
    bound.push_back(eg.Bind(c.type, v, nul));
  }
  Scope sc;
  sc.virt = bound;
  sc.child.push_back(bound);
  CVal fv = eg.Emit(filter, sc);
  ks.L("f[u] = !(" + fv.n + ") && (" + fv.v + ");");
  ks.Close();
  ks.Close();
  // ordered compaction of the tile: thread t holds rows 4t..4t+3
  ks.L("const unsigned mine = (unsigned)f[0] + (unsigned)f[1] + (unsigned)f[2] + (unsigned)f[3];");
  ks.L("unsigned incl = mine;");
  ks.L("for (int d = 1; d < 32; d <<= 1) { unsigned y = __shfl_up_sync(0xffffffffu, incl, d); if (lane >= d) incl += y; }");
  ks.L("if (lane == 31) kdb_wsum[warp] = incl;");
  ks.L("__syncthreads();");
  ks.L("unsigned before = 0, total = 0;");
  ks.L("for (int w = 0; w < (int)(blockDim.x >> 5); w++) { unsigned x = kdb_wsum[w]; if (w < warp) before += x; total += x; }");
  ks.L("unsigned at = before + incl - mine;");
  ks.L("int32_t* dst = " + sp + " + tile * 1024;");
  ks.L("for (int u = 0; u < 4; u++) if (f[u]) dst[at++] = (int32_t)(base + u);");
  ks.L("if (threadIdx.x == 0) " + cp + "[tile] = total;");
  ks.L("__syncthreads();");
  ks.Close();
  const std::string name = "kdb_scan_select_rows";
  CUfunction fn = ctx.Kernel(ks.Kernel(name, 256), name);
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(ntiles, ctx.num_sms * 8)));
  if (ntiles > 0) ctx.Launch(fn, grid, 256, ks.Args(), 0, "scan select");
  ctx.ScanU64(counts, ntiles, "scan select offsets");
  uint64_t total = 0;
  ctx.D2H(&total, counts + ntiles, sizeof(total));
  ctx.CheckDeviceError("scan select");
  sv->n = static_cast<int64_t>(total);
  sv->rows = static_cast<int32_t*>(nullptr);
  void* out = nullptr;
  KDB_CUDA(cudaMallocAsync(&out, sizeof(int32_t) * std::max<uint64_t>(total, 1), ctx.stream));
  sv->rows = static_cast<int32_t*>(out);
  sv->ctx = &ctx;
  ops::GatherTiles(ctx, scratch, counts, ntiles, sv->rows);
  KDB_CUDA(cudaStreamSynchronize(ctx.stream));
  return sv;
}

}  // namespace kdb
