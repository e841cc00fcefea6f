/* kdb_plan_json.h -- KushDB-side serialiser of plan::Operator trees into the
 * JSON that kdb_query_execute / kdb_skinner_execute take.
 *
 * Header-only C++17, meant to be included by KushDB itself (the caller of
 * the C ABI in kdb_b200.h): it walks a tree through the reference's own
 * visitor interfaces (plan/operator/operator_visitor.h:33-46,
 * plan/expression/expression_visitor.h:31-44) and public accessors
 * (Relation(), ScanSchema(), Filters(), LeftColumns()/RightColumns(),
 * GroupByExprs(), AggExprs(), KeyExprs()/Ascending(), Conditions()/
 * PrefixOrder(), Schema().Columns(), GetChildIdx()/GetColumnIdx(),
 * OpType(), AggType(), LiteralExpression::Visit, Values(), Type()/
 * Nullable()), and writes per node the fields kushdb_b200/csrc/plan.h
 * parses.  The reference's own plan::Operator::ToJson() is a debug dump
 * without column indices, literal types or child indices, hence this file.
 *
 * Usage on the KushDB side:
 *   #include "kdb_plan_json.h"
 *   std::string json = kdb_b200::ToBackendJson(root);   // root: plan::Operator
 *   kdb_query_execute(ctx, json.c_str(), &result);
 *
 * RegexpMatchingExpression is written with its RE2 pattern text; the
 * backend runs the patterns the planner makes from SQL LIKE
 * (plan/planner.cc:283-321: ^...$ over escaped bytes, "." and ".*") and
 * rejects any other regular expression with KDB_ERR_UNSUPPORTED.
 */
#ifndef KDB_PLAN_JSON_H_
#define KDB_PLAN_JSON_H_

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "plan/expression/aggregate_expression.h"
#include "plan/expression/arithmetic_expression.h"
#include "plan/expression/case_expression.h"
#include "plan/expression/column_ref_expression.h"
#include "plan/expression/conversion_expression.h"
#include "plan/expression/enum_in_expression.h"
#include "plan/expression/expression_visitor.h"
#include "plan/expression/extract_expression.h"
#include "plan/expression/literal_expression.h"
#include "plan/expression/virtual_column_ref_expression.h"
#include "plan/operator/aggregate_operator.h"
#include "plan/operator/cross_product_operator.h"
#include "plan/operator/group_by_aggregate_operator.h"
#include "plan/operator/hash_join_operator.h"
#include "plan/operator/operator_visitor.h"
#include "plan/operator/order_by_operator.h"
#include "plan/operator/output_operator.h"
#include "plan/operator/scan_operator.h"
#include "plan/operator/scan_select_operator.h"
#include "plan/operator/select_operator.h"
#include "plan/operator/simd_scan_select_operator.h"
#include "plan/operator/skinner_join_operator.h"

namespace kdb_b200 {

namespace plan_json_detail {

inline std::string Quote(std::string_view s) {
  std::string o = "\"";
  for (unsigned char c : s) {
    switch (c) {
      case '"': o += "\\\""; break;
      case '\\': o += "\\\\"; break;
      case '\n': o += "\\n"; break;
      case '\r': o += "\\r"; break;
      case '\t': o += "\\t"; break;
      default:
        if (c < 0x20) {
          char buf[8];
          std::snprintf(buf, sizeof(buf), "\\u%04x", c);
          o += buf;
        } else {
          o += static_cast<char>(c);
        }
    }
  }
  return o + "\"";
}

// catalog::Type -> "SMALLINT" ... "ENUM:<id>" (catalog/sql_type.h)
inline std::string TypeName(const kush::catalog::Type& t) {
  using kush::catalog::TypeId;
  switch (t.type_id) {
    case TypeId::SMALLINT: return "SMALLINT";
    case TypeId::INT: return "INT";
    case TypeId::BIGINT: return "BIGINT";
    case TypeId::REAL: return "REAL";
    case TypeId::DATE: return "DATE";
    case TypeId::TEXT: return "TEXT";
    case TypeId::BOOLEAN: return "BOOLEAN";
    case TypeId::ENUM: return "ENUM:" + std::to_string(t.enum_id);
  }
  throw std::runtime_error("unknown type");
}

inline std::string Bool(bool b) { return b ? "true" : "false"; }

// Shortest text that parses back to the same double.
inline std::string Real(double d) {
  if (!std::isfinite(d)) throw std::runtime_error("non-finite REAL literal");
  char buf[40];
  for (int prec = 15; prec <= 17; prec++) {
    std::snprintf(buf, sizeof(buf), "%.*g", prec, d);
    if (std::strtod(buf, nullptr) == d) break;
  }
  std::string s = buf;
  if (s.find_first_of(".eE") == std::string::npos) s += ".0";
  return s;
}

// Julian day of a civil date (the reference's DateBuilder::Build,
// runtime/date.cc:10-25); kept here so the header needs no runtime library.
inline int64_t JulianDay(int32_t year, int32_t month, int32_t day) {
  uint32_t y = static_cast<uint32_t>(year), m = static_cast<uint32_t>(month);
  if (m > 2) {
    m += 1;
    y += 4800;
  } else {
    m += 13;
    y += 4799;
  }
  int32_t century = static_cast<int32_t>(y / 100);
  int32_t julian = static_cast<int32_t>(y * 365 - 32167);
  julian += static_cast<int32_t>(y / 4) - century + century / 4;
  julian += static_cast<int32_t>(7834 * m / 256 + static_cast<uint32_t>(day));
  return julian;
}

class ExprWriter : public kush::plan::ImmutableExpressionVisitor {
 public:
  std::string out;

  static std::string Of(const kush::plan::Expression& e) {
    ExprWriter w;
    e.Accept(w);
    return w.out;
  }

  void Visit(const kush::plan::UnaryArithmeticExpression& e) override {
    const char* op = e.OpType() == kush::plan::UnaryArithmeticExpressionType::NOT ? "NOT" : "IS_NULL";
    out = "{\"e\":\"un\",\"op\":\"" + std::string(op) + "\"," + Head(e) + ",\"c\":" + Of(e.Child()) + "}";
  }
  void Visit(const kush::plan::BinaryArithmeticExpression& e) override {
    static const char* names[] = {"ADD", "SUB", "MUL", "DIV", "EQ", "NEQ", "LT", "LEQ",
                                  "GT", "GEQ", "AND", "OR", "STARTS_WITH", "ENDS_WITH", "CONTAINS"};
    const int k = static_cast<int>(e.OpType());
    if (k < 0 || k >= 15) throw std::runtime_error("unknown binary operator");
    out = "{\"e\":\"bin\",\"op\":\"" + std::string(names[k]) + "\"," + Head(e) + ",\"l\":" + Of(e.LeftChild()) +
          ",\"r\":" + Of(e.RightChild()) + "}";
  }
  void Visit(const kush::plan::AggregateExpression& e) override {
    using kush::plan::AggregateType;
    std::string a;
    switch (e.AggType()) {
      case AggregateType::SUM: a = "SUM"; break;
      case AggregateType::AVG: a = "AVG"; break;
      case AggregateType::COUNT: a = "COUNT"; break;
      case AggregateType::MAX: a = "MAX"; break;
      case AggregateType::MIN: a = "MIN"; break;
    }
    out = "{\"e\":\"agg\",\"agg\":\"" + a + "\"," + Head(e) + ",\"c\":" + Of(e.Child()) + "}";
  }
  void Visit(const kush::plan::ColumnRefExpression& e) override {
    out = "{\"e\":\"colref\"," + Head(e) + ",\"child\":" + std::to_string(e.GetChildIdx()) +
          ",\"idx\":" + std::to_string(e.GetColumnIdx()) + "}";
  }
  void Visit(const kush::plan::VirtualColumnRefExpression& e) override {
    out = "{\"e\":\"vcolref\"," + Head(e) + ",\"idx\":" + std::to_string(e.GetColumnIdx()) + "}";
  }
  void Visit(const kush::plan::LiteralExpression& e) override {
    std::string v;
    bool null = false;
    e.Visit([&](int16_t x, bool n) { v = std::to_string(x), null = n; },
            [&](int32_t x, bool n) { v = std::to_string(x), null = n; },
            [&](int64_t x, bool n) { v = std::to_string(x), null = n; },
            [&](double x, bool n) { v = n ? "0.0" : Real(x), null = n; },
            [&](std::string x, bool n) { v = Quote(x), null = n; },
            [&](bool x, bool n) { v = Bool(x), null = n; },
            [&](kush::runtime::Date::DateBuilder d, bool n) {
              v = std::to_string(JulianDay(d.year, d.month, d.day)), null = n;
            },
            [&](int32_t /*enum id*/, int32_t key, bool n) { v = std::to_string(key), null = n; });
    out = "{\"e\":\"lit\",\"type\":" + Quote(TypeName(e.Type())) + ",\"null\":" + Bool(null) + ",\"v\":" + v + "}";
  }
  void Visit(const kush::plan::CaseExpression& e) override {
    out = "{\"e\":\"case\"," + Head(e) + ",\"c\":" + Of(e.Cond()) + ",\"t\":" + Of(e.Then()) +
          ",\"f\":" + Of(e.Else()) + "}";
  }
  void Visit(const kush::plan::IntToFloatConversionExpression& e) override {
    out = "{\"e\":\"i2f\"," + Head(e) + ",\"c\":" + Of(e.Child()) + "}";
  }
  void Visit(const kush::plan::ExtractExpression& e) override {
    out = "{\"e\":\"extract\",\"what\":\"YEAR\"," + Head(e) + ",\"c\":" + Of(e.Child()) + "}";
  }
  void Visit(const kush::plan::RegexpMatchingExpression& e) override {
    out = "{\"e\":\"regex\"," + Head(e) + ",\"c\":" + Of(e.Child()) + ",\"pattern\":" +
          Quote(e.Regex()->pattern()) + "}";
  }
  void Visit(const kush::plan::EnumInExpression& e) override {
    std::string vals;
    for (int v : e.Values()) vals += (vals.empty() ? "" : ",") + std::to_string(v);
    out = "{\"e\":\"enum_in\"," + Head(e) + ",\"c\":" + Of(e.Child()) + ",\"values\":[" + vals + "]}";
  }

 private:
  static std::string Head(const kush::plan::Expression& e) {
    return "\"type\":" + Quote(TypeName(e.Type())) + ",\"nullable\":" + Bool(e.Nullable());
  }
};

template <typename Range>
std::string ExprList(const Range& exprs) {
  std::string o = "[";
  bool first = true;
  for (const auto& e : exprs) {
    o += (first ? "" : ",") + ExprWriter::Of(e.get());
    first = false;
  }
  return o + "]";
}

inline std::string Schema(const kush::plan::OperatorSchema& s) {
  std::string o = "[";
  bool first = true;
  for (const auto& c : s.Columns()) {
    o += (first ? "" : ",") + std::string("{\"name\":") + Quote(c.Name()) + ",\"expr\":" + ExprWriter::Of(c.Expr()) +
         "}";
    first = false;
  }
  return o + "]";
}

// the scanned catalog columns of a scan schema (name, type, nullability)
inline std::string ScanColumns(const kush::plan::OperatorSchema& s, const kush::catalog::Table& rel) {
  std::string o = "[";
  bool first = true;
  for (const auto& c : s.Columns()) {
    const auto& cat = rel[c.Name()];
    o += (first ? "" : ",") + std::string("{\"name\":") + Quote(c.Name()) + ",\"type\":" +
         Quote(TypeName(cat.GetType())) + ",\"nullable\":" + Bool(cat.Nullable()) + "}";
    first = false;
  }
  return o + "]";
}

class OpWriter : public kush::plan::ImmutableOperatorVisitor {
 public:
  std::string out;

  static std::string Of(const kush::plan::Operator& op) {
    OpWriter w;
    op.Accept(w);
    return w.out;
  }

  void Visit(const kush::plan::ScanOperator& op) override {
    out = "{\"op\":\"SCAN\",\"relation\":" + Quote(op.Relation().Name()) + ",\"columns\":" +
          ScanColumns(op.Schema(), op.Relation()) + ",\"output\":" + Schema(op.Schema()) + "}";
  }
  void Visit(const kush::plan::SelectOperator& op) override {
    out = "{\"op\":\"SELECT\",\"child\":" + Of(op.Child()) + ",\"cond\":" + ExprWriter::Of(op.Expr()) +
          ",\"output\":" + Schema(op.Schema()) + "}";
  }
  void Visit(const kush::plan::ScanSelectOperator& op) override { ScanSelect(op, "SCAN_SELECT"); }
  void Visit(const kush::plan::SimdScanSelectOperator& op) override { ScanSelect(op, "SIMD_SCAN_SELECT"); }
  void Visit(const kush::plan::OutputOperator& op) override { out = "{\"op\":\"OUTPUT\",\"child\":" + Of(op.Child()) + "}"; }
  void Visit(const kush::plan::HashJoinOperator& op) override {
    out = "{\"op\":\"HASH_JOIN\",\"left\":" + Of(op.LeftChild()) + ",\"right\":" + Of(op.RightChild()) +
          ",\"left_keys\":" + ExprList(op.LeftColumns()) + ",\"right_keys\":" + ExprList(op.RightColumns()) +
          ",\"output\":" + Schema(op.Schema()) + "}";
  }
  void Visit(const kush::plan::SkinnerJoinOperator& op) override {
    std::string ch = "[";
    bool first = true;
    for (const auto& c : op.Children()) {
      ch += (first ? "" : ",") + Of(c.get());
      first = false;
    }
    std::string prefix;
    for (int p : op.PrefixOrder()) prefix += (prefix.empty() ? "" : ",") + std::to_string(p);
    out = "{\"op\":\"SKINNER_JOIN\",\"children\":" + ch + "],\"conditions\":" + ExprList(op.Conditions()) +
          ",\"prefix_order\":[" + prefix + "],\"output\":" + Schema(op.Schema()) + "}";
  }
  void Visit(const kush::plan::GroupByAggregateOperator& op) override {
    out = "{\"op\":\"GROUP_BY_AGGREGATE\",\"child\":" + Of(op.Child()) + ",\"group_by\":" +
          ExprList(op.GroupByExprs()) + ",\"aggs\":" + ExprList(op.AggExprs()) + ",\"output\":" +
          Schema(op.Schema()) + "}";
  }
  void Visit(const kush::plan::AggregateOperator& op) override {
    out = "{\"op\":\"AGGREGATE\",\"child\":" + Of(op.Child()) + ",\"aggs\":" + ExprList(op.AggExprs()) +
          ",\"output\":" + Schema(op.Schema()) + "}";
  }
  void Visit(const kush::plan::OrderByOperator& op) override {
    std::string asc;
    for (bool a : op.Ascending()) asc += (asc.empty() ? "" : ",") + Bool(a);
    out = "{\"op\":\"ORDER_BY\",\"child\":" + Of(op.Child()) + ",\"keys\":" + ExprList(op.KeyExprs()) +
          ",\"asc\":[" + asc + "],\"output\":" + Schema(op.Schema()) + "}";
  }
  void Visit(const kush::plan::CrossProductOperator& op) override {
    const auto ch = op.Children();
    if (ch.size() != 2) throw std::runtime_error("CrossProduct takes two children");
    out = "{\"op\":\"CROSS_PRODUCT\",\"left\":" + Of(ch[0].get()) + ",\"right\":" + Of(ch[1].get()) +
          ",\"output\":" + Schema(op.Schema()) + "}";
  }

 private:
  void ScanSelect(const kush::plan::ScanSelectOperator& op, const char* name) {
    out = "{\"op\":\"" + std::string(name) + "\",\"relation\":" + Quote(op.Relation().Name()) + ",\"columns\":" +
          ScanColumns(op.ScanSchema(), op.Relation()) + ",\"output\":" + Schema(op.Schema()) + ",\"filters\":" +
          ExprList(op.Filters()) + "}";
  }
};

}  // namespace plan_json_detail

// The plan JSON of the tree rooted at `root` (an OutputOperator, or any
// operator the backend runs on its own, e.g. a SkinnerJoinOperator for
// kdb_skinner_execute).
inline std::string ToBackendJson(const kush::plan::Operator& root) {
  return plan_json_detail::OpWriter::Of(root);
}

}  // namespace kdb_b200

#endif  // KDB_PLAN_JSON_H_
