// C++ plan model: the operator / expression trees the engine consumes.
//
// Mirrors the reference's plan library (plan/operator/*.h, plan/expression/*.h,
// catalog/sql_type.h:7-85) class for class, but is built from the JSON text
// that crosses the C ABI instead of being linked against the reference (its
// plan library needs absl, nlohmann/json and magic_enum).
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "json.h"

namespace kdb::plan {

// catalog::TypeId (catalog/sql_type.h:7-16)
enum class TypeId { SMALLINT, INT, BIGINT, REAL, DATE, TEXT, BOOLEAN, ENUM };

struct Type {
  TypeId id = TypeId::INT;
  int32_t enum_id = 0;
  bool operator==(const Type& o) const { return id == o.id && enum_id == o.enum_id; }
  bool operator!=(const Type& o) const { return !(*this == o); }
};

inline Type ParseType(const std::string& s) {
  if (s.rfind("ENUM:", 0) == 0) return Type{TypeId::ENUM, std::stoi(s.substr(5))};
  if (s == "SMALLINT") return Type{TypeId::SMALLINT, 0};
  if (s == "INT") return Type{TypeId::INT, 0};
  if (s == "BIGINT") return Type{TypeId::BIGINT, 0};
  if (s == "REAL") return Type{TypeId::REAL, 0};
  if (s == "DATE") return Type{TypeId::DATE, 0};
  if (s == "TEXT") return Type{TypeId::TEXT, 0};
  if (s == "BOOLEAN") return Type{TypeId::BOOLEAN, 0};
  throw std::runtime_error("unknown type '" + s + "'");
}

inline const char* TypeName(TypeId t) {
  switch (t) {
    case TypeId::SMALLINT: return "SMALLINT";
    case TypeId::INT: return "INT";
    case TypeId::BIGINT: return "BIGINT";
    case TypeId::REAL: return "REAL";
    case TypeId::DATE: return "DATE";
    case TypeId::TEXT: return "TEXT";
    case TypeId::BOOLEAN: return "BOOLEAN";
    case TypeId::ENUM: return "ENUM";
  }
  return "?";
}

// Physical width in bytes of a fixed-width type (TEXT is variable).
inline int TypeWidth(TypeId t) {
  switch (t) {
    case TypeId::SMALLINT: return 2;
    case TypeId::INT:
    case TypeId::DATE:
    case TypeId::ENUM: return 4;
    case TypeId::BIGINT:
    case TypeId::REAL: return 8;
    case TypeId::BOOLEAN: return 1;
    case TypeId::TEXT: return 0;
  }
  return 0;
}

// plan::BinaryArithmeticExpressionType (plan/expression/arithmetic_expression.h:34-50)
enum class BinOp {
  ADD, SUB, MUL, DIV, EQ, NEQ, LT, LEQ, GT, GEQ, AND, OR, STARTS_WITH, ENDS_WITH, CONTAINS
};
// plan::UnaryArithmeticExpressionType (arithmetic_expression.h:13-16)
enum class UnOp { NOT, IS_NULL };
// plan::AggregateType (plan/expression/aggregate_expression.h)
enum class AggType { SUM, MIN, MAX, AVG, COUNT };

enum class ExprKind { ColRef, VirtColRef, Literal, Binary, Unary, Agg, Case, IntToFloat, Extract, EnumIn, Regexp };

struct Expr {
  ExprKind kind = ExprKind::Literal;
  Type type;
  bool nullable = false;
  // ColumnRefExpression / VirtualColumnRefExpression
  int child_idx = 0;
  int column_idx = 0;
  // LiteralExpression
  bool lit_null = false;
  int64_t ival = 0;  // SMALLINT/INT/BIGINT/DATE(JDN)/ENUM(key)/BOOLEAN
  double fval = 0;   // REAL
  std::string sval;  // TEXT
  BinOp bop = BinOp::ADD;
  UnOp uop = UnOp::NOT;
  AggType agg = AggType::SUM;
  std::vector<std::unique_ptr<Expr>> kids;  // binary: l, r; unary/agg/i2f/extract/in: c; case: c, t, f
  std::vector<int32_t> in_values;           // EnumInExpression
  std::string regex;                        // RegexpMatchingExpression (a LIKE pattern's regex)

  const Expr& kid(size_t i) const { return *kids.at(i); }
};

// plan::Operator kinds (plan/operator/operator_visitor.h:5-15)
enum class OpKind { SCAN, SCAN_SELECT, SELECT, HASH_JOIN, GROUP_BY_AGGREGATE, AGGREGATE, ORDER_BY,
                    SKINNER_JOIN, OUTPUT, CROSS_PRODUCT };

struct SchemaCol {
  std::string name;
  std::unique_ptr<Expr> expr;
};

struct ScanCol {
  std::string name;
  Type type;
  bool nullable = false;
};

struct Operator {
  OpKind kind = OpKind::SCAN;
  std::vector<SchemaCol> output;  // OperatorSchema (for OUTPUT: the child's)
  std::vector<std::unique_ptr<Operator>> children;
  // SCAN / SCAN_SELECT
  std::string relation;
  std::vector<ScanCol> scan_columns;
  // SCAN_SELECT filters, SELECT condition (one entry)
  std::vector<std::unique_ptr<Expr>> filters;
  // HASH_JOIN
  std::vector<std::unique_ptr<Expr>> left_keys, right_keys;
  // GROUP_BY_AGGREGATE / AGGREGATE
  std::vector<std::unique_ptr<Expr>> group_by, aggs;
  // ORDER_BY
  std::vector<std::unique_ptr<Expr>> sort_keys;
  std::vector<bool> asc;
  // SKINNER_JOIN
  std::vector<std::unique_ptr<Expr>> conditions;
  std::vector<int> prefix_order;

  const Operator& child(size_t i = 0) const { return *children.at(i); }
};

// ---------------------------------------------------------------------------
// JSON -> tree
// ---------------------------------------------------------------------------

inline BinOp ParseBinOp(const std::string& s) {
  static const char* names[] = {"ADD", "SUB", "MUL", "DIV", "EQ", "NEQ", "LT", "LEQ",
                                "GT", "GEQ", "AND", "OR", "STARTS_WITH", "ENDS_WITH",
                                "CONTAINS"};
  for (int i = 0; i < 15; i++)
    if (s == names[i]) return static_cast<BinOp>(i);
  throw std::runtime_error("unknown binary op " + s);
}

inline AggType ParseAgg(const std::string& s) {
  if (s == "SUM") return AggType::SUM;
  if (s == "MIN") return AggType::MIN;
  if (s == "MAX") return AggType::MAX;
  if (s == "AVG") return AggType::AVG;
  if (s == "COUNT") return AggType::COUNT;
  throw std::runtime_error("unknown aggregate " + s);
}

// The regex the reference's planner makes of a general LIKE pattern
// (plan/planner.cc:283-323): '^', then per pattern byte an escaped literal,
// '.' for '_' or ".*" for '%', then '$'.  Tokens: {0, byte} a literal,
// {1, 0} any one byte but '\n', {2, 0} any run of such bytes (RE2's '.'
// does not match a newline).  Anything else is not a LIKE regex.
inline std::vector<std::pair<int, unsigned char>> LikeTokens(const std::string& re) {
  if (re.size() < 2 || re.front() != '^' || re.back() != '$')
    throw std::runtime_error("unsupported regex (not a LIKE pattern): " + re);
  std::vector<std::pair<int, unsigned char>> t;
  for (size_t i = 1; i + 1 < re.size(); i++) {
    const char c = re[i];
    if (c == '\\') {
      if (i + 2 >= re.size()) throw std::runtime_error("dangling escape in regex " + re);
      t.emplace_back(0, static_cast<unsigned char>(re[++i]));
    } else if (c == '.') {
      if (i + 2 < re.size() && re[i + 1] == '*') {
        t.emplace_back(2, 0);
        i++;
      } else {
        t.emplace_back(1, 0);
      }
    } else if (std::string(".+*?^$()[]{}|").find(c) != std::string::npos) {
      throw std::runtime_error("unsupported regex (not a LIKE pattern): " + re);
    } else {
      t.emplace_back(0, static_cast<unsigned char>(c));
    }
  }
  return t;
}

inline std::unique_ptr<Expr> ParseExpr(const json::Value& j) {
  auto e = std::make_unique<Expr>();
  const std::string& k = j.at("e").str();
  e->type = ParseType(j.at("type").str());
  e->nullable = j.has("nullable") ? j.at("nullable").as_bool() : false;
  if (k == "colref") {
    e->kind = ExprKind::ColRef;
    e->child_idx = static_cast<int>(j.at("child").as_int());
    e->column_idx = static_cast<int>(j.at("idx").as_int());
  } else if (k == "vcolref") {
    e->kind = ExprKind::VirtColRef;
    e->column_idx = static_cast<int>(j.at("idx").as_int());
  } else if (k == "lit") {
    e->kind = ExprKind::Literal;
    e->lit_null = j.at("null").as_bool();
    e->nullable = e->lit_null;
    const auto& v = j.at("v");
    switch (e->type.id) {
      case TypeId::REAL: e->fval = v.as_double(); break;
      case TypeId::TEXT: e->sval = v.str(); break;
      case TypeId::BOOLEAN: e->ival = v.as_bool() ? 1 : 0; break;
      default: e->ival = v.as_int(); break;
    }
  } else if (k == "bin") {
    e->kind = ExprKind::Binary;
    e->bop = ParseBinOp(j.at("op").str());
    e->kids.push_back(ParseExpr(j.at("l")));
    e->kids.push_back(ParseExpr(j.at("r")));
  } else if (k == "un") {
    e->kind = ExprKind::Unary;
    const std::string& op = j.at("op").str();
    if (op == "NOT") e->uop = UnOp::NOT;
    else if (op == "IS_NULL") e->uop = UnOp::IS_NULL;
    else throw std::runtime_error("unknown unary op " + op);
    e->kids.push_back(ParseExpr(j.at("c")));
  } else if (k == "agg") {
    e->kind = ExprKind::Agg;
    e->agg = ParseAgg(j.at("agg").str());
    e->kids.push_back(ParseExpr(j.at("c")));
  } else if (k == "case") {
    e->kind = ExprKind::Case;
    e->kids.push_back(ParseExpr(j.at("c")));
    e->kids.push_back(ParseExpr(j.at("t")));
    e->kids.push_back(ParseExpr(j.at("f")));
  } else if (k == "i2f") {
    e->kind = ExprKind::IntToFloat;
    e->kids.push_back(ParseExpr(j.at("c")));
  } else if (k == "extract") {
    e->kind = ExprKind::Extract;
    if (j.at("what").str() != "YEAR") throw std::runtime_error("only EXTRACT(YEAR)");
    e->kids.push_back(ParseExpr(j.at("c")));
  } else if (k == "regex") {
    // RegexpMatchingExpression: the planner's regex of a general LIKE
    // pattern (plan/planner.cc:283-323), fully matched
    e->kind = ExprKind::Regexp;
    e->regex = j.at("pattern").str();
    e->kids.push_back(ParseExpr(j.at("c")));
  } else if (k == "enum_in") {
    e->kind = ExprKind::EnumIn;
    e->kids.push_back(ParseExpr(j.at("c")));
    for (size_t i = 0; i < j.at("values").size(); i++)
      e->in_values.push_back(static_cast<int32_t>(j.at("values")[i].as_int()));
  } else {
    throw std::runtime_error("unknown expression kind " + k);
  }
  return e;
}

inline std::vector<SchemaCol> ParseSchema(const json::Value& j) {
  std::vector<SchemaCol> out;
  for (size_t i = 0; i < j.size(); i++) {
    SchemaCol c;
    c.name = j[i].at("name").str();
    c.expr = ParseExpr(j[i].at("expr"));
    out.push_back(std::move(c));
  }
  return out;
}

inline std::vector<std::unique_ptr<Expr>> ParseExprList(const json::Value& j) {
  std::vector<std::unique_ptr<Expr>> out;
  for (size_t i = 0; i < j.size(); i++) out.push_back(ParseExpr(j[i]));
  return out;
}

inline std::unique_ptr<Operator> ParseOperator(const json::Value& j) {
  auto op = std::make_unique<Operator>();
  const std::string& k = j.at("op").str();
  auto scan_cols = [&]() {
    const auto& cols = j.at("columns");
    for (size_t i = 0; i < cols.size(); i++) {
      ScanCol c;
      c.name = cols[i].at("name").str();
      c.type = ParseType(cols[i].at("type").str());
      c.nullable = cols[i].at("nullable").as_bool();
      op->scan_columns.push_back(c);
    }
  };
  if (k == "SCAN") {
    op->kind = OpKind::SCAN;
    op->relation = j.at("relation").str();
    scan_cols();
    op->output = ParseSchema(j.at("output"));
  } else if (k == "SCAN_SELECT" || k == "SIMD_SCAN_SELECT") {
    op->kind = OpKind::SCAN_SELECT;
    op->relation = j.at("relation").str();
    scan_cols();
    op->output = ParseSchema(j.at("output"));
    op->filters = ParseExprList(j.at("filters"));
  } else if (k == "SELECT") {
    op->kind = OpKind::SELECT;
    op->children.push_back(ParseOperator(j.at("child")));
    op->filters.push_back(ParseExpr(j.at("cond")));
    op->output = ParseSchema(j.at("output"));
  } else if (k == "HASH_JOIN") {
    op->kind = OpKind::HASH_JOIN;
    op->children.push_back(ParseOperator(j.at("left")));
    op->children.push_back(ParseOperator(j.at("right")));
    op->left_keys = ParseExprList(j.at("left_keys"));
    op->right_keys = ParseExprList(j.at("right_keys"));
    op->output = ParseSchema(j.at("output"));
  } else if (k == "CROSS_PRODUCT") {
    // plan/operator/cross_product_operator.h: exactly two children
    op->kind = OpKind::CROSS_PRODUCT;
    op->children.push_back(ParseOperator(j.at("left")));
    op->children.push_back(ParseOperator(j.at("right")));
    op->output = ParseSchema(j.at("output"));
  } else if (k == "GROUP_BY_AGGREGATE") {
    op->kind = OpKind::GROUP_BY_AGGREGATE;
    op->children.push_back(ParseOperator(j.at("child")));
    op->group_by = ParseExprList(j.at("group_by"));
    op->aggs = ParseExprList(j.at("aggs"));
    op->output = ParseSchema(j.at("output"));
  } else if (k == "AGGREGATE") {
    op->kind = OpKind::AGGREGATE;
    op->children.push_back(ParseOperator(j.at("child")));
    op->aggs = ParseExprList(j.at("aggs"));
    op->output = ParseSchema(j.at("output"));
  } else if (k == "ORDER_BY") {
    op->kind = OpKind::ORDER_BY;
    op->children.push_back(ParseOperator(j.at("child")));
    op->sort_keys = ParseExprList(j.at("keys"));
    for (size_t i = 0; i < j.at("asc").size(); i++) op->asc.push_back(j.at("asc")[i].as_bool());
    op->output = ParseSchema(j.at("output"));
  } else if (k == "SKINNER_JOIN") {
    op->kind = OpKind::SKINNER_JOIN;
    const auto& ch = j.at("children");
    for (size_t i = 0; i < ch.size(); i++) op->children.push_back(ParseOperator(ch[i]));
    op->conditions = ParseExprList(j.at("conditions"));
    if (j.has("prefix_order"))
      for (size_t i = 0; i < j.at("prefix_order").size(); i++)
        op->prefix_order.push_back(static_cast<int>(j.at("prefix_order")[i].as_int()));
    op->output = ParseSchema(j.at("output"));
  } else if (k == "OUTPUT") {
    op->kind = OpKind::OUTPUT;
    op->children.push_back(ParseOperator(j.at("child")));
  } else {
    throw std::runtime_error("unsupported operator " + k);
  }
  return op;
}

inline std::unique_ptr<Operator> ParsePlan(const std::string& text) {
  return ParseOperator(json::Parse(text));
}

// The schema an operator exposes to its parent (OUTPUT passes its child's).
inline const std::vector<SchemaCol>& SchemaOf(const Operator& op) {
  return op.kind == OpKind::OUTPUT ? SchemaOf(op.child()) : op.output;
}

}  // namespace kdb::plan
