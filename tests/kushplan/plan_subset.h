// A source-compatible subset of the reference's catalog / plan class shapes
// (catalog/catalog.h, catalog/sql_type.h, runtime/date.h, plan/expression/*,
// plan/operator/*): the class names, enums, constructors and accessors that
// include/kdb_plan_json.h and the plan builders of tests/kushplan use, with
// implementations of this project's own.  Test infrastructure only: it lets
// the KushDB-side serialiser compile and run here, where the reference's
// plan library (absl, nlohmann/json, magic_enum, re2) cannot be built.
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <optional>
#include <stdexcept>
#include <string>
#include <string_view>
#include <utility>
#include <variant>
#include <vector>

namespace re2 {
// Stand-in for re2::RE2: only the pattern text the serialiser reads.
class RE2 {
 public:
  explicit RE2(std::string pattern) : pattern_(std::move(pattern)) {}
  const std::string& pattern() const { return pattern_; }

 private:
  std::string pattern_;
};
}  // namespace re2

namespace kush::catalog {

enum class TypeId { SMALLINT, INT, BIGINT, REAL, DATE, TEXT, BOOLEAN, ENUM };

struct Type {
  TypeId type_id;
  int32_t enum_id;
  bool operator==(const Type& o) const { return type_id == o.type_id && enum_id == o.enum_id; }
  bool operator!=(const Type& o) const { return !(*this == o); }
  static Type SmallInt() { return {TypeId::SMALLINT, 0}; }
  static Type Int() { return {TypeId::INT, 0}; }
  static Type BigInt() { return {TypeId::BIGINT, 0}; }
  static Type Real() { return {TypeId::REAL, 0}; }
  static Type Date() { return {TypeId::DATE, 0}; }
  static Type Text() { return {TypeId::TEXT, 0}; }
  static Type Boolean() { return {TypeId::BOOLEAN, 0}; }
  static Type Enum(int32_t id) { return {TypeId::ENUM, id}; }
};

class Column {
 public:
  Column(std::string_view name, const Type& type, std::string_view path, std::string_view null_path,
         std::string_view index_path)
      : name_(name), type_(type), path_(path), null_path_(null_path), index_path_(index_path) {}
  std::string_view Name() const { return name_; }
  const Type& GetType() const { return type_; }
  std::string_view Path() const { return path_; }
  std::string_view NullPath() const { return null_path_; }
  bool Nullable() const { return !null_path_.empty(); }
  std::string_view IndexPath() const { return index_path_; }
  bool HasIndex() const { return !index_path_.empty(); }

 private:
  std::string name_;
  Type type_;
  std::string path_, null_path_, index_path_;
};

class Table {
 public:
  explicit Table(std::string_view name) : name_(name) {}
  std::string_view Name() const { return name_; }
  Column& Insert(std::string_view attr, const Type& type, std::string_view path, std::string_view null_path,
                 std::string_view index_path) {
    order_.emplace_back(attr);
    return cols_.emplace(std::string(attr), Column(attr, type, path, null_path, index_path)).first->second;
  }
  const Column& operator[](std::string_view attr) const { return cols_.at(std::string(attr)); }
  std::vector<std::reference_wrapper<const Column>> Columns() const {
    std::vector<std::reference_wrapper<const Column>> out;
    for (const auto& n : order_) out.push_back(cols_.at(n));
    return out;
  }

 private:
  std::string name_;
  std::map<std::string, Column> cols_;
  std::vector<std::string> order_;
};

class Database {
 public:
  Table& Insert(std::string_view table) {
    return tables_.emplace(std::string(table), Table(table)).first->second;
  }
  const Table& operator[](std::string_view table) const { return tables_.at(std::string(table)); }
  bool Contains(std::string_view table) const { return tables_.count(std::string(table)) != 0; }

 private:
  std::map<std::string, Table> tables_;
};

}  // namespace kush::catalog

namespace kush::runtime::Date {
class DateBuilder {
 public:
  int32_t year, month, day;
  DateBuilder(int32_t y, int32_t m, int32_t d) : year(y), month(m), day(d) {}
};
}  // namespace kush::runtime::Date

namespace kush::plan {

class AggregateExpression;
class ColumnRefExpression;
class LiteralExpression;
class VirtualColumnRefExpression;
class UnaryArithmeticExpression;
class BinaryArithmeticExpression;
class CaseExpression;
class IntToFloatConversionExpression;
class ExtractExpression;
class RegexpMatchingExpression;
class EnumInExpression;

class ImmutableExpressionVisitor {
 public:
  virtual ~ImmutableExpressionVisitor() = default;
  virtual void Visit(const UnaryArithmeticExpression& arith) = 0;
  virtual void Visit(const BinaryArithmeticExpression& arith) = 0;
  virtual void Visit(const AggregateExpression& agg) = 0;
  virtual void Visit(const ColumnRefExpression& col_ref) = 0;
  virtual void Visit(const VirtualColumnRefExpression& virtual_col_ref) = 0;
  virtual void Visit(const LiteralExpression& literal) = 0;
  virtual void Visit(const CaseExpression& case_expr) = 0;
  virtual void Visit(const IntToFloatConversionExpression& conv) = 0;
  virtual void Visit(const ExtractExpression& extract) = 0;
  virtual void Visit(const RegexpMatchingExpression& match) = 0;
  virtual void Visit(const EnumInExpression& in_expr) = 0;
};

class Expression {
 public:
  Expression(const catalog::Type& type, bool nullable, std::vector<std::unique_ptr<Expression>> children)
      : type_(type), nullable_(nullable), children_(std::move(children)) {}
  virtual ~Expression() = default;
  std::vector<std::reference_wrapper<const Expression>> Children() const {
    std::vector<std::reference_wrapper<const Expression>> out;
    for (const auto& c : children_) out.push_back(*c);
    return out;
  }
  const catalog::Type& Type() const { return type_; }
  bool Nullable() const { return nullable_; }
  virtual void Accept(ImmutableExpressionVisitor& visitor) const = 0;

 protected:
  // derived classes set their type after taking their children (a type
  // computed from a child in the same constructor call as the child's move
  // would read a moved-from pointer)
  void SetType(const catalog::Type& t, bool nullable) {
    type_ = t;
    nullable_ = nullable;
  }

 private:
  catalog::Type type_;
  bool nullable_;

 protected:
  std::vector<std::unique_ptr<Expression>> children_;
};

inline std::vector<std::unique_ptr<Expression>> One(std::unique_ptr<Expression> e) {
  std::vector<std::unique_ptr<Expression>> v;
  v.push_back(std::move(e));
  return v;
}

class UnaryExpression : public Expression {
 public:
  UnaryExpression(const catalog::Type& type, bool nullable, std::unique_ptr<Expression> child)
      : Expression(type, nullable, One(std::move(child))) {}
  const Expression& Child() const { return *children_[0]; }
};

class BinaryExpression : public Expression {
 public:
  BinaryExpression(const catalog::Type& type, bool nullable, std::unique_ptr<Expression> l,
                   std::unique_ptr<Expression> r)
      : Expression(type, nullable, Two(std::move(l), std::move(r))) {}
  const Expression& LeftChild() const { return *children_[0]; }
  const Expression& RightChild() const { return *children_[1]; }

 private:
  static std::vector<std::unique_ptr<Expression>> Two(std::unique_ptr<Expression> a, std::unique_ptr<Expression> b) {
    std::vector<std::unique_ptr<Expression>> v;
    v.push_back(std::move(a));
    v.push_back(std::move(b));
    return v;
  }
};

class ColumnRefExpression : public Expression {
 public:
  ColumnRefExpression(const catalog::Type& type, bool nullable, int child_idx, int column_idx)
      : Expression(type, nullable, {}), child_idx_(child_idx), column_idx_(column_idx) {}
  int GetChildIdx() const { return child_idx_; }
  int GetColumnIdx() const { return column_idx_; }
  void Accept(ImmutableExpressionVisitor& v) const override { v.Visit(*this); }

 private:
  int child_idx_, column_idx_;
};

class VirtualColumnRefExpression : public Expression {
 public:
  VirtualColumnRefExpression(const catalog::Type& type, bool nullable, int column_idx)
      : Expression(type, nullable, {}), column_idx_(column_idx) {}
  int GetColumnIdx() const { return column_idx_; }
  void Accept(ImmutableExpressionVisitor& v) const override { v.Visit(*this); }

 private:
  int column_idx_;
};

// enum dictionaries of the literals built by string (the reference resolves
// them through its EnumManager)
inline std::map<int32_t, std::vector<std::string>>& EnumDicts() {
  static std::map<int32_t, std::vector<std::string>> d;
  return d;
}

class LiteralExpression : public Expression {
 public:
  explicit LiteralExpression(int16_t v) : Expression(catalog::Type::SmallInt(), false, {}), value_(v) {}
  explicit LiteralExpression(int32_t v) : Expression(catalog::Type::Int(), false, {}), value_(v) {}
  explicit LiteralExpression(int64_t v) : Expression(catalog::Type::BigInt(), false, {}), value_(v) {}
  explicit LiteralExpression(double v) : Expression(catalog::Type::Real(), false, {}), value_(v) {}
  explicit LiteralExpression(runtime::Date::DateBuilder d)
      : Expression(catalog::Type::Date(), false, {}), value_(d) {}
  explicit LiteralExpression(std::string_view v) : Expression(catalog::Type::Text(), false, {}), value_(std::string(v)) {}
  explicit LiteralExpression(bool v) : Expression(catalog::Type::Boolean(), false, {}), value_(v) {}
  LiteralExpression(int32_t enum_id, std::string_view v)
      : Expression(catalog::Type::Enum(enum_id), false, {}), value_(EnumValue{Key(enum_id, v)}) {}

  void Visit(std::function<void(int16_t, bool)> i16, std::function<void(int32_t, bool)> i32,
             std::function<void(int64_t, bool)> i64, std::function<void(double, bool)> f64,
             std::function<void(std::string, bool)> text, std::function<void(bool, bool)> boolean,
             std::function<void(runtime::Date::DateBuilder, bool)> date,
             std::function<void(int32_t, int32_t, bool)> enum_value) const {
    if (auto p = std::get_if<int16_t>(&value_)) return i16(*p, false);
    if (auto p = std::get_if<int32_t>(&value_)) return i32(*p, false);
    if (auto p = std::get_if<int64_t>(&value_)) return i64(*p, false);
    if (auto p = std::get_if<double>(&value_)) return f64(*p, false);
    if (auto p = std::get_if<std::string>(&value_)) return text(*p, false);
    if (auto p = std::get_if<bool>(&value_)) return boolean(*p, false);
    if (auto p = std::get_if<runtime::Date::DateBuilder>(&value_)) return date(*p, false);
    enum_value(Type().enum_id, std::get<EnumValue>(value_).value, false);
  }
  void Accept(ImmutableExpressionVisitor& v) const override { v.Visit(*this); }

 private:
  struct EnumValue {
    int32_t value;
  };
  static int32_t Key(int32_t enum_id, std::string_view s) {
    const auto& d = EnumDicts()[enum_id];
    for (size_t i = 0; i < d.size(); i++)
      if (d[i] == s) return static_cast<int32_t>(i);
    return -1;
  }
  std::variant<int16_t, int32_t, int64_t, double, std::string, bool, runtime::Date::DateBuilder, EnumValue> value_;
};

enum class UnaryArithmeticExpressionType { NOT, IS_NULL };

class UnaryArithmeticExpression : public UnaryExpression {
 public:
  UnaryArithmeticExpression(UnaryArithmeticExpressionType type, std::unique_ptr<Expression> child)
      : UnaryExpression(catalog::Type::Boolean(), false, std::move(child)), type_(type) {
    SetType(catalog::Type::Boolean(), type == UnaryArithmeticExpressionType::NOT ? Child().Nullable() : false);
  }
  UnaryArithmeticExpressionType OpType() const { return type_; }
  void Accept(ImmutableExpressionVisitor& v) const override { v.Visit(*this); }

 private:
  UnaryArithmeticExpressionType type_;
};

enum class BinaryArithmeticExpressionType {
  ADD, SUB, MUL, DIV, EQ, NEQ, LT, LEQ, GT, GEQ, AND, OR, STARTS_WITH, ENDS_WITH, CONTAINS
};

class BinaryArithmeticExpression : public BinaryExpression {
 public:
  BinaryArithmeticExpression(BinaryArithmeticExpressionType type, std::unique_ptr<Expression> l,
                             std::unique_ptr<Expression> r)
      : BinaryExpression(catalog::Type::Boolean(), false, std::move(l), std::move(r)), type_(type) {
    SetType(ResultType(type, LeftChild().Type()), LeftChild().Nullable() || RightChild().Nullable());
  }
  BinaryArithmeticExpressionType OpType() const { return type_; }
  void Accept(ImmutableExpressionVisitor& v) const override { v.Visit(*this); }

 private:
  static catalog::Type ResultType(BinaryArithmeticExpressionType t, const catalog::Type& left) {
    return static_cast<int>(t) >= static_cast<int>(BinaryArithmeticExpressionType::EQ) ? catalog::Type::Boolean()
                                                                                      : left;
  }
  BinaryArithmeticExpressionType type_;
};

enum class AggregateType { SUM, AVG, COUNT, MAX, MIN };

class AggregateExpression : public UnaryExpression {
 public:
  AggregateExpression(AggregateType type, std::unique_ptr<Expression> child)
      : UnaryExpression(catalog::Type::BigInt(), false, std::move(child)), type_(type) {
    SetType(ResultType(type, Child().Type()), type != AggregateType::COUNT);
  }
  AggregateType AggType() const { return type_; }
  void Accept(ImmutableExpressionVisitor& v) const override { v.Visit(*this); }

 private:
  static catalog::Type ResultType(AggregateType a, const catalog::Type& c) {
    if (a == AggregateType::COUNT) return catalog::Type::BigInt();
    if (a == AggregateType::AVG) return catalog::Type::Real();
    return c;
  }
  AggregateType type_;
};

class CaseExpression : public Expression {
 public:
  CaseExpression(std::unique_ptr<Expression> cond, std::unique_ptr<Expression> then,
                 std::unique_ptr<Expression> otherwise)
      : Expression(catalog::Type::Boolean(), false, Three(std::move(cond), std::move(then), std::move(otherwise))) {
    SetType(Then().Type(), Then().Nullable() || Else().Nullable());
  }
  const Expression& Cond() const { return *children_[0]; }
  const Expression& Then() const { return *children_[1]; }
  const Expression& Else() const { return *children_[2]; }
  void Accept(ImmutableExpressionVisitor& v) const override { v.Visit(*this); }

 private:
  static std::vector<std::unique_ptr<Expression>> Three(std::unique_ptr<Expression> a, std::unique_ptr<Expression> b,
                                                        std::unique_ptr<Expression> c) {
    std::vector<std::unique_ptr<Expression>> v;
    v.push_back(std::move(a));
    v.push_back(std::move(b));
    v.push_back(std::move(c));
    return v;
  }
};

class IntToFloatConversionExpression : public UnaryExpression {
 public:
  explicit IntToFloatConversionExpression(std::unique_ptr<Expression> child)
      : UnaryExpression(catalog::Type::Real(), false, std::move(child)) {
    SetType(catalog::Type::Real(), Child().Nullable());
  }
  void Accept(ImmutableExpressionVisitor& v) const override { v.Visit(*this); }
};

enum class ExtractValue { YEAR };

class ExtractExpression : public UnaryExpression {
 public:
  ExtractExpression(std::unique_ptr<Expression> child, ExtractValue value)
      : UnaryExpression(catalog::Type::Int(), false, std::move(child)), value_(value) {
    SetType(catalog::Type::Int(), Child().Nullable());
  }
  ExtractValue ValueToExtract() const { return value_; }
  void Accept(ImmutableExpressionVisitor& v) const override { v.Visit(*this); }

 private:
  ExtractValue value_;
};

class RegexpMatchingExpression : public UnaryExpression {
 public:
  RegexpMatchingExpression(std::unique_ptr<Expression> child, std::unique_ptr<re2::RE2> regexp)
      : UnaryExpression(catalog::Type::Boolean(), false, std::move(child)), regexp_(std::move(regexp)) {}
  void Accept(ImmutableExpressionVisitor& v) const override { v.Visit(*this); }
  re2::RE2* Regex() const { return regexp_.get(); }

 private:
  std::unique_ptr<re2::RE2> regexp_;
};

class EnumInExpression : public UnaryExpression {
 public:
  EnumInExpression(std::unique_ptr<Expression> child, std::vector<int> values)
      : UnaryExpression(catalog::Type::Boolean(), false, std::move(child)), values_(std::move(values)) {}
  const std::vector<int>& Values() const { return values_; }
  void Accept(ImmutableExpressionVisitor& v) const override { v.Visit(*this); }

 private:
  std::vector<int> values_;
};

// ---- operators ------------------------------------------------------------------
class OperatorSchemaProvider;

class OperatorSchema {
 public:
  class Column {
   public:
    Column(std::string_view name, std::unique_ptr<Expression> expr) : name_(name), expr_(std::move(expr)) {}
    std::string_view Name() const { return name_; }
    const Expression& Expr() const { return *expr_; }

   private:
    std::string name_;
    std::unique_ptr<Expression> expr_;
  };

  const std::vector<Column>& Columns() const { return columns_; }
  int GetColumnIndex(std::string_view name) const {
    for (size_t i = 0; i < columns_.size(); i++)
      if (columns_[i].Name() == name) return static_cast<int>(i);
    throw std::runtime_error("Unknown column " + std::string(name));
  }
  void AddDerivedColumn(std::string_view name, std::unique_ptr<Expression> expr) {
    columns_.emplace_back(name, std::move(expr));
  }
  void AddPassthroughColumns(const OperatorSchemaProvider& op, int child_idx = 0);
  void AddPassthroughColumns(const OperatorSchemaProvider& op, const std::vector<std::string>& columns,
                             int child_idx = 0);
  void AddVirtualPassthroughColumns(const OperatorSchema& schema, const std::vector<std::string>& columns) {
    for (const auto& n : columns) {
      const int idx = schema.GetColumnIndex(n);
      const auto& e = schema.columns_[idx].Expr();
      AddDerivedColumn(n, std::make_unique<VirtualColumnRefExpression>(e.Type(), e.Nullable(), idx));
    }
  }
  void AddGeneratedColumns(const catalog::Table& table, const std::vector<std::string>& columns) {
    for (const auto& n : columns) {
      const auto& c = table[n];
      AddDerivedColumn(n, std::make_unique<ColumnRefExpression>(c.GetType(), c.Nullable(), 0,
                                                                static_cast<int>(columns_.size())));
    }
  }

 private:
  std::vector<Column> columns_;
};

class OperatorSchemaProvider {
 public:
  virtual ~OperatorSchemaProvider() = default;
  virtual const OperatorSchema& Schema() const = 0;
};

inline void OperatorSchema::AddPassthroughColumns(const OperatorSchemaProvider& op,
                                                  const std::vector<std::string>& columns, int child_idx) {
  const OperatorSchema& s = op.Schema();
  for (const auto& n : columns) {
    const int idx = s.GetColumnIndex(n);
    const auto& e = s.columns_[idx].Expr();
    AddDerivedColumn(n, std::make_unique<ColumnRefExpression>(e.Type(), e.Nullable(), child_idx, idx));
  }
}
inline void OperatorSchema::AddPassthroughColumns(const OperatorSchemaProvider& op, int child_idx) {
  std::vector<std::string> names;
  for (const auto& c : op.Schema().Columns()) names.emplace_back(c.Name());
  AddPassthroughColumns(op, names, child_idx);
}

class ScanOperator;
class SelectOperator;
class ScanSelectOperator;
class SimdScanSelectOperator;
class OutputOperator;
class HashJoinOperator;
class SkinnerJoinOperator;
class AggregateOperator;
class GroupByAggregateOperator;
class OrderByOperator;
class CrossProductOperator;

class ImmutableOperatorVisitor {
 public:
  virtual ~ImmutableOperatorVisitor() = default;
  virtual void Visit(const ScanOperator& scan) = 0;
  virtual void Visit(const SelectOperator& select) = 0;
  virtual void Visit(const ScanSelectOperator& scan_select) = 0;
  virtual void Visit(const SimdScanSelectOperator& scan_select) = 0;
  virtual void Visit(const OutputOperator& output) = 0;
  virtual void Visit(const HashJoinOperator& hash_join) = 0;
  virtual void Visit(const SkinnerJoinOperator& skinner_join) = 0;
  virtual void Visit(const GroupByAggregateOperator& group_by_agg) = 0;
  virtual void Visit(const AggregateOperator& agg) = 0;
  virtual void Visit(const OrderByOperator& order_by) = 0;
  virtual void Visit(const CrossProductOperator& cross_product) = 0;
};

class Operator : public OperatorSchemaProvider {
 public:
  Operator(OperatorSchema schema, std::vector<std::unique_ptr<Operator>> children)
      : schema_(std::move(schema)), children_(std::move(children)) {}
  const OperatorSchema& Schema() const override { return schema_; }
  virtual void Accept(ImmutableOperatorVisitor& visitor) const = 0;
  std::vector<std::reference_wrapper<const Operator>> Children() const {
    std::vector<std::reference_wrapper<const Operator>> out;
    for (const auto& c : children_) out.push_back(*c);
    return out;
  }

 private:
  OperatorSchema schema_;

 protected:
  std::vector<std::unique_ptr<Operator>> children_;
};

inline std::vector<std::unique_ptr<Operator>> Kids(std::unique_ptr<Operator> a, std::unique_ptr<Operator> b = {}) {
  std::vector<std::unique_ptr<Operator>> v;
  if (a) v.push_back(std::move(a));
  if (b) v.push_back(std::move(b));
  return v;
}

class UnaryOperator : public Operator {
 public:
  UnaryOperator(OperatorSchema schema, std::unique_ptr<Operator> child)
      : Operator(std::move(schema), Kids(std::move(child))) {}
  const Operator& Child() const { return *children_[0]; }
};

class BinaryOperator : public Operator {
 public:
  BinaryOperator(OperatorSchema schema, std::unique_ptr<Operator> l, std::unique_ptr<Operator> r)
      : Operator(std::move(schema), Kids(std::move(l), std::move(r))) {}
  const Operator& LeftChild() const { return *children_[0]; }
  const Operator& RightChild() const { return *children_[1]; }
};

class ScanOperator final : public Operator {
 public:
  ScanOperator(OperatorSchema schema, const catalog::Table& relation)
      : Operator(std::move(schema), {}), relation_(relation) {}
  const catalog::Table& Relation() const { return relation_; }
  void Accept(ImmutableOperatorVisitor& v) const override { v.Visit(*this); }

 private:
  const catalog::Table& relation_;
};

template <typename T>
std::vector<std::reference_wrapper<const T>> Refs(const std::vector<std::unique_ptr<T>>& v) {
  std::vector<std::reference_wrapper<const T>> out;
  for (const auto& x : v) out.push_back(*x);
  return out;
}

class ScanSelectOperator : public Operator {
 public:
  ScanSelectOperator(OperatorSchema schema, OperatorSchema scan_schema, const catalog::Table& relation,
                     std::vector<std::unique_ptr<Expression>> filters)
      : Operator(std::move(schema), {}), scan_schema_(std::move(scan_schema)), relation_(relation),
        filters_(std::move(filters)) {}
  const catalog::Table& Relation() const { return relation_; }
  const OperatorSchema& ScanSchema() const { return scan_schema_; }
  std::vector<std::reference_wrapper<const Expression>> Filters() const { return Refs(filters_); }
  void Accept(ImmutableOperatorVisitor& v) const override { v.Visit(*this); }

 private:
  OperatorSchema scan_schema_;
  const catalog::Table& relation_;
  std::vector<std::unique_ptr<Expression>> filters_;
};

class SimdScanSelectOperator final : public ScanSelectOperator {
 public:
  using ScanSelectOperator::ScanSelectOperator;
  void Accept(ImmutableOperatorVisitor& v) const override { v.Visit(*this); }
};

class SelectOperator final : public UnaryOperator {
 public:
  SelectOperator(OperatorSchema schema, std::unique_ptr<Operator> child, std::unique_ptr<Expression> expr)
      : UnaryOperator(std::move(schema), std::move(child)), expr_(std::move(expr)) {}
  const Expression& Expr() const { return *expr_; }
  void Accept(ImmutableOperatorVisitor& v) const override { v.Visit(*this); }

 private:
  std::unique_ptr<Expression> expr_;
};

class OutputOperator final : public UnaryOperator {
 public:
  explicit OutputOperator(std::unique_ptr<Operator> child) : UnaryOperator(OperatorSchema(), std::move(child)) {}
  void Accept(ImmutableOperatorVisitor& v) const override { v.Visit(*this); }
};

class HashJoinOperator final : public BinaryOperator {
 public:
  HashJoinOperator(OperatorSchema schema, std::unique_ptr<Operator> l, std::unique_ptr<Operator> r,
                   std::vector<std::unique_ptr<ColumnRefExpression>> left_columns,
                   std::vector<std::unique_ptr<ColumnRefExpression>> right_columns)
      : BinaryOperator(std::move(schema), std::move(l), std::move(r)), left_(std::move(left_columns)),
        right_(std::move(right_columns)) {}
  std::vector<std::reference_wrapper<const ColumnRefExpression>> LeftColumns() const { return Refs(left_); }
  std::vector<std::reference_wrapper<const ColumnRefExpression>> RightColumns() const { return Refs(right_); }
  void Accept(ImmutableOperatorVisitor& v) const override { v.Visit(*this); }

 private:
  std::vector<std::unique_ptr<ColumnRefExpression>> left_, right_;
};

class SkinnerJoinOperator final : public Operator {
 public:
  SkinnerJoinOperator(OperatorSchema schema, std::vector<std::unique_ptr<Operator>> children,
                      std::vector<std::unique_ptr<Expression>> conditions, std::vector<int> prefix_order = {})
      : Operator(std::move(schema), std::move(children)), conditions_(std::move(conditions)),
        prefix_order_(std::move(prefix_order)) {}
  std::vector<std::reference_wrapper<const Expression>> Conditions() const { return Refs(conditions_); }
  const std::vector<int>& PrefixOrder() const { return prefix_order_; }
  void Accept(ImmutableOperatorVisitor& v) const override { v.Visit(*this); }

 private:
  std::vector<std::unique_ptr<Expression>> conditions_;
  std::vector<int> prefix_order_;
};

class GroupByAggregateOperator final : public UnaryOperator {
 public:
  GroupByAggregateOperator(OperatorSchema schema, std::unique_ptr<Operator> child,
                           std::vector<std::unique_ptr<Expression>> group_by,
                           std::vector<std::unique_ptr<AggregateExpression>> aggs)
      : UnaryOperator(std::move(schema), std::move(child)), group_by_(std::move(group_by)), aggs_(std::move(aggs)) {}
  std::vector<std::reference_wrapper<const Expression>> GroupByExprs() const { return Refs(group_by_); }
  std::vector<std::reference_wrapper<const AggregateExpression>> AggExprs() const { return Refs(aggs_); }
  void Accept(ImmutableOperatorVisitor& v) const override { v.Visit(*this); }

 private:
  std::vector<std::unique_ptr<Expression>> group_by_;
  std::vector<std::unique_ptr<AggregateExpression>> aggs_;
};

class AggregateOperator final : public UnaryOperator {
 public:
  AggregateOperator(OperatorSchema schema, std::unique_ptr<Operator> child,
                    std::vector<std::unique_ptr<AggregateExpression>> aggs)
      : UnaryOperator(std::move(schema), std::move(child)), aggs_(std::move(aggs)) {}
  std::vector<std::reference_wrapper<const AggregateExpression>> AggExprs() const { return Refs(aggs_); }
  void Accept(ImmutableOperatorVisitor& v) const override { v.Visit(*this); }

 private:
  std::vector<std::unique_ptr<AggregateExpression>> aggs_;
};

class OrderByOperator final : public UnaryOperator {
 public:
  OrderByOperator(OperatorSchema schema, std::unique_ptr<Operator> child,
                  std::vector<std::unique_ptr<ColumnRefExpression>> keys, std::vector<bool> asc)
      : UnaryOperator(std::move(schema), std::move(child)), keys_(std::move(keys)), asc_(std::move(asc)) {}
  std::vector<std::reference_wrapper<const ColumnRefExpression>> KeyExprs() const { return Refs(keys_); }
  const std::vector<bool>& Ascending() const { return asc_; }
  void Accept(ImmutableOperatorVisitor& v) const override { v.Visit(*this); }

 private:
  std::vector<std::unique_ptr<ColumnRefExpression>> keys_;
  std::vector<bool> asc_;
};

class CrossProductOperator final : public Operator {
 public:
  using Operator::Operator;
  void Accept(ImmutableOperatorVisitor& v) const override { v.Visit(*this); }
};

}  // namespace kush::plan
