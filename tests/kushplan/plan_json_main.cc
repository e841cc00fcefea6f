// Builds the benchmark plans (scan-select + aggregate, Q1-shape group-by,
// Q3-shape join + group-by + order-by, a Skinner star join with LIKE
// filters, and a plan with CASE / EXTRACT / IN / IS NULL / SELECT) with the
// plan classes KushDB uses, serialises each with kdb_b200::ToBackendJson and
// prints one JSON document per line.  tests/test_plan_json.py compiles this
// against the class subset in plan_subset.h and compares every line with
// the JSON that kushdb_b200/plan.py writes for the same plan.
#include <cstdio>
#include <iostream>

#include "kdb_plan_json.h"

using namespace kush;
using namespace kush::plan;
using catalog::Type;
using B = BinaryArithmeticExpressionType;

namespace {

constexpr int32_t kEpochJdn = 2440588;

// civil date of `days` since 1970-01-01 (proleptic Gregorian)
runtime::Date::DateBuilder CivilFromDays(int64_t days) {
  days += 719468;
  const int64_t era = (days >= 0 ? days : days - 146096) / 146097;
  const int64_t doe = days - era * 146097;
  const int64_t yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
  const int64_t doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
  const int64_t mp = (5 * doy + 2) / 153;
  const int64_t d = doy - (153 * mp + 2) / 5 + 1;
  const int64_t m = mp < 10 ? mp + 3 : mp - 9;
  const int64_t y = yoe + era * 400 + (m <= 2);
  return runtime::Date::DateBuilder(static_cast<int32_t>(y), static_cast<int32_t>(m), static_cast<int32_t>(d));
}

std::unique_ptr<Expression> ColRef(const Operator& op, const std::string& col, int child_idx = 0) {
  const int idx = op.Schema().GetColumnIndex(col);
  const auto& e = op.Schema().Columns()[idx].Expr();
  return std::make_unique<ColumnRefExpression>(e.Type(), e.Nullable(), child_idx, idx);
}
std::unique_ptr<ColumnRefExpression> KeyRef(const Operator& op, const std::string& col, int child_idx = 0) {
  const int idx = op.Schema().GetColumnIndex(col);
  const auto& e = op.Schema().Columns()[idx].Expr();
  return std::make_unique<ColumnRefExpression>(e.Type(), e.Nullable(), child_idx, idx);
}
std::unique_ptr<Expression> VirtColRef(const OperatorSchema& s, const std::string& col) {
  const int idx = s.GetColumnIndex(col);
  const auto& e = s.Columns()[idx].Expr();
  return std::make_unique<VirtualColumnRefExpression>(e.Type(), e.Nullable(), idx);
}
std::unique_ptr<Expression> VirtColRef(const Expression& e, int idx) {
  return std::make_unique<VirtualColumnRefExpression>(e.Type(), e.Nullable(), idx);
}
std::unique_ptr<Expression> Bin(B op, std::unique_ptr<Expression> l, std::unique_ptr<Expression> r) {
  return std::make_unique<BinaryArithmeticExpression>(op, std::move(l), std::move(r));
}
std::unique_ptr<Expression> Lit(double v) { return std::make_unique<LiteralExpression>(v); }
std::unique_ptr<Expression> DateLit(int64_t days_since_epoch) {
  return std::make_unique<LiteralExpression>(CivilFromDays(days_since_epoch));
}
std::unique_ptr<AggregateExpression> Agg(AggregateType a, std::unique_ptr<Expression> c) {
  return std::make_unique<AggregateExpression>(a, std::move(c));
}
std::unique_ptr<AggregateExpression> Count() {
  return Agg(AggregateType::COUNT, std::make_unique<LiteralExpression>(true));
}
template <typename T>
std::vector<std::unique_ptr<T>> Vec(std::unique_ptr<T> a) {
  std::vector<std::unique_ptr<T>> v;
  v.push_back(std::move(a));
  return v;
}

// scan_agg_plan (workloads.py): sales, date < 9300, 0.05 <= discount <= 0.07
std::string ScanAgg(const catalog::Database& db) {
  const auto& rel = db["sales"];
  OperatorSchema scan;
  scan.AddGeneratedColumns(rel, {"s_date", "s_discount", "s_price"});
  std::vector<std::unique_ptr<Expression>> filters;
  filters.push_back(Bin(B::LT, VirtColRef(scan, "s_date"), DateLit(9300)));
  filters.push_back(Bin(B::GEQ, VirtColRef(scan, "s_discount"), Lit(0.05)));
  filters.push_back(Bin(B::LEQ, VirtColRef(scan, "s_discount"), Lit(0.07)));
  OperatorSchema out;
  out.AddVirtualPassthroughColumns(scan, {"s_price", "s_discount"});
  auto sel = std::make_unique<ScanSelectOperator>(std::move(out), std::move(scan), rel, std::move(filters));
  auto revenue = Agg(AggregateType::SUM, Bin(B::MUL, ColRef(*sel, "s_price"), ColRef(*sel, "s_discount")));
  auto cnt = Count();
  OperatorSchema schema;
  schema.AddDerivedColumn("revenue", VirtColRef(*revenue, 0));
  schema.AddDerivedColumn("count", VirtColRef(*cnt, 1));
  std::vector<std::unique_ptr<AggregateExpression>> aggs;
  aggs.push_back(std::move(revenue));
  aggs.push_back(std::move(cnt));
  OutputOperator root(std::make_unique<AggregateOperator>(std::move(schema), std::move(sel), std::move(aggs)));
  return kdb_b200::ToBackendJson(root);
}

// group_by_plan (workloads.py): Q1 shape
std::string GroupBy(const catalog::Database& db) {
  const auto& rel = db["lineitem_q1"];
  const std::vector<std::string> cols = {"l_returnflag", "l_linestatus", "l_quantity", "l_extendedprice",
                                         "l_discount", "l_tax", "l_shipdate"};
  OperatorSchema scan;
  scan.AddGeneratedColumns(rel, cols);
  std::vector<std::unique_ptr<Expression>> filters;
  filters.push_back(Bin(B::LEQ, VirtColRef(scan, "l_shipdate"), DateLit(10471)));
  OperatorSchema out;
  out.AddVirtualPassthroughColumns(scan, std::vector<std::string>(cols.begin(), cols.end() - 1));
  auto sel = std::make_unique<ScanSelectOperator>(std::move(out), std::move(scan), rel, std::move(filters));
  auto rf = ColRef(*sel, "l_returnflag");
  auto ls = ColRef(*sel, "l_linestatus");
  auto disc_price = [&]() {
    return Bin(B::MUL, ColRef(*sel, "l_extendedprice"), Bin(B::SUB, Lit(1.0), ColRef(*sel, "l_discount")));
  };
  std::vector<std::unique_ptr<AggregateExpression>> aggs;
  aggs.push_back(Agg(AggregateType::SUM, ColRef(*sel, "l_quantity")));
  aggs.push_back(Agg(AggregateType::SUM, ColRef(*sel, "l_extendedprice")));
  aggs.push_back(Agg(AggregateType::SUM, disc_price()));
  aggs.push_back(Agg(AggregateType::SUM, Bin(B::MUL, disc_price(), Bin(B::ADD, Lit(1.0), ColRef(*sel, "l_tax")))));
  aggs.push_back(Agg(AggregateType::AVG, ColRef(*sel, "l_quantity")));
  aggs.push_back(Agg(AggregateType::AVG, ColRef(*sel, "l_extendedprice")));
  aggs.push_back(Agg(AggregateType::AVG, ColRef(*sel, "l_discount")));
  aggs.push_back(Count());
  OperatorSchema g;
  g.AddDerivedColumn("l_returnflag", VirtColRef(*rf, 0));
  g.AddDerivedColumn("l_linestatus", VirtColRef(*ls, 1));
  const char* names[] = {"sum_qty", "sum_base_price", "sum_disc_price", "sum_charge", "avg_qty", "avg_price",
                         "avg_disc", "count_order"};
  for (int i = 0; i < 8; i++) g.AddDerivedColumn(names[i], VirtColRef(*aggs[i], i + 2));
  std::vector<std::unique_ptr<Expression>> keys;
  keys.push_back(std::move(rf));
  keys.push_back(std::move(ls));
  auto agg = std::make_unique<GroupByAggregateOperator>(std::move(g), std::move(sel), std::move(keys), std::move(aggs));
  OperatorSchema o;
  o.AddPassthroughColumns(*agg);
  std::vector<std::unique_ptr<ColumnRefExpression>> sort;
  sort.push_back(KeyRef(*agg, "l_returnflag"));
  sort.push_back(KeyRef(*agg, "l_linestatus"));
  OutputOperator root(
      std::make_unique<OrderByOperator>(std::move(o), std::move(agg), std::move(sort), std::vector<bool>{true, true}));
  return kdb_b200::ToBackendJson(root);
}

// join_plan (workloads.py): Q3 shape
std::string Join(const catalog::Database& db) {
  const auto& brel = db["customer_q3"];
  const auto& prel = db["orders_q3"];
  OperatorSchema bs;
  bs.AddGeneratedColumns(brel, {"c_custkey", "c_date", "c_segment"});
  std::vector<std::unique_ptr<Expression>> bf;
  bf.push_back(Bin(B::LT, VirtColRef(bs, "c_date"), DateLit(9204)));
  bf.push_back(Bin(B::EQ, VirtColRef(bs, "c_segment"), std::make_unique<LiteralExpression>(102, "BUILDING")));
  OperatorSchema bout;
  bout.AddVirtualPassthroughColumns(bs, {"c_custkey"});
  auto bsel = std::make_unique<ScanSelectOperator>(std::move(bout), std::move(bs), brel, std::move(bf));
  OperatorSchema ps;
  ps.AddGeneratedColumns(prel, {"o_custkey", "o_price", "o_discount"});
  auto pscan = std::make_unique<ScanOperator>(std::move(ps), prel);
  OperatorSchema js;
  js.AddPassthroughColumns(*bsel, {"c_custkey"}, 0);
  js.AddPassthroughColumns(*pscan, {"o_price", "o_discount"}, 1);
  auto lk = Vec(KeyRef(*bsel, "c_custkey", 0));
  auto rk = Vec(KeyRef(*pscan, "o_custkey", 1));
  auto join = std::make_unique<HashJoinOperator>(std::move(js), std::move(bsel), std::move(pscan), std::move(lk),
                                                 std::move(rk));
  auto key = ColRef(*join, "c_custkey");
  auto revenue = Agg(AggregateType::SUM, Bin(B::MUL, ColRef(*join, "o_price"),
                                             Bin(B::SUB, Lit(1.0), ColRef(*join, "o_discount"))));
  OperatorSchema gs;
  gs.AddDerivedColumn("c_custkey", VirtColRef(*key, 0));
  gs.AddDerivedColumn("revenue", VirtColRef(*revenue, 1));
  auto agg = std::make_unique<GroupByAggregateOperator>(std::move(gs), std::move(join), Vec(std::move(key)),
                                                        Vec(std::move(revenue)));
  OperatorSchema os;
  os.AddPassthroughColumns(*agg);
  auto sort = Vec(KeyRef(*agg, "revenue"));
  OutputOperator root(
      std::make_unique<OrderByOperator>(std::move(os), std::move(agg), std::move(sort), std::vector<bool>{false}));
  return kdb_b200::ToBackendJson(root);
}

// skinner_plan (workloads.py), star of 3 tables, LIKE on tables 1 and 2
std::string Skinner(const catalog::Database& db) {
  std::vector<std::unique_ptr<Operator>> children;
  const char* toks[] = {"abc", "XYZ", "q!r"};
  for (int i = 0; i < 3; i++) {
    const auto& rel = db["sk" + std::to_string(i)];
    std::vector<std::string> cols = {"pk"};
    if (i == 0) cols = {"pk", "fk1", "fk2"};
    OperatorSchema scan;
    std::vector<std::string> scols = cols;
    if (i > 0) scols.push_back("note");
    scan.AddGeneratedColumns(rel, scols);
    std::vector<std::unique_ptr<Expression>> filters;
    if (i > 0)
      filters.push_back(Bin(B::CONTAINS, VirtColRef(scan, "note"), std::make_unique<LiteralExpression>(std::string_view(toks[i]))));
    OperatorSchema out;
    out.AddVirtualPassthroughColumns(scan, cols);
    children.push_back(std::make_unique<ScanSelectOperator>(std::move(out), std::move(scan), rel, std::move(filters)));
  }
  std::vector<std::unique_ptr<Expression>> conds;
  for (int i = 1; i < 3; i++)
    conds.push_back(Bin(B::EQ, ColRef(*children[0], "fk" + std::to_string(i), 0), ColRef(*children[i], "pk", i)));
  OperatorSchema js;
  js.AddPassthroughColumns(*children[0], {"pk"}, 0);
  auto join = std::make_unique<SkinnerJoinOperator>(std::move(js), std::move(children), std::move(conds));
  auto cnt = Count();
  auto mn = Agg(AggregateType::MIN, ColRef(*join, "pk"));
  OperatorSchema s;
  s.AddDerivedColumn("count", VirtColRef(*cnt, 0));
  s.AddDerivedColumn("min_pk", VirtColRef(*mn, 1));
  std::vector<std::unique_ptr<AggregateExpression>> aggs;
  aggs.push_back(std::move(cnt));
  aggs.push_back(std::move(mn));
  OutputOperator root(std::make_unique<AggregateOperator>(std::move(s), std::move(join), std::move(aggs)));
  return kdb_b200::ToBackendJson(root);
}

// SELECT over a scan with CASE, EXTRACT, enum IN, IS NULL, NOT and LIKE
std::string Misc(const catalog::Database& db) {
  const auto& rel = db["misc"];
  OperatorSchema ss;
  ss.AddGeneratedColumns(rel, {"d", "c", "v", "n"});
  auto scan = std::make_unique<ScanOperator>(std::move(ss), rel);
  auto cond = Bin(B::OR, std::make_unique<EnumInExpression>(ColRef(*scan, "c"), std::vector<int>{0, 2}),
                  std::make_unique<UnaryArithmeticExpression>(
                      UnaryArithmeticExpressionType::NOT,
                      std::make_unique<UnaryArithmeticExpression>(UnaryArithmeticExpressionType::IS_NULL,
                                                                  ColRef(*scan, "n"))));
  OperatorSchema out;
  out.AddDerivedColumn("y", std::make_unique<ExtractExpression>(ColRef(*scan, "d"), ExtractValue::YEAR));
  out.AddDerivedColumn("w", std::make_unique<CaseExpression>(Bin(B::GT, ColRef(*scan, "v"), Lit(0.5)),
                                                             std::make_unique<IntToFloatConversionExpression>(
                                                                 ColRef(*scan, "n")),
                                                             Lit(-1.25)));
  // LIKE '%(B)%_N%' on an enum, as the planner writes it
  out.AddDerivedColumn("m", std::make_unique<RegexpMatchingExpression>(
                                ColRef(*scan, "c"), std::make_unique<re2::RE2>("^.*\\(B\\).*.N.*$")));
  OutputOperator root(std::make_unique<SelectOperator>(std::move(out), std::move(scan), std::move(cond)));
  return kdb_b200::ToBackendJson(root);
}

}  // namespace

int main() {
  EnumDicts()[102] = {"AUTOMOBILE", "BUILDING", "FURNITURE", "HOUSEHOLD", "MACHINERY"};
  catalog::Database db;
  auto& sales = db.Insert("sales");
  sales.Insert("s_key", Type::Int(), "", "", "");
  sales.Insert("s_price", Type::Real(), "", "", "");
  sales.Insert("s_discount", Type::Real(), "", "", "");
  sales.Insert("s_date", Type::Date(), "", "", "");
  auto& li = db.Insert("lineitem_q1");
  li.Insert("l_shipdate", Type::Date(), "", "", "");
  li.Insert("l_returnflag", Type::Enum(100), "", "", "");
  li.Insert("l_linestatus", Type::Enum(101), "", "", "");
  for (const char* c : {"l_quantity", "l_extendedprice", "l_discount", "l_tax"}) li.Insert(c, Type::Real(), "", "", "");
  auto& cu = db.Insert("customer_q3");
  cu.Insert("c_custkey", Type::Int(), "", "", "");
  cu.Insert("c_date", Type::Date(), "", "", "");
  cu.Insert("c_segment", Type::Enum(102), "", "", "");
  auto& ord = db.Insert("orders_q3");
  ord.Insert("o_custkey", Type::Int(), "", "", "");
  ord.Insert("o_price", Type::Real(), "", "", "");
  ord.Insert("o_discount", Type::Real(), "", "", "");
  for (int i = 0; i < 3; i++) {
    auto& t = db.Insert("sk" + std::to_string(i));
    t.Insert("pk", Type::Int(), "", "", "");
    t.Insert("note", Type::Text(), "", "", "");
    if (i == 0) {
      t.Insert("fk1", Type::Int(), "", "", "");
      t.Insert("fk2", Type::Int(), "", "", "");
    }
  }
  auto& misc = db.Insert("misc");
  misc.Insert("d", Type::Date(), "", "null", "");
  misc.Insert("c", Type::Enum(102), "", "", "");
  misc.Insert("v", Type::Real(), "", "", "");
  misc.Insert("n", Type::Int(), "", "null", "");
  std::cout << ScanAgg(db) << "\n" << GroupBy(db) << "\n" << Join(db) << "\n" << Skinner(db) << "\n"
            << Misc(db) << "\n";
  return 0;
}
