"""The reference's end-to-end test plans, restated with the Python plan builder.

Each case mirrors one ``end_to_end_test/<operator>/<type>_test.cc`` (or
``end_to_end_test/tpch/qNN_test.cc``) of the reference: same operators, same
expressions, same expected table, same comparison:

* ``sorted``  -- both sides sorted as line multisets, then compared exactly
  (e.g. end_to_end_test/hash_join/int_test.cc:72-79);
* ``ordered`` -- compared line by line exactly (order_by/*_test.cc);
  ``desc`` cases reverse the expected file first (order_by/int_test.cc:69-71);
* ``tbl``     -- CHECK_EQ_TBL (util/test_util.h:82-175): ordered, REAL within
  1e-5 absolute.
"""

from __future__ import annotations

import os
from dataclasses import dataclass
from typing import Callable, Dict, List

from kushdb_b200.data import HostTable, catalog_of, load_golden
from kushdb_b200.plan import (INT_MIN, INT_MAX, And, Avg, BigIntLiteral, Case, ColRef, ColRefE,
                              Count, Eq, Geq, GroupByAggregateOperator, Gt, HashJoinOperator,
                              Leq, Literal, Lt, Max, Min, Mul, OperatorSchema, OrderByOperator,
                              OutputOperator, ScanOperator, ScanSelectOperator, SelectOperator,
                              SkinnerJoinOperator, SmallIntLiteral, Sub, Add, Sum, VirtColRef,
                              AggregateOperator, SimdScanSelectOperator, CrossProductOperator)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

_TABLES: Dict[str, HostTable] = {}


def golden_tables() -> Dict[str, HostTable]:
    if not _TABLES:
        _TABLES.update(load_golden(GOLDEN))
    return _TABLES


def db():
    return catalog_of(golden_tables().values())


@dataclass
class Case_:
    name: str
    build: Callable
    expected: str
    mode: str          # sorted | ordered | tbl
    desc: bool = False

    def expected_lines(self) -> List[str]:
        with open(os.path.join(GOLDEN, "expected", self.expected)) as f:
            lines = f.read().split("\n")
        if lines and lines[-1] == "":
            lines.pop()
        if self.desc:
            lines.reverse()
        return lines


# ---------------------------------------------------------------------------
# scan_select/*, simd_scan_select/*, select/*
# ---------------------------------------------------------------------------


def _scan_select(relation, cols, filters, out_cols=None, simd=False):
    d = db()
    scan_schema = OperatorSchema()
    scan_schema.AddGeneratedColumns(d[relation], cols)
    fs = [f(scan_schema) for f in filters]
    schema = OperatorSchema()
    schema.AddVirtualPassthroughColumns(scan_schema, out_cols or cols)
    cls = SimdScanSelectOperator if simd else ScanSelectOperator
    return OutputOperator(cls(schema, scan_schema, d[relation], fs))


def _select(relation, col, make_filter):
    d = db()
    s = OperatorSchema()
    s.AddGeneratedColumns(d[relation], [col])
    base = ScanOperator(s, d[relation])
    schema = OperatorSchema()
    schema.AddPassthroughColumns(base)
    return OutputOperator(SelectOperator(schema, base, make_filter(base)))


V = VirtColRef
CASES: List[Case_] = []


def _add(name, build, expected, mode, desc=False):
    CASES.append(Case_(name, build, expected, mode, desc))


_add("scan_select/bigint", lambda: _scan_select("info", ["num2"], [lambda s: Gt(V(s, "num2"), BigIntLiteral(0))]),
     "scan_select/bigint_expected.tbl", "sorted")
_add("scan_select/boolean_eq", lambda: _scan_select("info", ["cheated"], [lambda s: Eq(V(s, "cheated"), Literal(True))]),
     "scan_select/boolean_eq_expected.tbl", "sorted")
_add("scan_select/boolean", lambda: _scan_select("info", ["cheated"], [lambda s: V(s, "cheated")]),
     "scan_select/boolean_expected.tbl", "sorted")
_add("scan_select/date", lambda: _scan_select("info", ["date"], [lambda s: Geq(V(s, "date"), Literal(2021, 1, 1))]),
     "scan_select/date_expected.tbl", "sorted")
_add("scan_select/enum", lambda: _scan_select("people_enum", ["name"], [lambda s: Gt(V(s, "name"), Literal("M"))]),
     "scan_select/enum_expected.tbl", "sorted")
_add("scan_select/int_eq", lambda: _scan_select("customer", ["c_custkey"], [lambda s: Eq(V(s, "c_custkey"), Literal(555))]),
     "scan_select/int_eq_expected.tbl", "sorted")
_add("scan_select/int", lambda: _scan_select("info", ["id"], [lambda s: Gt(V(s, "id"), Literal(29))]),
     "scan_select/int_expected.tbl", "sorted")
_add("scan_select/multiple_eq", lambda: _scan_select(
    "info", ["cheated", "date"],
    [lambda s: Eq(V(s, "cheated"), Literal(True)), lambda s: Eq(V(s, "date"), Literal(2021, 1, 29))]),
    "scan_select/multiple_eq_expected.tbl", "sorted")
_add("scan_select/real", lambda: _scan_select("info", ["zscore"], [lambda s: Gt(V(s, "zscore"), Literal(-0.5))]),
     "scan_select/real_expected.tbl", "sorted")
_add("scan_select/smallint", lambda: _scan_select("info", ["num1"], [lambda s: Lt(V(s, "num1"), SmallIntLiteral(0))]),
     "scan_select/smallint_expected.tbl", "sorted")
_add("scan_select/text", lambda: _scan_select("people", ["name"], [lambda s: Gt(V(s, "name"), Literal("M"))]),
     "scan_select/text_expected.tbl", "sorted")

_add("simd_scan_select/date_range", lambda: _scan_select(
    "lineitem_enum", ["l_shipdate"],
    [lambda s: Leq(V(s, "l_shipdate"), Literal(1998, 12, 31)), lambda s: Geq(V(s, "l_shipdate"), Literal(1998, 1, 1))],
    simd=True), "simd_scan_select/date_range_expected.tbl", "sorted")
_add("simd_scan_select/date", lambda: _scan_select(
    "lineitem_enum", ["l_shipdate"], [lambda s: Leq(V(s, "l_shipdate"), Literal(1998, 9, 13))], simd=True),
    "simd_scan_select/date_expected.tbl", "sorted")
_add("simd_scan_select/enum", lambda: _scan_select(
    "lineitem_enum", ["l_returnflag"], [lambda s: Eq(V(s, "l_returnflag"), Literal("R"))], simd=True),
    "simd_scan_select/enum_expected.tbl", "sorted")
_add("simd_scan_select/int", lambda: _scan_select(
    "nation", ["n_nationkey"], [lambda s: Gt(V(s, "n_nationkey"), Literal(5))], simd=True),
    "simd_scan_select/int_expected.tbl", "sorted")


def _simd_multiple_col():
    return _scan_select(
        "lineitem_enum", ["l_shipdate", "l_returnflag"],
        [lambda s: Leq(V(s, "l_shipdate"), Literal(1994, 12, 31)),
         lambda s: Geq(V(s, "l_shipdate"), Literal(1994, 1, 1)),
         lambda s: Eq(V(s, "l_returnflag"), Literal("R"))], simd=True)


_add("simd_scan_select/multiple_col", _simd_multiple_col, "simd_scan_select/multiple_col_expected.tbl", "sorted")

_add("select/bigint", lambda: _select("info", "num2", lambda b: Gt(ColRef(b, "num2"), BigIntLiteral(0))),
     "select/bigint_expected.tbl", "sorted")
_add("select/boolean", lambda: _select("info", "cheated", lambda b: ColRef(b, "cheated")),
     "select/boolean_expected.tbl", "sorted")
_add("select/date", lambda: _select("info", "date", lambda b: Geq(ColRef(b, "date"), Literal(2021, 1, 1))),
     "select/date_expected.tbl", "sorted")
_add("select/enum", lambda: _select("people_enum", "name", lambda b: Gt(ColRef(b, "name"), Literal("M"))),
     "select/enum_expected.tbl", "sorted")
_add("select/int", lambda: _select("info", "id", lambda b: Gt(ColRef(b, "id"), Literal(29))),
     "select/int_expected.tbl", "sorted")
_add("select/real", lambda: _select("info", "zscore", lambda b: Gt(ColRef(b, "zscore"), Literal(-0.5))),
     "select/real_expected.tbl", "sorted")
_add("select/smallint", lambda: _select("info", "num1", lambda b: Lt(ColRef(b, "num1"), SmallIntLiteral(0))),
     "select/smallint_expected.tbl", "sorted")
_add("select/text", lambda: _select("people", "name", lambda b: Gt(ColRef(b, "name"), Literal("M"))),
     "select/text_expected.tbl", "sorted")


# ---------------------------------------------------------------------------
# aggregate/*, group_by_aggregate/*
# ---------------------------------------------------------------------------


def _aggregate(empty: bool):
    d = db()
    s = OperatorSchema()
    s.AddGeneratedColumns(d["info"], ["cheated", "id"])
    base = ScanOperator(s, d["info"])
    if empty:
        # aggregate/empty_test.cc: Select(false) under the aggregate
        sel_schema = OperatorSchema()
        sel_schema.AddPassthroughColumns(base)
        base = SelectOperator(sel_schema, base, Literal(False))
    aggs = [Sum(ColRef(base, "id")), Min(ColRef(base, "id")), Max(ColRef(base, "id")),
            Avg(ColRef(base, "id")), Count(), Count(ColRef(base, "id"))]
    schema = OperatorSchema()
    for i, n in enumerate(["sum", "min", "max", "avg", "count1", "count2"]):
        schema.AddDerivedColumn(n, VirtColRef(aggs[i], i))
    return OutputOperator(AggregateOperator(schema, base, aggs))


_add("aggregate/int", lambda: _aggregate(False), "aggregate/int_expected.tbl", "sorted")
_add("aggregate/empty", lambda: _aggregate(True), "aggregate/empty_expected.tbl", "sorted")


def _group_by(relation, cols, key_fn, agg_col, numeric: bool):
    d = db()
    s = OperatorSchema()
    s.AddGeneratedColumns(d[relation], cols)
    base = ScanOperator(s, d[relation])
    key = key_fn(base)
    if numeric:
        aggs = [Sum(ColRef(base, agg_col)), Min(ColRef(base, agg_col)), Max(ColRef(base, agg_col)),
                Avg(ColRef(base, agg_col)), Count(), Count(ColRef(base, agg_col))]
        names = ["sum", "min", "max", "avg", "count1", "count2"]
    else:
        aggs = [Min(ColRef(base, agg_col)), Max(ColRef(base, agg_col)), Count(),
                Count(ColRef(base, agg_col))]
        names = ["min", "max", "count1", "count2"]
    schema = OperatorSchema()
    for i, n in enumerate(names):
        schema.AddDerivedColumn(n, VirtColRef(aggs[i], i + 1))
    return OutputOperator(GroupByAggregateOperator(schema, base, [key], aggs))


_add("group_by_aggregate/bigint", lambda: _group_by(
    "info", ["cheated", "num2"],
    lambda b: Case(ColRefE(b, "cheated"), BigIntLiteral(2**63 - 1), BigIntLiteral(-2**63)), "num2", True),
    "group_by_aggregate/bigint_expected.tbl", "sorted")
_add("group_by_aggregate/date", lambda: _group_by(
    "info", ["cheated", "date"],
    lambda b: Case(ColRefE(b, "cheated"), Literal(1993, 1, 1), Literal(1200, 12, 31)), "date", False),
    "group_by_aggregate/date_expected.tbl", "sorted")
_add("group_by_aggregate/enum", lambda: _group_by(
    "people_enum", ["name"], lambda b: ColRef(b, "name"), "name", False),
    "group_by_aggregate/enum_expected.tbl", "sorted")
_add("group_by_aggregate/int", lambda: _group_by(
    "info", ["cheated", "id"],
    lambda b: Case(ColRefE(b, "cheated"), Literal(INT_MIN), Literal(INT_MAX)), "id", True),
    "group_by_aggregate/int_expected.tbl", "sorted")
_add("group_by_aggregate/real", lambda: _group_by(
    "info", ["cheated", "zscore"],
    lambda b: Case(ColRefE(b, "cheated"), Literal(2.2250738585072014e-308), Literal(1.7976931348623157e308)),
    "zscore", True),
    "group_by_aggregate/real_expected.tbl", "sorted")
_add("group_by_aggregate/smallint", lambda: _group_by(
    "info", ["cheated", "num1"],
    lambda b: Case(ColRefE(b, "cheated"), SmallIntLiteral(-32768), SmallIntLiteral(32767)), "num1", True),
    "group_by_aggregate/smallint_expected.tbl", "sorted")
_add("group_by_aggregate/text", lambda: _group_by(
    "people", ["id", "name"],
    lambda b: Case(Gt(ColRef(b, "id"), Literal(500)), Literal("hello"), Literal("")), "name", False),
    "group_by_aggregate/text_expected.tbl", "sorted")


# ---------------------------------------------------------------------------
# hash_join/*, skinner_join/*
# ---------------------------------------------------------------------------


def _two_scans(rel1, col1, rel2, col2):
    d = db()
    s1 = OperatorSchema()
    s1.AddGeneratedColumns(d[rel1], [col1])
    s2 = OperatorSchema()
    s2.AddGeneratedColumns(d[rel2], [col2])
    return ScanOperator(s1, d[rel1]), ScanOperator(s2, d[rel2])


def _hash_join(rel1, rel2, col):
    a, b = _two_scans(rel1, col, rel2, col)
    schema = OperatorSchema()
    schema.AddPassthroughColumns(a, 0)
    schema.AddPassthroughColumns(b, 1)
    return OutputOperator(HashJoinOperator(schema, a, b, [ColRef(a, col, 0)], [ColRef(b, col, 1)]))


def _skinner(rel, col):
    a, b = _two_scans(rel, col, rel, col)
    schema = OperatorSchema()
    schema.AddPassthroughColumns(a, 0)
    schema.AddPassthroughColumns(b, 1)
    return OutputOperator(SkinnerJoinOperator(schema, [a, b], [Eq(ColRef(a, col, 0), ColRef(b, col, 1))]))


for _t, _rel, _col in [("bigint", "info", "num2"), ("boolean", "info", "cheated"), ("date", "info", "date"),
                       ("enum", "people_enum", "name"), ("real", "info", "zscore"),
                       ("smallint", "info", "num1"), ("text", "people", "name")]:
    _add(f"hash_join/{_t}", (lambda r=_rel, c=_col: _hash_join(r, r, c)), f"hash_join/{_t}_expected.tbl", "sorted")
    _add(f"skinner_join/{_t}", (lambda r=_rel, c=_col: _skinner(r, c)), f"skinner_join/{_t}_expected.tbl", "sorted")
_add("hash_join/int", lambda: _hash_join("people", "info", "id"), "hash_join/int_expected.tbl", "sorted")


def _cross_product():
    # end_to_end_test/cross_product/cross_product_test.cc: region x region on r_name
    a, b = _two_scans("region", "r_name", "region", "r_name")
    schema = OperatorSchema()
    schema.AddPassthroughColumns(a, 0)
    schema.AddPassthroughColumns(b, 1)
    return OutputOperator(CrossProductOperator(schema, [a, b]))


_add("cross_product/text", _cross_product, "cross_product/cross_product_expected.tbl", "sorted")
_add("skinner_join/int", lambda: _skinner("info", "id"), "skinner_join/int_expected.tbl", "sorted")


def _skinner_multi():
    d = db()
    scans = []
    for _ in range(4):
        s = OperatorSchema()
        s.AddGeneratedColumns(d["info"], ["id", "num2"])
        scans.append(ScanOperator(s, d["info"]))
    s1, s2, s3, s4 = scans
    conds = [Eq(ColRef(s1, "id", 0), ColRef(s2, "id", 1)),
             Eq(ColRef(s2, "num2", 1), ColRef(s3, "num2", 2)),
             Eq(ColRef(s2, "id", 1), ColRef(s4, "id", 3))]
    schema = OperatorSchema()
    schema.AddPassthroughColumns(s1, ["id"], 0)
    schema.AddPassthroughColumns(s2, ["id"], 1)
    schema.AddPassthroughColumns(s3, ["id"], 2)
    schema.AddPassthroughColumns(s4, ["id"], 3)
    return OutputOperator(SkinnerJoinOperator(schema, scans, conds))


_add("skinner_join/multiple_tables_join", _skinner_multi, "skinner_join/multiple_tables_join_expected.tbl",
     "sorted")


# ---------------------------------------------------------------------------
# order_by/*
# ---------------------------------------------------------------------------


def _order_by(relation, cols, keys, asc):
    d = db()
    s = OperatorSchema()
    s.AddGeneratedColumns(d[relation], cols)
    base = ScanOperator(s, d[relation])
    schema = OperatorSchema()
    schema.AddPassthroughColumns(base)
    return OutputOperator(OrderByOperator(schema, base, [ColRef(base, k) for k in keys], [asc] * len(keys)))


for _t, _rel, _cols, _keys in [("bigint", "info", ["num2", "id"], ["num2", "id"]),
                               ("date", "info", ["date", "id"], ["date", "id"]),
                               ("enum", "people_enum", ["id", "name"], ["name", "id"]),
                               ("int", "info", ["id"], ["id"]),
                               ("real", "info", ["zscore", "id"], ["zscore", "id"]),
                               ("smallint", "info", ["num1", "id"], ["num1", "id"]),
                               ("text", "people", ["id", "name"], ["name", "id"])]:
    for _asc in (True, False):
        _add(f"order_by/{_t}_{'asc' if _asc else 'desc'}",
             (lambda r=_rel, c=_cols, k=_keys, a=_asc: _order_by(r, c, k, a)),
             f"order_by/{_t}_expected.tbl", "ordered", desc=not _asc)


# ---------------------------------------------------------------------------
# tpch/q01, q06, q03 (skinner)
# ---------------------------------------------------------------------------


def tpch_q01(lineitem="lineitem"):
    """end_to_end_test/tpch/q01_test.cc:42-136."""
    d = db()
    scan_schema = OperatorSchema()
    scan_schema.AddGeneratedColumns(d[lineitem], ["l_returnflag", "l_linestatus", "l_quantity",
                                                  "l_extendedprice", "l_discount", "l_tax", "l_shipdate"])
    leq = Leq(VirtColRef(scan_schema, "l_shipdate"), Literal(1998, 9, 13))
    schema = OperatorSchema()
    schema.AddVirtualPassthroughColumns(scan_schema, ["l_returnflag", "l_linestatus", "l_quantity",
                                                      "l_extendedprice", "l_discount", "l_tax"])
    sel = ScanSelectOperator(schema, scan_schema, d[lineitem], [leq])
    rf, ls = ColRefE(sel, "l_returnflag"), ColRefE(sel, "l_linestatus")
    aggs = [Sum(ColRef(sel, "l_quantity")), Sum(ColRef(sel, "l_extendedprice")),
            Sum(Mul(ColRef(sel, "l_extendedprice"), Sub(Literal(1.0), ColRef(sel, "l_discount")))),
            Sum(Mul(Mul(ColRef(sel, "l_extendedprice"), Sub(Literal(1.0), ColRef(sel, "l_discount"))),
                    Add(Literal(1.0), ColRef(sel, "l_tax")))),
            Avg(ColRef(sel, "l_quantity")), Avg(ColRef(sel, "l_extendedprice")),
            Avg(ColRef(sel, "l_discount")), Count()]
    gschema = OperatorSchema()
    gschema.AddDerivedColumn("l_returnflag", VirtColRef(rf, 0))
    gschema.AddDerivedColumn("l_linestatus", VirtColRef(ls, 1))
    for i, n in enumerate(["sum_qty", "sum_base_price", "sum_disc_price", "sum_charge", "avg_qty",
                           "avg_price", "avg_disc", "count_order"]):
        gschema.AddDerivedColumn(n, VirtColRef(aggs[i], i + 2))
    agg = GroupByAggregateOperator(gschema, sel, [rf, ls], aggs)
    oschema = OperatorSchema()
    oschema.AddPassthroughColumns(agg)
    return OutputOperator(OrderByOperator(oschema, agg, [ColRef(agg, "l_returnflag"),
                                                         ColRef(agg, "l_linestatus")], [True, True]))


def tpch_q06():
    """end_to_end_test/tpch/q06_test.cc:43-99."""
    d = db()
    s = OperatorSchema()
    s.AddGeneratedColumns(d["lineitem"], ["l_extendedprice", "l_discount", "l_shipdate", "l_quantity"])
    li = ScanOperator(s, d["lineitem"])
    cond = And([Geq(ColRef(li, "l_shipdate"), Literal(1993, 1, 1)),
                Lt(ColRef(li, "l_shipdate"), Literal(1994, 1, 1)),
                Geq(ColRef(li, "l_discount"), Literal(0.02)),
                Leq(ColRef(li, "l_discount"), Literal(0.04)),
                Lt(ColRef(li, "l_quantity"), Literal(25.0))])
    sschema = OperatorSchema()
    sschema.AddPassthroughColumns(li, ["l_extendedprice", "l_discount"])
    sel = SelectOperator(sschema, li, cond)
    revenue = Sum(Mul(ColRef(sel, "l_extendedprice"), ColRef(sel, "l_discount")))
    schema = OperatorSchema()
    schema.AddDerivedColumn("revenue", VirtColRef(revenue, 0))
    return OutputOperator(AggregateOperator(schema, sel, [revenue]))


def tpch_q03_skinner():
    """end_to_end_test/tpch/q03_skinner_test.cc (Skinner join of customer,
    orders, lineitem -> group by -> order by revenue desc, o_orderdate)."""
    d = db()
    cs = OperatorSchema()
    cs.AddGeneratedColumns(d["customer"], ["c_mktsegment", "c_custkey"])
    cust_f = Eq(VirtColRef(cs, "c_mktsegment"), Literal("AUTOMOBILE"))
    c_out = OperatorSchema()
    c_out.AddVirtualPassthroughColumns(cs, ["c_custkey"])
    customer = ScanSelectOperator(c_out, cs, d["customer"], [cust_f])

    os_ = OperatorSchema()
    ocols = ["o_orderdate", "o_shippriority", "o_custkey", "o_orderkey"]
    os_.AddGeneratedColumns(d["orders"], ocols)
    o_f = Lt(VirtColRef(os_, "o_orderdate"), Literal(1995, 3, 30))
    o_out = OperatorSchema()
    o_out.AddVirtualPassthroughColumns(os_, ocols)
    orders = ScanSelectOperator(o_out, os_, d["orders"], [o_f])

    ls = OperatorSchema()
    ls.AddGeneratedColumns(d["lineitem"], ["l_orderkey", "l_extendedprice", "l_shipdate", "l_discount"])
    l_f = Gt(VirtColRef(ls, "l_shipdate"), Literal(1995, 3, 30))
    l_out = OperatorSchema()
    l_out.AddVirtualPassthroughColumns(ls, ["l_orderkey", "l_extendedprice", "l_discount"])
    lineitem = ScanSelectOperator(l_out, ls, d["lineitem"], [l_f])

    conds = [Eq(ColRef(customer, "c_custkey", 0), ColRef(orders, "o_custkey", 1)),
             Eq(ColRef(lineitem, "l_orderkey", 2), ColRef(orders, "o_orderkey", 1))]
    js = OperatorSchema()
    js.AddPassthroughColumns(orders, ["o_orderdate", "o_shippriority"], 1)
    js.AddPassthroughColumns(lineitem, ["l_orderkey", "l_extendedprice", "l_discount"], 2)
    join = SkinnerJoinOperator(js, [customer, orders, lineitem], conds)

    lo, od, sp = ColRefE(join, "l_orderkey"), ColRefE(join, "o_orderdate"), ColRefE(join, "o_shippriority")
    revenue = Sum(Mul(ColRef(join, "l_extendedprice"), Sub(Literal(1.0), ColRef(join, "l_discount"))))
    gs = OperatorSchema()
    gs.AddDerivedColumn("l_orderkey", VirtColRef(lo, 0))
    gs.AddDerivedColumn("revenue", VirtColRef(revenue, 3))
    gs.AddDerivedColumn("o_orderdate", VirtColRef(od, 1))
    gs.AddDerivedColumn("o_shippriority", VirtColRef(sp, 2))
    agg = GroupByAggregateOperator(gs, join, [lo, od, sp], [revenue])
    oschema = OperatorSchema()
    oschema.AddPassthroughColumns(agg)
    return OutputOperator(OrderByOperator(oschema, agg, [ColRef(agg, "revenue"), ColRef(agg, "o_orderdate")],
                                          [False, True]))


_add("tpch/q01", tpch_q01, "tpch/q01_expected.tbl", "tbl")
_add("tpch/q06", tpch_q06, "tpch/q06_expected.tbl", "tbl")
_add("tpch/q03_skinner", tpch_q03_skinner, "tpch/q03_expected.tbl", "tbl")


# Float64 tolerance of GPU results against the reference's expected tables:
# the reference's absolute 1e-5, or 1e-12 relative, whichever is larger.
# Sums on the GPU add in another order than the reference's sequential loop
# (atomics in the general group table, per-CTA partials elsewhere), and for a
# sum near 1e9 an absolute 1e-5 is 1e-14 relative, a few dozen ulps.
GPU_REL = 1e-12


def check(case: Case_, lines: List[str], types, rel: float = 0.0) -> str:
    """Compare engine output lines with the expected table the way the
    reference test does (REAL also within `rel` relative, for GPU results).
    Returns '' when equal."""
    from kushdb_b200.result import compare_tbl
    exp = case.expected_lines()
    if case.mode == "sorted":
        if sorted(lines) != sorted(exp):
            a, b = sorted(lines), sorted(exp)
            for i, (x, y) in enumerate(zip(a, b)):
                if x != y:
                    return f"first difference at sorted line {i}: got {x!r} expected {y!r}"
            return f"line count {len(a)} vs expected {len(b)}"
        return ""
    if case.mode == "ordered":
        if lines != exp:
            for i, (x, y) in enumerate(zip(lines, exp)):
                if x != y:
                    return f"line {i}: got {x!r} expected {y!r}"
            return f"line count {len(lines)} vs expected {len(exp)}"
        return ""
    err = compare_tbl(exp, lines, types, rel=rel)
    return err or ""
