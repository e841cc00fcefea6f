"""GPU parity, against the CPU oracle, of the expression forms beyond the
benchmark shapes: EXTRACT(YEAR FROM date) (runtime/date.cc:46-50) as a
projection and as a group key, enum IN lists (plan/expression/
enum_in_expression.h), STARTS_WITH / ENDS_WITH / CONTAINS on TEXT
(runtime/string.cc:14-40) and general LIKE (RegexpMatchingExpression, the
planner's ^...$ pattern) on TEXT and ENUM, with NULL inputs."""

import numpy as np
import pytest

from kushdb_b200.data import HostColumn, HostTable, catalog_of
from kushdb_b200.plan import (ColRef, Contains, Count, EndsWith, EnumRegistry, Extract, GroupByAggregateOperator,
                              In, Like, Literal, Max, Min, Not, OperatorSchema, Or, OutputOperator, ScanOperator,
                              ScanSelectOperator, StartsWith, Sum, Type, VirtColRef, EPOCH_JDN)
from parity import compare

pytestmark = pytest.mark.gpu

ENUM_ID = 41
COLORS = ["red", "green", "blue", "cyan", "magenta", "yellow", "black"]


@pytest.fixture(scope="module")
def setup():
    from kushdb_b200.engine import Engine
    from oracle import Oracle
    EnumRegistry.register(ENUM_ID, COLORS)
    rng = np.random.default_rng(17)
    n = 200_000
    words = np.array(["apple", "apricot", "banana", "grape", "grapefruit", "pineapple", "melon", "lemon",
                      "", "peach", "plum", "appleplum"])
    t = HostTable("expr_t")
    t.add(HostColumn("d", Type.Date(), values=(rng.integers(-30000, 30000, n) + EPOCH_JDN).astype(np.int32),
                     nulls=(rng.random(n) < 0.05).astype(np.int8)))
    t.add(HostColumn("c", Type.Enum(ENUM_ID), values=rng.integers(0, len(COLORS), n).astype(np.int32),
                     nulls=(rng.random(n) < 0.05).astype(np.int8)))
    strings = [words[i] + ("" if j % 3 else words[(i + 3) % len(words)]) for i, j in
               zip(rng.integers(0, len(words), n), rng.integers(0, 9, n))]
    t.add(HostColumn.from_strings("s", strings, nulls=(rng.random(n) < 0.05).astype(np.int8)))
    t.add(HostColumn("v", Type.Real(), values=rng.random(n) * 100))
    e, o = Engine(0), Oracle()
    e.register_table(t)
    o.register_table(t)
    yield t, e, o
    e.close()
    o.close()


def _select(t, filters, out_cols):
    rel = catalog_of([t])[t.name]
    scan = OperatorSchema()
    scan.AddGeneratedColumns(rel, ["d", "c", "s", "v"])
    out = OperatorSchema()
    out.AddVirtualPassthroughColumns(scan, out_cols)
    return scan, OutputOperator(ScanSelectOperator(out, scan, rel, [f(scan) for f in filters]))


@pytest.mark.parametrize("name,make", [
    ("starts_with", lambda s: StartsWith(VirtColRef(s, "s"), Literal("app"))),
    ("ends_with", lambda s: EndsWith(VirtColRef(s, "s"), Literal("plum"))),
    ("contains", lambda s: Contains(VirtColRef(s, "s"), Literal("ape"))),
    ("not_starts_with", lambda s: Not(StartsWith(VirtColRef(s, "s"), Literal("p")))),
    ("enum_in", lambda s: In(VirtColRef(s, "c"), ["red", "cyan", "black"])),
    ("enum_in_or_text", lambda s: Or([In(VirtColRef(s, "c"), ["green"]), EndsWith(VirtColRef(s, "s"), Literal("on"))])),
    ("like_inner", lambda s: Like(VirtColRef(s, "s"), "%p_e%")),
    ("like_anchored", lambda s: Like(VirtColRef(s, "s"), "a%e")),
    ("like_repeat", lambda s: Like(VirtColRef(s, "s"), "%a%a%a%")),
    ("like_enum", lambda s: Like(VirtColRef(s, "c"), "%e_")),
    ("not_like", lambda s: Not(Like(VirtColRef(s, "s"), "%l%m%"))),
])
def test_text_and_enum_filters_match_oracle(setup, name, make):
    t, e, o = setup
    _, plan = _select(t, [make], ["s", "c", "v"])
    g, r = e.execute(plan), o.execute(plan)
    assert g.num_rows > 0
    # a scan-select's rows come out in no particular order (the reference
    # tests compare them as sorted multisets)
    assert compare(g, r, ordered=False) == ""


def test_extract_year_projection_matches_oracle(setup):
    t, e, o = setup
    rel = catalog_of([t])[t.name]
    scan = OperatorSchema()
    scan.AddGeneratedColumns(rel, ["d", "v"])
    sc = ScanOperator(scan, rel)
    out = OperatorSchema()
    out.AddDerivedColumn("y", Extract(ColRef(sc, "d")))
    out.AddDerivedColumn("d", ColRef(sc, "d"))
    from kushdb_b200.plan import SelectOperator, Geq
    plan = OutputOperator(SelectOperator(out, sc, Geq(ColRef(sc, "v"), Literal(0.0))))
    g, r = e.execute(plan), o.execute(plan)
    assert compare(g, r, ordered=False) == ""


def test_group_by_extract_year_and_enum(setup):
    t, e, o = setup
    rel = catalog_of([t])[t.name]
    scan = OperatorSchema()
    scan.AddGeneratedColumns(rel, ["d", "c", "v"])
    sc = ScanOperator(scan, rel)
    year = Extract(ColRef(sc, "d"))
    col = ColRef(sc, "c")
    aggs = [Sum(ColRef(sc, "v")), Count(), Min(ColRef(sc, "d")), Max(ColRef(sc, "v"))]
    g = OperatorSchema()
    g.AddDerivedColumn("y", VirtColRef(year, 0))
    g.AddDerivedColumn("c", VirtColRef(col, 1))
    for i in range(len(aggs)):
        g.AddDerivedColumn(f"a{i}", VirtColRef(aggs[i], 2 + i))
    plan = OutputOperator(GroupByAggregateOperator(g, sc, [year, col], aggs))
    gr, rr = e.execute(plan), o.execute(plan)
    assert gr.num_rows > 100
    assert compare(gr, rr) == ""


def test_cross_product_under_select_and_group_by(setup):
    """CROSS_PRODUCT (cross_product_translator.cc): left rows buffered in
    their stream order, every right row paired with each; a SELECT over the
    pairs and a GROUP BY above, whose first-insertion order follows the
    pairs' stream order, against the oracle."""
    from kushdb_b200.plan import (Add, CrossProductOperator, Gt, Literal, Lt, ScanSelectOperator, SelectOperator,
                                  Sum, VirtColRef as VC)
    _, e, o = setup
    rng = np.random.default_rng(23)
    left = HostTable("cp_left")
    left.add(HostColumn("a", Type.Int(), values=rng.integers(0, 100, 400).astype(np.int32)))
    left.add(HostColumn("g", Type.Int(), values=rng.integers(0, 7, 400).astype(np.int32)))
    right = HostTable("cp_right")
    right.add(HostColumn("b", Type.Int(), values=rng.integers(0, 100, 3000).astype(np.int32)))
    right.add(HostColumn("w", Type.Real(), values=rng.random(3000)))
    for t in (left, right):
        e.register_table(t)
        o.register_table(t)
    db = catalog_of([left, right])
    ls = OperatorSchema()
    ls.AddGeneratedColumns(db["cp_left"], ["a", "g"])
    lout = OperatorSchema()
    lout.AddVirtualPassthroughColumns(ls, ["a", "g"])
    lsel = ScanSelectOperator(lout, ls, db["cp_left"], [Lt(VC(ls, "a"), Literal(60))])
    rs = OperatorSchema()
    rs.AddGeneratedColumns(db["cp_right"], ["b", "w"])
    rscan = ScanOperator(rs, db["cp_right"])
    cs = OperatorSchema()
    cs.AddPassthroughColumns(lsel, 0)
    cs.AddPassthroughColumns(rscan, 1)
    cp = CrossProductOperator(cs, [lsel, rscan])
    ss = OperatorSchema()
    ss.AddPassthroughColumns(cp)
    sel = SelectOperator(ss, cp, Gt(Add(ColRef(cp, "a"), ColRef(cp, "b")), Literal(150)))
    g = ColRef(sel, "g")
    s = Sum(ColRef(sel, "w"))
    gs = OperatorSchema()
    gs.AddDerivedColumn("g", VC(g, 0))
    gs.AddDerivedColumn("s", VC(s, 1))
    plan = OutputOperator(GroupByAggregateOperator(gs, sel, [g], [s]))
    gr, rr = e.execute(plan), o.execute(plan)
    assert gr.num_rows == 6  # group 0 has no pair with a + b > 150
    assert compare(gr, rr) == ""
    # the pairs themselves, as a multiset
    flat = OutputOperator(CrossProductOperator(cs, [lsel, rscan]))
    assert compare(e.execute(flat), o.execute(flat), ordered=False) == ""


@pytest.mark.parametrize("pattern", ["%", "", "a%", "%a%b%", "a_b", "%.%", "%(%", "%\n%", "_%_", "ab.c",
                                     "%xy%xy%", "_" * 6, "%" + "_%" * 30])
def test_like_random_strings(setup, pattern):
    """Short random strings over the pattern's own metacharacters and '\n'
    (which '_' and '%' do not match), 10% NULL."""
    import zlib
    from oracle import Oracle
    _, e, _ = setup
    o = Oracle()
    rng = np.random.default_rng(len(pattern))
    alphabet = list("ab.c%_(\n") + ["xy"]
    n = 50_000
    strings = ["".join(alphabet[int(i)] for i in rng.integers(0, len(alphabet), int(k)))
               for k in rng.integers(0, 8, n)]
    t = HostTable(f"like_rand_{zlib.crc32(pattern.encode())}")
    t.add(HostColumn.from_strings("s", strings, nulls=(rng.random(n) < 0.1).astype(np.int8)))
    e.register_table(t)
    o.register_table(t)
    rel = catalog_of([t])[t.name]
    scan = OperatorSchema()
    scan.AddGeneratedColumns(rel, ["s"])
    out = OperatorSchema()
    out.AddVirtualPassthroughColumns(scan, ["s"])
    plan = OutputOperator(ScanSelectOperator(out, scan, rel, [Like(VirtColRef(scan, "s"), pattern)]))
    assert compare(e.execute(plan), o.execute(plan), ordered=False) == ""
    o.close()
