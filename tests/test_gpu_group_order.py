"""GROUP BY under an ORDER BY: the group table hands its groups over in table
order with their first-appearance position, and the ORDER BY puts them in
order itself.  Sort keys with and without ties (ties must come out in the
reference merge sort's order over the groups' first-appearance order), for
the group-per-build-row path and the general group table, above and below
the one-block ORDER BY size, against the oracle and against the path that
sorts the groups first."""


import numpy as np
import pytest

from kushdb_b200 import workloads as wl
from kushdb_b200.data import HostColumn, HostTable, catalog_of
from kushdb_b200.plan import (ColRef, Count, GroupByAggregateOperator, HashJoinOperator, Max, OperatorSchema,
                              OrderByOperator, OutputOperator, ScanOperator, Sum, Type, VirtColRef)
from parity import compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from kushdb_b200.engine import Engine
    e = Engine(0)
    e.set_prepared_queries(False)
    yield e
    e.close()


def _register(engine, oracle, *tables):
    for t in tables:
        try:
            engine.drop_table(t.name)
        except Exception:
            pass
        engine.register_table(t)
        oracle.register_table(t)


def _run(engine, plan, env=None):
    text = plan.to_json()
    for k, v in (env or {}).items():
        engine.set_option(k, v)
    try:
        return engine.execute(text)
    finally:
        for k in (env or {}):
            engine.set_option(k, None)


def _join_group_plan(b, p, order_col, asc):
    db = catalog_of([b, p])
    brel, prel = db[b.name], db[p.name]
    bs = OperatorSchema()
    bs.AddGeneratedColumns(brel, ["c_custkey"])
    bscan = ScanOperator(bs, brel)
    ps = OperatorSchema()
    ps.AddGeneratedColumns(prel, ["o_custkey", "o_price"])
    pscan = ScanOperator(ps, prel)
    js = OperatorSchema()
    js.AddPassthroughColumns(bscan, ["c_custkey"], 0)
    js.AddPassthroughColumns(pscan, ["o_price"], 1)
    join = HashJoinOperator(js, bscan, pscan, [ColRef(bscan, "c_custkey", 0)], [ColRef(pscan, "o_custkey", 1)])
    key = ColRef(join, "c_custkey")
    cnt = Count()
    rev = Sum(ColRef(join, "o_price"))
    gs = OperatorSchema()
    gs.AddDerivedColumn("c_custkey", VirtColRef(key, 0))
    gs.AddDerivedColumn("n", VirtColRef(cnt, 1))
    gs.AddDerivedColumn("revenue", VirtColRef(rev, 2))
    agg = GroupByAggregateOperator(gs, join, [key], [cnt, rev])
    os_ = OperatorSchema()
    os_.AddPassthroughColumns(agg)
    return OutputOperator(OrderByOperator(os_, agg, [ColRef(agg, order_col)], [asc]))


def _table_group_plan(t, order_col, asc):
    rel = catalog_of([t])[t.name]
    s = OperatorSchema()
    s.AddGeneratedColumns(rel, ["g", "x", "y"])
    scan = ScanOperator(s, rel)
    key = ColRef(scan, "g")
    tot = Sum(ColRef(scan, "x"))
    top = Max(ColRef(scan, "y"))
    gs = OperatorSchema()
    gs.AddDerivedColumn("g", VirtColRef(key, 0))
    gs.AddDerivedColumn("total", VirtColRef(tot, 1))
    gs.AddDerivedColumn("top", VirtColRef(top, 2))
    agg = GroupByAggregateOperator(gs, scan, [key], [tot, top])
    os_ = OperatorSchema()
    os_.AddPassthroughColumns(agg)
    return OutputOperator(OrderByOperator(os_, agg, [ColRef(agg, order_col)], [asc]))


@pytest.mark.parametrize("build_rows", [3_000, 40_000])
@pytest.mark.parametrize("order_col,asc", [("n", False), ("n", True), ("revenue", False), ("c_custkey", True)])
@pytest.mark.parametrize("build_row_groups", [True, False])
def test_join_group_order(engine, build_rows, order_col, asc, build_row_groups):
    from oracle import Oracle
    o = Oracle()
    b, p = wl.join_tables(build_rows, build_rows * 4, seed=31)
    _register(engine, o, b, p)
    plan = _join_group_plan(b, p, order_col, asc)
    env = {} if build_row_groups else {"KDB_NO_BUILD_ROW_GROUPS": "1"}
    got = _run(engine, plan, env)
    assert compare(got, o.execute(plan.to_json()), ordered=True) == ""
    sorted_first = _run(engine, plan, dict(env, KDB_GROUP_ORDER_SORT="1"))
    assert compare(got, sorted_first, ordered=True) == ""


@pytest.mark.parametrize("groups", [1_000, 30_000])
@pytest.mark.parametrize("order_col,asc", [("total", True), ("total", False), ("top", False), ("g", True)])
def test_table_group_order(engine, groups, order_col, asc):
    from oracle import Oracle
    o = Oracle()
    rng = np.random.default_rng(groups)
    n = groups * 6
    t = HostTable("grouped_rows")
    t.add(HostColumn("g", Type.Int(), values=rng.integers(0, groups, n).astype(np.int32)))
    t.add(HostColumn("x", Type.Int(), values=rng.integers(0, 4, n).astype(np.int32)))
    t.add(HostColumn("y", Type.Real(), values=rng.integers(0, 1 << 20, n).astype(np.float64) * 0.5))
    _register(engine, o, t)
    plan = _table_group_plan(t, order_col, asc)
    got = _run(engine, plan)
    assert compare(got, o.execute(plan.to_json()), ordered=True) == ""


@pytest.mark.parametrize("keys_asc", [((0, True), (1, True)), ((0, False), (1, True)), ((1, False),),
                                      ((1, True), (0, False))])
@pytest.mark.parametrize("rows", [500, 200_000])
def test_dense_group_order_fused(engine, keys_asc, rows):
    """An ORDER BY over enum GROUP BY keys (one of them nullable) is done by
    the dense group-by itself: same rows and order as the oracle and as the
    separate one-block ORDER BY."""
    from oracle import Oracle
    from kushdb_b200.plan import EnumRegistry
    EnumRegistry.register(61, ["zeta", "alpha", "mu"])
    EnumRegistry.register(62, ["b", "a"])
    o = Oracle()
    rng = np.random.default_rng(rows)
    t = HostTable("dense_order")
    t.add(HostColumn("k1", Type.Enum(61), values=rng.integers(0, 3, rows).astype(np.int32)))
    t.add(HostColumn("k2", Type.Enum(62), values=rng.integers(0, 2, rows).astype(np.int32),
                     nulls=(rng.random(rows) < 0.2).astype(np.int8)))
    t.add(HostColumn("v", Type.Real(), values=rng.random(rows)))
    _register(engine, o, t)
    rel = catalog_of([t])[t.name]
    ss = OperatorSchema()
    ss.AddGeneratedColumns(rel, ["k1", "k2", "v"])
    scan = ScanOperator(ss, rel)
    k1, k2 = ColRef(scan, "k1"), ColRef(scan, "k2")
    aggs = [Sum(ColRef(scan, "v")), Count()]
    g = OperatorSchema()
    g.AddDerivedColumn("k1", VirtColRef(k1, 0))
    g.AddDerivedColumn("k2", VirtColRef(k2, 1))
    g.AddDerivedColumn("s", VirtColRef(aggs[0], 2))
    g.AddDerivedColumn("n", VirtColRef(aggs[1], 3))
    agg = GroupByAggregateOperator(g, scan, [k1, k2], aggs)
    out = OperatorSchema()
    out.AddPassthroughColumns(agg)
    names = ["k1", "k2"]
    plan = OutputOperator(OrderByOperator(out, agg, [ColRef(agg, names[k]) for k, _ in keys_asc],
                                          [a for _, a in keys_asc]))
    fused = _run(engine, plan)
    assert compare(fused, o.execute(plan.to_json()), ordered=True) == ""
    separate = _run(engine, plan, {"KDB_NO_GROUP_ORDER_FUSE": "1"})
    assert compare(fused, separate, ordered=True) == ""
