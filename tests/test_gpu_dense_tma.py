"""The small-domain group-by with its scan staged through shared memory by
TMA bulk copies (KDB_DENSE_TMA; register and shared-memory accumulators)
against the oracle and against the register-load scan: row counts around
the tile size (ragged last tiles, fewer rows than one 16-byte unit),
nullable keys and measures (their null arrays staged too), BOOLEAN,
SMALLINT, ENUM and DATE columns, and several tile / stage shapes."""

import numpy as np
import pytest

from kushdb_b200.data import HostColumn, HostTable, catalog_of
from kushdb_b200.plan import (Avg, ColRef, Count, EnumRegistry, GroupByAggregateOperator, Leq, LiteralExpression,
                              Max, Min, OperatorSchema, OutputOperator, ScanSelectOperator, Sum, Type, VirtColRef)
from kushdb_b200 import workloads as wl
from parity import compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from kushdb_b200.engine import Engine
    e = Engine(0)
    e.set_prepared_queries(False)
    yield e
    e.close()


def _table(name, rows, seed):
    EnumRegistry.register(71, ["x", "y", "z"])
    rng = np.random.default_rng(seed)
    t = HostTable(name)
    t.add(HostColumn("e", Type.Enum(71), values=rng.integers(0, 3, rows).astype(np.int32),
                     nulls=(rng.random(rows) < 0.1).astype(np.int8)))
    t.add(HostColumn("b", Type.Boolean(), values=(rng.random(rows) < 0.5).astype(np.int8)))
    t.add(HostColumn("s", Type.SmallInt(), values=rng.integers(-300, 300, rows).astype(np.int16)))
    t.add(HostColumn("d", Type.Date(), values=rng.integers(2_440_000, 2_450_000, rows).astype(np.int32)))
    t.add(HostColumn("v", Type.Real(), values=rng.random(rows) * 100,
                     nulls=(rng.random(rows) < 0.05).astype(np.int8)))
    return t


def _plan(t):
    rel = catalog_of([t])[t.name]
    ss = OperatorSchema()
    ss.AddGeneratedColumns(rel, ["e", "b", "s", "d", "v"])
    out = OperatorSchema()
    out.AddVirtualPassthroughColumns(ss, ["e", "s", "v"])
    # the BOOLEAN column is a filter of its own (staged like the others)
    scan = ScanSelectOperator(out, ss, rel, [Leq(VirtColRef(ss, "d"), LiteralExpression(Type.Date(), 2_449_000)),
                                             VirtColRef(ss, "b")])
    e = ColRef(scan, "e")
    aggs = [Sum(ColRef(scan, "v")), Avg(ColRef(scan, "s")), Min(ColRef(scan, "v")), Max(ColRef(scan, "s")),
            Count(ColRef(scan, "v")), Count()]
    g = OperatorSchema()
    g.AddDerivedColumn("e", VirtColRef(e, 0))
    for i, n in enumerate(["sv", "as", "mv", "ms", "cv", "n"]):
        g.AddDerivedColumn(n, VirtColRef(aggs[i], i + 1))
    return OutputOperator(GroupByAggregateOperator(g, scan, [e], aggs))


def _run(engine, plan, opts):
    for k, v in opts.items():
        engine.set_option(k, v)
    try:
        return engine.execute(plan)
    finally:
        for k in opts:
            engine.set_option(k, None)


@pytest.mark.parametrize("rows", [1, 3, 15, 511, 512, 513, 4099, 200_003])
@pytest.mark.parametrize("shape", [{}, {"KDB_DENSE_SMEM": "1"}, {"KDB_TMA_TILE": "256", "KDB_TMA_STAGES": "2"},
                                   {"KDB_TMA_TILE": "1024", "KDB_TMA_STAGES": "4", "KDB_TMA_BLOCK": "64",
                                    "KDB_DENSE_SMEM": "1"}])
def test_tma_dense_group_by_matches_oracle(engine, rows, shape):
    from oracle import Oracle
    t = _table(f"tma_{rows}", rows, rows)
    engine.register_table(t)
    o = Oracle()
    o.register_table(t)
    plan = _plan(t).to_json()
    got = _run(engine, plan, dict(shape, KDB_DENSE_TMA="1"))
    assert compare(got, o.execute(plan)) == ""
    assert compare(got, _run(engine, plan, {})) == ""
    o.close()


def test_tma_q1_shape_at_config_size(engine):
    """The Q1-shape group-by at 6,000,000 rows, staged, against the oracle."""
    from oracle import Oracle
    t = wl.group_by_table(rows=6_000_000, name="tma_q1")
    engine.register_table(t)
    o = Oracle()
    o.register_table(t)
    plan = wl.group_by_plan(t).to_json()
    got = _run(engine, plan, {"KDB_DENSE_TMA": "1"})
    assert compare(got, o.execute(plan), ordered=True) == ""
    o.close()
