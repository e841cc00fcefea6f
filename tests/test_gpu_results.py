"""Results own their downloaded columns (a pinned block from the context's
pool): a result read after later queries ran, after many results were held
at once, or after the engine was closed still holds its own values."""

import numpy as np
import pytest

from kushdb_b200 import workloads as wl
from parity import compare

pytestmark = pytest.mark.gpu


def _tables():
    t = wl.group_by_table(200_000)
    b, p = wl.join_tables(20_000, 80_000, seed=7)
    return t, b, p


def _oracle(*tables):
    from oracle import Oracle
    o = Oracle()
    for t in tables:
        o.register_table(t)
    return o


def test_results_survive_later_queries():
    from kushdb_b200.engine import Engine
    t, b, p = _tables()
    q1 = wl.group_by_plan(t).to_json()
    q2 = wl.join_plan(b, p).to_json()
    o = _oracle(t, b, p)
    want1, want2 = o.execute(q1), o.execute(q2)
    e = Engine(0)
    try:
        for x in (t, b, p):
            e.register_table(x)
        held = []
        for _ in range(3):  # first run, first replay (graph capture), replay
            held.append(e.execute(q1))
            held.append(e.execute(q2))
        for i, r in enumerate(held):  # columns are read only now
            assert compare(r, want1 if i % 2 == 0 else want2) == "", i
    finally:
        e.close()


def test_many_results_held_and_freed_out_of_order():
    from kushdb_b200.engine import Engine
    t, _, _ = _tables()
    q = wl.group_by_plan(t).to_json()
    want = _oracle(t).execute(q)
    e = Engine(0)
    try:
        e.register_table(t)
        held = [e.execute(q) for _ in range(24)]  # more than the pool keeps
        for r in held[::3]:
            r.close()
        rest = [r for i, r in enumerate(held) if i % 3]
        again = [e.execute(q) for _ in range(8)]
        for r in rest + again:
            assert compare(r, want) == ""
    finally:
        e.close()


def test_result_read_after_engine_close():
    from kushdb_b200.engine import Engine
    _, b, p = _tables()
    q = wl.join_plan(b, p).to_json()
    want = _oracle(b, p).execute(q)
    e = Engine(0)
    e.register_table(b)
    e.register_table(p)
    r = e.execute(q)
    e.close()
    cols = r.columns  # read through the result handle alone
    assert len(cols[0].nulls) == want.num_rows
    assert np.array_equal(np.asarray(cols[0].values), np.asarray(want.columns[0].values))
    r.close()


def test_large_results_held_beyond_the_pool():
    """Results above the small-result size keep their pinned blocks: more of
    them held at once than the pool keeps, freed out of order, each still
    holds its own rows."""
    from kushdb_b200.engine import Engine
    from kushdb_b200.data import HostColumn, HostTable, catalog_of
    from kushdb_b200.plan import ColRef, OperatorSchema, OrderByOperator, OutputOperator, ScanOperator, Type
    n = 20_000  # 20k rows x 12 bytes downloaded: well above 64 KB
    rng = np.random.default_rng(3)
    t = HostTable("held_rows")
    t.add(HostColumn("id", Type.Int(), values=np.arange(n, dtype=np.int32)))
    t.add(HostColumn("x", Type.Real(), values=rng.permutation(n).astype(np.float64)))
    rel = catalog_of([t])[t.name]
    s = OperatorSchema()
    s.AddGeneratedColumns(rel, ["id", "x"])
    scan = ScanOperator(s, rel)
    out = OperatorSchema()
    out.AddPassthroughColumns(scan)
    q = OutputOperator(OrderByOperator(out, scan, [ColRef(scan, "x")], [True])).to_json()
    want = _oracle(t).execute(q)
    e = Engine(0)
    try:
        e.register_table(t)
        held = [e.execute(q) for _ in range(20)]
        for r in held[1::2]:
            r.close()
        more = [e.execute(q) for _ in range(4)]
        for r in held[0::2] + more:
            assert compare(r, want) == ""
    finally:
        e.close()
