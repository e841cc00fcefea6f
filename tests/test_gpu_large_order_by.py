"""ORDER BY above the one-block size against the oracle's merge sort, line
by line: single numeric keys (block sort + merge path), NULLs and several
keys (radix passes); float and integer keys with and without ties (ties must
come out in the reference merge sort's order), ascending and descending."""

import numpy as np
import pytest

from kushdb_b200.data import HostColumn, HostTable, catalog_of
from kushdb_b200.plan import ColRef, OperatorSchema, OrderByOperator, OutputOperator, ScanOperator, Type
from parity import compare

pytestmark = pytest.mark.gpu

N = 30_000


@pytest.fixture(scope="module")
def setup():
    from kushdb_b200.engine import Engine
    from oracle import Oracle
    rng = np.random.default_rng(12)
    t = HostTable("ob_rows")
    t.add(HostColumn("id", Type.Int(), values=np.arange(N, dtype=np.int32)))
    t.add(HostColumn("distinct_r", Type.Real(), values=rng.permutation(N).astype(np.float64) * 0.37 - 1000.0))
    t.add(HostColumn("tied_r", Type.Real(), values=rng.integers(0, 50, N).astype(np.float64) / 4.0))
    nulls = (rng.random(N) < 0.1).astype(np.int8)
    t.add(HostColumn("null_r", Type.Real(), values=rng.integers(0, 20, N).astype(np.float64), nulls=nulls))
    t.add(HostColumn("tied_i", Type.Int(), values=rng.integers(-5, 5, N).astype(np.int32)))
    e = Engine(0)
    e.register_table(t)
    o = Oracle()
    o.register_table(t)
    yield e, o, t
    e.close()


def _plan(t, keys, asc):
    rel = catalog_of([t])[t.name]
    s = OperatorSchema()
    s.AddGeneratedColumns(rel, ["id", "distinct_r", "tied_r", "null_r", "tied_i"])
    base = ScanOperator(s, rel)
    out = OperatorSchema()
    out.AddPassthroughColumns(base)
    return OutputOperator(OrderByOperator(out, base, [ColRef(base, k) for k in keys], asc))


@pytest.mark.parametrize("keys,asc", [(["distinct_r"], [True]), (["distinct_r"], [False]),
                                      (["tied_r"], [True]), (["tied_r"], [False]),
                                      (["null_r"], [True]), (["null_r"], [False]),
                                      (["tied_r", "null_r"], [False, True]),
                                      (["tied_i"], [True]), (["tied_i"], [False]), (["id"], [False])])
@pytest.mark.parametrize("sort", [None, "KDB_ORDER_MERGE", "KDB_ORDER_SAMPLE", "KDB_ORDER_RADIX",
                                  "KDB_ORDER_TIE_PASS", "KDB_ORDER_ROWS_PASS", "KDB_ORDER_FUSED_RANGE",
                                  "KDB_ORDER_MERGE,KDB_SORT_SHAPE=4096,8,512,2",
                                  "KDB_ORDER_MERGE,KDB_SORT_SHAPE=8192,8,1024,4"])
def test_order_matches_reference_merge_sort(setup, keys, asc, sort):
    """Each device sort (the default key-range bucket sort, merge passes of
    several tile shapes, sample sort, radix passes) gives the reference merge
    sort's order (the bucket sorts fall back to the merge passes when ties
    pile up in one bucket)."""
    e, o, t = setup
    plan = _plan(t, keys, asc).to_json()
    opts = []
    if sort:
        first, _, shape = sort.partition(",")
        opts.append((first, "1"))
        if shape:
            name, _, value = shape.partition("=")
            opts.append((name, value))
    for name, value in opts:
        e.set_option(name, value)
    try:
        got = e.execute(plan)
    finally:
        for name, _ in opts:
            e.set_option(name, None)
    assert compare(got, o.execute(plan), ordered=True) == ""
