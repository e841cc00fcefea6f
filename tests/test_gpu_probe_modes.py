"""The join probe's load schedules give the oracle's results: the default
(one row per thread, next row's columns prefetched), the 4-row vector probe
that loads each vector's join-filter words and first slots together
(KDB_PROBE_VEC), the row-ahead forms (KDB_PROBE_AHEAD=1 / word), the build
side written in one unordered pass (KDB_BUILD_MAT_ATOMIC), the join filter in
shared memory (KDB_SMEM_BLOOM), the two-kernel probe and aggregation
(KDB_SPLIT_PROBE_GROUPS), and the separate join build and key-check kernels
(KDB_JOIN_BUILD_PASS, KDB_KEY_CHECK_PASS), on the
Q3-shape join + group-by (uniform and Zipf foreign keys), a join whose probe
keys are nullable SMALLINTs with duplicates on the build side, and a join
materialised without a group-by."""

import numpy as np
import pytest

from kushdb_b200 import workloads as wl
from kushdb_b200.data import HostColumn, HostTable, catalog_of
from kushdb_b200.plan import (ColRef, HashJoinOperator, OperatorSchema, OutputOperator, ScanOperator, Type)
from parity import compare

pytestmark = pytest.mark.gpu

MODES = [{}, {"KDB_PROBE_VEC": "1"}, {"KDB_PROBE_AHEAD": "1"}, {"KDB_PROBE_AHEAD": "word"},
         {"KDB_BUILD_MAT_ATOMIC": "1"}, {"KDB_SMEM_BLOOM": "1"}, {"KDB_SPLIT_PROBE_GROUPS": "1"},
         {"KDB_JOIN_BUILD_PASS": "1", "KDB_KEY_CHECK_PASS": "1"}]


@pytest.fixture(scope="module")
def engine():
    from kushdb_b200.engine import Engine
    e = Engine(0)
    e.set_prepared_queries(False)
    yield e
    e.close()


def _run(engine, plan, opts):
    for k, v in opts.items():
        engine.set_option(k, v)
    try:
        return engine.execute(plan)
    finally:
        for k in opts:
            engine.set_option(k, None)


@pytest.mark.parametrize("mode", MODES, ids=lambda m: ",".join(f"{k}={v}" for k, v in m.items()) or "default")
@pytest.mark.parametrize("zipf", [False, True])
def test_q3_shape(engine, mode, zipf):
    from oracle import Oracle
    b, p = wl.join_tables(build_rows=150_000, probe_rows=600_003, zipf=zipf, seed=17)
    engine.register_table(b)
    engine.register_table(p)
    o = Oracle()
    o.register_table(b)
    o.register_table(p)
    plan = wl.join_plan(b, p).to_json()
    assert compare(_run(engine, plan, mode), o.execute(plan), ordered=True) == ""
    o.close()


@pytest.mark.parametrize("mode", MODES, ids=lambda m: ",".join(f"{k}={v}" for k, v in m.items()) or "default")
def test_nullable_smallint_keys_materialised(engine, mode):
    from oracle import Oracle
    rng = np.random.default_rng(5)
    nb, np_ = 5_000, 40_001
    bt = HostTable("pm_b")
    bt.add(HostColumn("k", Type.SmallInt(), values=rng.integers(-200, 200, nb).astype(np.int16)))
    bt.add(HostColumn("x", Type.Int(), values=np.arange(nb, dtype=np.int32)))
    pt = HostTable("pm_p")
    pt.add(HostColumn("k", Type.SmallInt(), values=rng.integers(-250, 250, np_).astype(np.int16),
                      nulls=(rng.random(np_) < 0.1).astype(np.int8)))
    pt.add(HostColumn("y", Type.Real(), values=rng.random(np_)))
    engine.register_table(bt)
    engine.register_table(pt)
    o = Oracle()
    o.register_table(bt)
    o.register_table(pt)
    db = catalog_of([bt, pt])
    bs = OperatorSchema()
    bs.AddGeneratedColumns(db["pm_b"], ["k", "x"])
    bscan = ScanOperator(bs, db["pm_b"])
    ps = OperatorSchema()
    ps.AddGeneratedColumns(db["pm_p"], ["k", "y"])
    pscan = ScanOperator(ps, db["pm_p"])
    js = OperatorSchema()
    js.AddPassthroughColumns(bscan, ["x"], 0)
    js.AddPassthroughColumns(pscan, ["k", "y"], 1)
    join = HashJoinOperator(js, bscan, pscan, [ColRef(bscan, "k", 0)], [ColRef(pscan, "k", 1)])
    plan = OutputOperator(join).to_json()
    got = _run(engine, plan, mode)
    assert got.num_rows > 100_000
    assert compare(got, o.execute(plan), ordered=False) == ""
    o.close()
