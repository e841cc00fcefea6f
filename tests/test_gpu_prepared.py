"""Prepared queries: the second and later runs of a plan replay its recorded
CUDA graph.  Replays must give the oracle's result every time, a table
refreshed in place (same shape, new values) must invalidate the recording,
and plans that cannot be replayed (Skinner joins) still run afresh."""

import numpy as np
import pytest

import reference_plans as rp
from kushdb_b200 import workloads as wl
from kushdb_b200.data import HostColumn
from parity import compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from kushdb_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()


def _oracle(*tables):
    from oracle import Oracle
    o = Oracle()
    for t in tables:
        o.register_table(t)
    return o


@pytest.mark.parametrize("case", rp.CASES, ids=[c.name for c in rp.CASES])
def test_reference_plans_replay(engine, case):
    for t in rp.golden_tables().values():
        engine.register_table(t)
    plan = case.build().to_json()
    first = engine.execute(plan)
    for _ in range(2):
        again = engine.execute(plan)
        # row order is the reference's only for ordered outputs
        assert compare(again, first, ordered=case.mode == "ordered") == ""
    res = engine.execute(plan)
    assert rp.check(case, res.lines, [c.type for c in res.columns], rel=rp.GPU_REL) == ""


@pytest.mark.parametrize("name", ["scan_agg", "group_by", "join_group"])
def test_workloads_replay_and_invalidate(engine, name):
    if name == "scan_agg":
        t = wl.scan_agg_table(300_000, seed=5, name="pq_sales")
        tables, plan = [t], wl.scan_agg_plan(t)
    elif name == "group_by":
        t = wl.group_by_table(400_000, seed=6, name="pq_lineitem")
        tables, plan = [t], wl.group_by_plan(t)
    else:
        b, p = wl.join_tables(30_000, 120_000, seed=7)
        tables, plan = [b, p], wl.join_plan(b, p)
    for t in tables:
        engine.register_table(t)
    text = plan.to_json()
    o = _oracle(*tables)
    ref = o.execute(text)
    for _ in range(3):
        assert compare(engine.execute(text), ref) == ""
    # refresh a column in place (same shape, new values): the recording is stale
    t = tables[-1]
    col = next(c for c in t.columns.values() if c.type.type_id == "REAL")
    t.columns[col.name] = HostColumn(col.name, col.type, values=np.asarray(col.values) * 2.0 + 1.0)
    engine.register_table(t)
    ref2 = _oracle(*tables).execute(text)
    for _ in range(2):
        assert compare(engine.execute(text), ref2) == ""


def test_skinner_plans_run_afresh(engine):
    tables, tokens = wl.skinner_tables("star", 4, min_rows=500, max_rows=5000, seed=4, prefix="pqsk")
    for t in tables:
        engine.register_table(t)
    plan = wl.skinner_plan(tables, tokens, "star").to_json()
    ref = _oracle(*tables).execute(plan)
    for _ in range(3):
        assert compare(engine.execute(plan), ref) == ""
        assert engine.last_skinner_episodes() >= 1


def test_prepared_off_matches(engine):
    t = wl.group_by_table(200_000, seed=8, name="pq_off")
    engine.register_table(t)
    text = wl.group_by_plan(t).to_json()
    on = engine.execute(text)
    engine.execute(text)
    engine.set_prepared_queries(False)
    try:
        off = engine.execute(text)
    finally:
        engine.set_prepared_queries(True)
    assert compare(on, off) == ""


@pytest.mark.parametrize("name", ["group_by", "join_group"])
def test_profiled_replay_times_every_kernel(engine, name):
    """Profiling a prepared query replays its recorded launches with an event
    pair around each kernel: the same kernel roles as a profiled fresh run,
    every time positive, and the query's result unchanged."""
    if name == "group_by":
        t = wl.group_by_table(300_000, seed=9, name="pq_prof_lineitem")
        tables, plan = [t], wl.group_by_plan(t)
    else:
        b, p = wl.join_tables(60_000, 240_000, seed=10)
        tables, plan = [b, p], wl.join_plan(b, p)
    for t in tables:
        try:  # an earlier test registered the join tables under these names
            engine.drop_table(t.name)
        except Exception:
            pass
        engine.register_table(t)
    text = plan.to_json()
    engine.set_profiling(True)
    try:
        fresh = engine.execute(text)  # profiling runs afresh when nothing is recorded
        fresh_tags = {k["tag"] for k in engine.last_kernels()}
    finally:
        engine.set_profiling(False)
    engine.execute(text)  # recorded
    engine.execute(text)  # replayed
    engine.set_profiling(True)
    try:
        replayed = engine.execute(text)
        kernels = engine.last_kernels()
    finally:
        engine.set_profiling(False)
    assert compare(replayed, fresh, ordered=True) == ""
    tags = {k["tag"] for k in kernels}
    assert "group by" in tags and tags <= fresh_tags
    assert all(k["ms"] > 0 for k in kernels)
    for t in tables:
        engine.drop_table(t.name)
