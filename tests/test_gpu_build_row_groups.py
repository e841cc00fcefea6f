"""GROUP BY over a hash join keyed by unique build rows: the group-per-build-
row path must give the oracle's result, in the same first-insertion order as
the general group table, and must not be taken when build keys repeat."""


import numpy as np
import pytest

from kushdb_b200 import workloads as wl
from kushdb_b200.data import HostColumn
from parity import compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from kushdb_b200.engine import Engine
    e = Engine(0)
    e.set_prepared_queries(False)  # every run generates its pipelines afresh
    yield e
    e.close()


def _oracle(*tables):
    from oracle import Oracle
    o = Oracle()
    for t in tables:
        o.register_table(t)
    return o


def _register(engine, *tables):
    for t in tables:  # the join tables reuse their names across tests
        try:
            engine.drop_table(t.name)
        except Exception:
            pass
        engine.register_table(t)


def _both_paths(engine, plan):
    text = plan.to_json()
    fast = engine.execute(text)
    engine.set_option("KDB_NO_BUILD_ROW_GROUPS", "1")
    try:
        general = engine.execute(text)
    finally:
        engine.set_option("KDB_NO_BUILD_ROW_GROUPS", None)
    return fast, general


@pytest.mark.parametrize("zipf", [False, True])
def test_unique_build_keys(engine, zipf):
    b, p = wl.join_tables(50_000, 200_000, zipf=zipf, seed=21)
    _register(engine, b, p)
    plan = wl.join_plan(b, p)
    fast, general = _both_paths(engine, plan)
    assert compare(fast, general) == ""
    assert compare(fast, _oracle(b, p).execute(plan.to_json())) == ""


def test_repeated_build_keys_take_the_general_path(engine):
    b, p = wl.join_tables(20_000, 80_000, seed=22)
    keys = np.asarray(b.columns["c_custkey"].values).copy()
    keys[1::2] = keys[0::2][: len(keys[1::2])]  # every key twice
    b.columns["c_custkey"] = HostColumn("c_custkey", b.columns["c_custkey"].type, values=keys)
    _register(engine, b, p)
    plan = wl.join_plan(b, p)
    fast, general = _both_paths(engine, plan)
    assert compare(fast, general) == ""
    assert compare(fast, _oracle(b, p).execute(plan.to_json())) == ""
