"""Every A/B switch's alternative code path still generates and compiles
(NVRTC, sm_100a) for the workload plans, in a compile-only context (no GPU):
the switches reproduce the measured comparisons, so their paths must not rot."""

import os

import pytest

from kushdb_b200 import workloads as wl
from kushdb_b200.engine import Engine

SWITCHES = ["KDB_NO_SCAN_PREFETCH", "KDB_NO_VECTOR_SCAN", "KDB_VECTOR_PROBE_SCAN", "KDB_NO_JOIN_FILTER",
            "KDB_NO_KEY_IN_SLOT", "KDB_NO_BUILD_ROW_GROUPS", "KDB_NO_DENSE_GROUPBY", "KDB_MATERIALIZE_ATOMIC",
            "KDB_GROUP_ORDER_SORT", "KDB_ORDER_RADIX", "KDB_ORDER_TIE_SORT", "KDB_SKINNER_DEPTH1",
            "KDB_SKINNER_NO_SPLIT", "KDB_NO_SKINNER_AGG", "KDB_DENSE_SMEM=0", "KDB_ORDER_SAMPLE",
            "KDB_NO_PROBE_PREFETCH", "KDB_LAZY_PROBE_COLUMNS", "KDB_NO_GROUP_ORDER_FUSE", "KDB_AGG_FUSED_FINALIZE",
            "KDB_DENSE_TMA", "KDB_DENSE_FIRST_MIN", "KDB_PROBE_AHEAD", "KDB_PROBE_AHEAD=word",
            "KDB_AGG_MINB=4", "KDB_PROBE_VEC", "KDB_SORT_SHAPE=8192,8,1024,4", "KDB_SCAN_BATCH=4", "KDB_DENSE_SMEM=1", "KDB_BUILD_MAT_ATOMIC", "KDB_ORDER_MERGE",
            "KDB_SPLIT_PROBE_GROUPS", "KDB_KEY_CHECK_PASS", "KDB_JOIN_BUILD_PASS",
            "KDB_NO_PDL", "KDB_DENSE_SWITCH", "KDB_SMEM_BLOOM",
            "KDB_ORDER_TIE_PASS", "KDB_ORDER_ROWS_PASS", "KDB_ORDER_FUSED_RANGE", "KDB_PROFILE_FRESH"]


@pytest.mark.parametrize("switch", SWITCHES)
def test_switch_path_compiles(switch):
    name, _, value = switch.partition("=")
    e = Engine(-1)
    try:
        e.set_option(name, value or "1")
        assert e.get_option(name) == (value or "1")
        t1 = wl.scan_agg_table(rows=1000)
        t2 = wl.group_by_table(rows=1000)
        b, p = wl.join_tables(build_rows=1000, probe_rows=4000)
        for t in (t1, t2, b, p):
            e.register_table(t)
        e.execute(wl.scan_agg_plan(t1))
        e.execute(wl.group_by_plan(t2))
        e.execute(wl.join_plan(b, p))
        tables, tokens = wl.skinner_tables("chain", 6, min_rows=100, max_rows=1000, prefix="sw")
        for t in tables:
            e.register_table(t)
        e.execute(wl.skinner_plan(tables, tokens, "chain"))
        assert e.kernel_launches() > 0
    finally:
        e.close()


def test_options_start_from_the_environment_and_can_be_removed():
    os.environ["KDB_NO_VECTOR_SCAN"] = "1"
    try:
        e = Engine(-1)
    finally:
        del os.environ["KDB_NO_VECTOR_SCAN"]
    assert e.get_option("KDB_NO_VECTOR_SCAN") == "1"
    e.set_option("KDB_NO_VECTOR_SCAN", None)
    assert e.get_option("KDB_NO_VECTOR_SCAN") is None
    e.close()
