"""The C-ABI library without a GPU: it loads, exports every symbol the
header declares, and every reference plan / workload plan generates and
compiles (NVRTC, sm_100a) in a compile-only context."""

import os
import re

import pytest

import reference_plans as rp
from kushdb_b200 import workloads as wl
from kushdb_b200.engine import EXPORTS, Engine, load_library

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "kdb_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(kdb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    lib = load_library()
    declared = header_symbols()
    assert set(declared) == set(EXPORTS), set(declared) ^ set(EXPORTS)
    for s in declared:
        assert hasattr(lib, s), s


@pytest.fixture(scope="module")
def dry_engine():
    e = Engine(-1)
    for t in rp.golden_tables().values():
        e.register_table(t)
    yield e
    e.close()


@pytest.mark.parametrize("case", rp.CASES, ids=[c.name for c in rp.CASES])
def test_reference_plan_compiles_for_sm100a(dry_engine, case):
    dry_engine.execute(case.build())


def test_workload_plans_compile_for_sm100a():
    e = Engine(-1)
    t1 = wl.scan_agg_table(rows=1000)
    t2 = wl.group_by_table(rows=1000)
    b, p = wl.join_tables(build_rows=1000, probe_rows=4000)
    for t in (t1, t2, b, p):
        e.register_table(t)
    e.execute(wl.scan_agg_plan(t1))
    e.execute(wl.group_by_plan(t2))
    e.execute(wl.join_plan(b, p))
    for shape in ("star", "chain"):
        tables, tokens = wl.skinner_tables(shape, 6, min_rows=100, max_rows=1000, prefix=shape)
        for t in tables:
            e.register_table(t)
        e.execute(wl.skinner_plan(tables, tokens, shape))
    assert e.kernel_launches() > 0
    e.close()


def test_errors_cross_the_abi_as_codes():
    e = Engine(-1)
    with pytest.raises(RuntimeError):
        e.execute('{"op":"OUTPUT","child":{"op":"SCAN","relation":"nope","columns":[],"output":[]}}')
    with pytest.raises(RuntimeError):
        e.execute("{not json")
    e.close()


def test_serving_needs_a_device_context():
    from kushdb_b200.engine import KdbError, Server
    e = Engine(-1)
    with pytest.raises(KdbError, match="GPU"):
        Server(e, slots=2)
    lib = load_library()
    assert lib.kdb_server_submit(None, b"{}") < 0
    assert lib.kdb_server_poll(None, 1, 0, None) < 0
    e.close()


def test_join_prior_needs_a_device_context():
    from kushdb_b200.engine import JoinPriorModel, KdbError
    e = Engine(-1)
    with pytest.raises(KdbError, match="GPU"):
        JoinPriorModel(e)
    with pytest.raises(KdbError):
        e.set_skinner_policy("prior")  # no model
    e.set_skinner_policy("random", log=True)
    e.set_skinner_policy("uct")
    lib = load_library()
    assert lib.kdb_mlp_num_params() == 41473 and lib.kdb_mlp_num_features() == 64
    e.close()
