"""GPU engine parity on the reference's own golden tables (and the oracle).

Each case runs the restated reference test plan through the C ABI on cuda:0
and compares with the expected table exactly as the reference test does.
"""

import pytest

import reference_plans as rp
from parity import compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engines():
    from kushdb_b200.engine import Engine
    from oracle import Oracle
    e, o = Engine(0), Oracle()
    for t in rp.golden_tables().values():
        e.register_table(t)
        o.register_table(t)
    yield e, o
    e.close()
    o.close()


@pytest.mark.parametrize("case", rp.CASES, ids=[c.name for c in rp.CASES])
def test_gpu_matches_reference_golden(engines, case):
    e, o = engines
    plan = case.build()
    res = e.execute(plan)
    err = rp.check(case, res.lines, [c.type for c in res.columns])
    assert err == "", err
    ref = o.execute(plan)
    ordered = case.mode != "sorted"
    assert compare(res, ref, ordered=ordered) == ""
