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
    err = rp.check(case, res.lines, [c.type for c in res.columns], rel=rp.GPU_REL)
    assert err == "", err
    ref = o.execute(plan)
    ordered = case.mode != "sorted"
    assert compare(res, ref, ordered=ordered) == ""


SKINNER_CASES = [c for c in rp.CASES if c.name.startswith("skinner_join/") or c.name == "tpch/q03_skinner"]


@pytest.mark.parametrize("budget,seed", [(10, 0), (1000, 7), (1 << 20, 3)])
@pytest.mark.parametrize("case", SKINNER_CASES, ids=[c.name for c in SKINNER_CASES])
def test_skinner_result_independent_of_budget_and_seed(engines, case, budget, seed):
    """The reference runs every Skinner test at budgets 10 and 10000 (many
    suspended episodes vs few) (end_to_end_test/test_macros.h:3-152): the
    result never depends on the episode budget or the join orders tried."""
    e, _ = engines
    e.set_skinner(budget, seed)
    try:
        res = e.execute(case.build())
        err = rp.check(case, res.lines, [c.type for c in res.columns], rel=rp.GPU_REL)
        assert err == "", err
        if budget == 10:
            assert e.last_skinner_episodes() > 1
    finally:
        e.set_skinner()
