"""The CPU oracle against the reference's own golden tables.

Every case restates one reference end-to-end test (plan, expected table and
comparison); the oracle must reproduce all of them before it is trusted as the
parity checker for the GPU engine.
"""

import pytest

import reference_plans as rp
from oracle import Oracle


@pytest.fixture(scope="module")
def oracle():
    o = Oracle()
    for t in rp.golden_tables().values():
        o.register_table(t)
    yield o
    o.close()


@pytest.mark.parametrize("case", rp.CASES, ids=[c.name for c in rp.CASES])
def test_oracle_matches_reference_golden(oracle, case):
    res = oracle.execute(case.build())
    err = rp.check(case, res.lines, [c.type for c in res.columns])
    assert err == "", err
