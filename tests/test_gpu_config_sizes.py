"""Parity at the configurations' own sizes for the batched form (C4) and the
served Skinner joins (C5).

C4: the full batch -- 256 queries, fact tables log-uniform in [1e4, 6e6] rows
(about 265M rows in all), dimension tables at a quarter of that -- every
query's batched result equal to the plain executor's (same groups in the
same first-occurrence order, sums within 1e-12 relative), three queries also
against the CPU oracle.
C5: star and chain multiway joins of 6-8 tables of 1e5-3e6 rows with Zipf
s=1.5 foreign keys and LIKE '%tok%' filters against the oracle, under two
budgets and all three join-order policies.
"""

import numpy as np
import pytest

from kushdb_b200 import workloads as wl
from parity import REL_TOL, compare

pytestmark = pytest.mark.gpu


def _close(a, b):
    return np.all(np.abs(a - b) <= REL_TOL * np.maximum(np.abs(b), 1e-300))


def test_full_batch_matches_plain_executor_and_oracle():
    from kushdb_b200.engine import Batch, Engine
    from oracle import Oracle
    e = Engine(0)
    try:
        qs = wl.batch_tables(n_queries=256, min_fact=10_000, max_fact=6_000_000, seed=21, prefix="cfgb")
        assert max(f.rows for _, f, _, _ in qs) > 3_000_000
        for d, f, _, _ in qs:
            e.register_table(d)
            e.register_table(f)
        b = Batch(e, [wl.batch_query_desc(*q) for q in qs])
        b.tune(reps=1)
        b.run()
        for i, q in enumerate(qs):
            keys, sums = b.result(i)
            plain = e.execute(wl.batch_plan(*q))
            assert np.array_equal(keys, np.asarray(plain.columns[0].values)), f"query {i}: keys"
            assert _close(sums, np.asarray(plain.columns[1].values)), f"query {i}: sums"
        # three against the oracle: the largest fact table, a middle and a small one
        by_size = sorted(range(len(qs)), key=lambda i: qs[i][1].rows)
        for i in (by_size[-1], by_size[len(qs) // 2], by_size[0]):
            o = Oracle()
            o.register_table(qs[i][0])
            o.register_table(qs[i][1])
            ref = o.execute(wl.batch_plan(*qs[i]))
            keys, sums = b.result(i)
            assert np.array_equal(keys, np.asarray(ref.columns[0].values)), f"query {i}: keys vs oracle"
            assert _close(sums, np.asarray(ref.columns[1].values)), f"query {i}: sums vs oracle"
        b.close()
    finally:
        e.close()


@pytest.fixture(scope="module")
def engine():
    from kushdb_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()


# (shape, tables, seed, tables carrying the LIKE filter): all non-empty joins
SKINNER = [("star", 6, 7, (1, 2)), ("star", 8, 5, (1, 2)), ("chain", 6, 6, (5,)), ("chain", 7, 5, (2,))]


@pytest.mark.parametrize("shape,n,seed,like", SKINNER, ids=[f"{s}{n}_{seed}" for s, n, seed, _ in SKINNER])
def test_skinner_at_config_size_matches_oracle(engine, shape, n, seed, like):
    from oracle import Oracle
    tables, tokens = wl.skinner_tables(shape, n, min_rows=100_000, max_rows=3_000_000, zipf_s=1.5, seed=seed,
                                       prefix=f"cfgs{shape}{n}_")
    assert max(t.rows for t in tables) > 1_000_000
    plan = wl.skinner_plan(tables, tokens, shape, like_tables=like)
    o = Oracle()
    for t in tables:
        engine.register_table(t)
        o.register_table(t)
    ref = o.execute(plan)
    assert ref.lines[0] != "||"  # a non-empty join
    try:
        for policy, budget in (("uct", 100_000), ("random", 10_000), ("uct", 1 << 22)):
            engine.set_skinner_policy(policy)
            engine.set_skinner(budget, seed=2)
            g = engine.execute(plan)
            assert compare(g, ref) == "", (policy, budget, g.lines, ref.lines)
    finally:
        engine.set_skinner_policy("uct")
        engine.set_skinner()
        for t in tables:
            engine.drop_table(t.name)
