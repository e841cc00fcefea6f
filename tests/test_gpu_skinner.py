"""Skinner multiway joins (JOB-style star and chain shapes, Zipf-skewed
foreign keys, LIKE '%tok%' filters) against the oracle: the adaptive
episode engine must return exactly the join's result for every budget."""

import pytest

from kushdb_b200 import workloads as wl
from parity import compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from kushdb_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("shape,n_tables,zipf", [("star", 6, 0.0), ("chain", 6, 0.0), ("star", 8, 1.5),
                                                 ("chain", 7, 1.5)])
@pytest.mark.parametrize("budget", [2000, 1 << 20])
def test_skinner_multiway_matches_oracle(engine, shape, n_tables, zipf, budget):
    from oracle import Oracle
    tables, tokens = wl.skinner_tables(shape, n_tables, min_rows=1000, max_rows=20_000, zipf_s=zipf,
                                       seed=11 + n_tables, prefix=f"{shape}{n_tables}{int(zipf)}_")
    plan = wl.skinner_plan(tables, tokens, shape)
    o = Oracle()
    for t in tables:
        engine.register_table(t)
        o.register_table(t)
    engine.set_skinner(budget, seed=1)
    try:
        g = engine.execute(plan)
    finally:
        engine.set_skinner()
    ref = o.execute(plan)
    assert compare(g, ref) == ""
    assert engine.last_skinner_episodes() >= 1


def test_aggregate_fused_into_episodes_matches_materialised(engine):
    """COUNT/MIN over the join evaluated inside the episode kernel equals the
    same aggregate over the materialised join result."""
    tables, tokens = wl.skinner_tables("chain", 6, min_rows=1000, max_rows=30_000, zipf_s=1.5, seed=77,
                                       prefix="fuse_")
    for t in tables:
        engine.register_table(t)
    plan = wl.skinner_plan(tables, tokens, "chain").to_json()
    engine.set_skinner(5000, seed=3)
    try:
        fused = engine.execute(plan)
        engine.set_option("KDB_NO_SKINNER_AGG", "1")
        try:
            plain = engine.execute(plan)
        finally:
            engine.set_option("KDB_NO_SKINNER_AGG", None)
    finally:
        engine.set_skinner()
    assert compare(fused, plain) == ""


@pytest.mark.parametrize("split,tasks", [(8, 1 << 16), (8, 16), (64, 1 << 16)])
@pytest.mark.parametrize("shape,n_tables", [("chain", 7), ("star", 8)])
@pytest.mark.parametrize("fused", [True, False])
def test_hot_runs_as_tasks_match_oracle(engine, split, tasks, shape, n_tables, fused):
    """Runs longer than `split` candidates at position 3 and deeper go to the
    task queues (a queue of `tasks` entries: with 16 it fills, and the rest
    is walked in place); the result stays exactly the join's."""
    from oracle import Oracle
    tables, tokens = wl.skinner_tables(shape, n_tables, min_rows=1000, max_rows=20_000, zipf_s=1.5,
                                       seed=31 + n_tables, prefix=f"hot{shape}{n_tables}_")
    plan = wl.skinner_plan(tables, tokens, shape)
    o = Oracle()
    for t in tables:
        engine.register_table(t)
        o.register_table(t)
    engine.set_option("KDB_SKINNER_SPLIT", str(split))
    engine.set_option("KDB_SKINNER_TASKS", str(tasks))
    if not fused:  # results materialised (slot allocation, regrowth) instead of folded
        engine.set_option("KDB_NO_SKINNER_AGG", "1")
    engine.set_skinner(3000, seed=2)
    try:
        g = engine.execute(plan)
    finally:
        for k in ("KDB_SKINNER_SPLIT", "KDB_SKINNER_TASKS", "KDB_NO_SKINNER_AGG"):
            engine.set_option(k, None)
        engine.set_skinner()
    assert compare(g, o.execute(plan)) == ""


@pytest.mark.parametrize("batch", [1, 4, 16])
@pytest.mark.parametrize("policy", ["uct", "random"])
def test_episode_batches_keep_the_result(engine, batch, policy):
    """Episodes run in batches (several join orders per launch, rewards
    corrected after the batch): the result is the join's for every batch
    size, and with more than one episode per batch there are fewer batches
    than episodes."""
    from oracle import Oracle
    tables, tokens = wl.skinner_tables("chain", 7, min_rows=2000, max_rows=40_000, zipf_s=1.5, seed=91,
                                       prefix=f"batch{batch}{policy}_")
    plan = wl.skinner_plan(tables, tokens, "chain", like_tables=(2,))
    o = Oracle()
    for t in tables:
        engine.register_table(t)
        o.register_table(t)
    engine.set_option("KDB_SKINNER_BATCH", str(batch))
    engine.set_skinner_policy(policy)
    engine.set_skinner(2000, seed=4)
    try:
        g = engine.execute(plan)
        episodes, batches = engine.last_skinner_episodes(), engine.last_skinner_batches()
    finally:
        engine.set_option("KDB_SKINNER_BATCH", None)
        engine.set_skinner_policy("uct")
        engine.set_skinner()
    assert compare(g, o.execute(plan)) == ""
    assert episodes >= batches >= 1
    if batch == 1:
        assert batches == episodes
    elif episodes > 4 * batch:
        assert batches < episodes
