"""Batched form: many uneven scan-select -> hash-join -> group-by queries in
one captured CUDA graph.  Every query's batched result must equal the plain
executor's result for the same plan (same groups in the same first-
occurrence order; sums within 1e-12 relative), and the oracle's for a few."""

import numpy as np
import pytest

from kushdb_b200 import workloads as wl
from parity import REL_TOL

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    from kushdb_b200.engine import Batch, Engine
    e = Engine(0)
    qs = wl.batch_tables(n_queries=48, min_fact=100, max_fact=200_000, seed=3, prefix="tb")
    for d, f, _, _ in qs:
        e.register_table(d)
        e.register_table(f)
    b = Batch(e, [wl.batch_query_desc(*q) for q in qs])
    yield e, b, qs
    b.close()
    e.close()


def _check_against_plain(e, b, qs):
    b.run()
    for i, q in enumerate(qs):
        keys, sums = b.result(i)
        plain = e.execute(wl.batch_plan(*q))
        pk = np.asarray(plain.columns[0].values)
        ps = np.asarray(plain.columns[1].values)
        assert np.array_equal(keys, pk), f"query {i}: keys differ"
        assert np.all(np.abs(sums - ps) <= REL_TOL * np.maximum(np.abs(ps), 1e-300)), f"query {i}: sums"


@pytest.mark.parametrize("block,lf,fanout", [(256, 0.5, 1), (128, 0.9, 64), (512, 0.7, 1024)])
def test_batch_matches_plain_executor(setup, block, lf, fanout):
    e, b, qs = setup
    b.configure(block, lf, fanout)
    _check_against_plain(e, b, qs)


def test_batch_matches_oracle(setup):
    from oracle import Oracle
    e, b, qs = setup
    b.configure()
    b.run()
    for i in (0, 7, 23):
        o = Oracle()
        o.register_table(qs[i][0])
        o.register_table(qs[i][1])
        ref = o.execute(wl.batch_plan(*qs[i]))
        keys, sums = b.result(i)
        assert np.array_equal(keys, np.asarray(ref.columns[0].values))
        rs = np.asarray(ref.columns[1].values)
        assert np.all(np.abs(sums - rs) <= REL_TOL * np.maximum(np.abs(rs), 1e-300))


def test_autotuner_picks_a_timed_configuration(setup):
    e, b, qs = setup
    report = b.tune(reps=1)
    assert len(report) == 3 * 3 * 4
    best = min(report, key=lambda r: r["ms"])
    cfg = b.config()
    assert (cfg["block"], cfg["fanout"]) == (best["block"], best["fanout"])
    assert abs(cfg["load_factor"] - best["load_factor"]) < 1e-9
    _check_against_plain(e, b, qs)


def test_batch_rejects_non_unique_dimension_keys():
    from kushdb_b200.data import HostColumn
    from kushdb_b200.engine import Batch, Engine, KdbError
    e = Engine(0)
    (d, f, lt, seg), = wl.batch_tables(n_queries=1, min_fact=1000, max_fact=1000, seed=9, prefix="dup")
    d.columns["d_key"] = HostColumn("d_key", wl.Type.Int(), values=np.zeros(d.rows, np.int32))
    e.register_table(d)
    e.register_table(f)
    b = Batch(e, [wl.batch_query_desc(d, f, lt + 10_000, seg)])
    with pytest.raises(KdbError):
        b.run()
    b.close()
    e.close()
