"""Serving form: a mix of query shapes (scan + aggregate, group-by, join +
group-by + ORDER BY, Skinner multiway joins) submitted concurrently to the
request loop must give, for every request, the same result as the query run
alone, and the standalone results match the oracle."""

import threading

import pytest

from kushdb_b200 import workloads as wl
from parity import compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    from kushdb_b200.engine import Engine
    from oracle import Oracle
    e = Engine(0)
    o = Oracle()
    sa = wl.scan_agg_table(200_000, seed=3, name="srv_sales")
    gb = wl.group_by_table(300_000, seed=4, name="srv_lineitem")
    build, probe = wl.join_tables(40_000, 160_000, seed=5)
    sk, tokens = wl.skinner_tables("star", 5, min_rows=2_000, max_rows=40_000, seed=6, prefix="srv_sk")
    for t in [sa, gb, build, probe] + sk:
        e.register_table(t)
        o.register_table(t)
    plans = []
    for d in (9000, 9300, 9800):
        plans.append(wl.scan_agg_plan(sa, date_lt=d))
    for d in (10000, 10471):
        plans.append(wl.group_by_plan(gb, date_leq=d))
    for d in (9000, 9204):
        plans.append(wl.join_plan(build, probe, date_lt=d))
    plans.append(wl.skinner_plan(sk, tokens, "star"))
    plans = [p.to_json() for p in plans]
    yield e, o, plans
    e.close()


def test_standalone_matches_oracle(setup):
    e, o, plans = setup
    for p in plans:
        assert compare(e.execute(p), o.execute(p)) == ""


@pytest.mark.parametrize("slots", [1, 4])
def test_mix_matches_alone(setup, slots):
    from kushdb_b200.engine import Server
    e, _, plans = setup
    alone = [e.execute(p) for p in plans]
    reps = 6
    order = [i % len(plans) for i in range(reps * len(plans))]
    tickets = [None] * len(order)
    with Server(e, slots=slots, hbm_budget_bytes=16 << 30) as srv:
        def client(k):  # three clients submit interleaved
            for j in range(k, len(order), 3):
                tickets[j] = srv.submit(plans[order[j]])
        th = [threading.Thread(target=client, args=(k,)) for k in range(3)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        results = [srv.wait(t) for t in tickets]
        st = srv.stats()
    for j, r in enumerate(results):
        assert compare(r, alone[order[j]]) == "", f"request {j} (plan {order[j]})"
    assert st["completed"] == len(order) and st["failed"] == 0
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["peak_in_flight"] <= slots
    if slots > 1:
        assert st["peak_in_flight"] > 1


def test_build_cache_reuses_skinner_children(setup):
    """Requests after the first reuse the Skinner join's filtered children and
    join indexes that the first built (build-cache hits, no new misses) and
    return the query's plain result."""
    from kushdb_b200.engine import Server
    e, _, plans = setup
    sk = plans[-1]
    alone = e.execute(sk)
    with Server(e, slots=2, hbm_budget_bytes=16 << 30) as srv:
        first = srv.wait(srv.submit(sk))
        st0 = srv.stats()
        again = [srv.wait(srv.submit(sk)) for _ in range(3)]
        st = srv.stats()
    assert compare(first, alone) == ""
    for r in again:
        assert compare(r, alone) == ""
    assert st0["build_cache_misses"] > 0 and st0["build_cache_hits"] == 0
    assert st0["build_cache_bytes"] > 0 and st0["build_cache_entries"] == st0["build_cache_misses"]
    assert st["build_cache_misses"] == st0["build_cache_misses"]
    assert st["build_cache_hits"] == 3 * st0["build_cache_misses"]


def test_admission_respects_budget(setup):
    """A budget below every request's footprint admits one query at a time."""
    from kushdb_b200.engine import Server
    e, _, plans = setup
    with Server(e, slots=4, hbm_budget_bytes=1) as srv:
        ts = [srv.submit(p) for p in plans * 2]
        for t in ts:
            srv.wait(t)
        st = srv.stats()
    assert st["completed"] == 2 * len(plans)
    assert st["peak_in_flight"] == 1


def test_errors(setup):
    from kushdb_b200.engine import KdbError, Server
    e, _, plans = setup
    bad = wl.scan_agg_plan(wl.scan_agg_table(10, name="srv_unknown_rel"))
    with Server(e, slots=2) as srv:
        with pytest.raises(KdbError):
            srv.submit("{not json")
        t_bad = srv.submit(bad)
        t_ok = srv.submit(plans[0])
        with pytest.raises(KdbError, match="unknown relation"):
            srv.wait(t_bad)
        assert compare(srv.wait(t_ok), e.execute(plans[0])) == ""
        st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == 1
