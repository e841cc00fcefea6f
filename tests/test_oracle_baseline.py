"""The compiled CPU baseline loops (timed as the CPU arm of the benchmark)
compute exactly what the oracle computes on the benchmark plans."""

import numpy as np

import oracle
from kushdb_b200 import workloads as wl
from kushdb_b200.plan import EPOCH_JDN


def _ranks(values):
    order = sorted(range(len(values)), key=lambda k: values[k])
    r = [0] * len(values)
    for i, k in enumerate(order):
        r[k] = i
    return r


def test_scan_agg_baseline_matches_oracle():
    t = wl.scan_agg_table(rows=200_000)
    o = oracle.oracle_for({"t": t})
    ref = o.execute(wl.scan_agg_plan(t))
    _, (s, n) = oracle.baseline_scan_agg(t, 9300 + EPOCH_JDN, 0.05, 0.07)
    assert ref.columns[0].values[0] == s  # same sequential order: bit-identical
    assert ref.columns[1].values[0] == n


def test_group_by_baseline_matches_oracle():
    t = wl.group_by_table(rows=200_000)
    o = oracle.oracle_for({"t": t})
    ref = o.execute(wl.group_by_plan(t))
    _, rows = oracle.baseline_group_by(t, 10471 + EPOCH_JDN, _ranks(wl.RF_VALUES), _ranks(wl.LS_VALUES))
    assert len(rows) == ref.num_rows
    for r in range(ref.num_rows):
        assert rows[r][0] == ref.columns[0].values[r] and rows[r][1] == ref.columns[1].values[r]
        for j in range(2, 9):
            assert rows[r][j] == ref.columns[j].values[r]
        assert int(rows[r][9]) == ref.columns[9].values[r]


def test_join_group_baseline_matches_oracle():
    b, p = wl.join_tables(build_rows=20_000, probe_rows=80_000)
    o = oracle.oracle_for({"b": b, "p": p})
    ref = o.execute(wl.join_plan(b, p))
    ng, keys, sums = oracle.baseline_join_group(b, p, 9204 + EPOCH_JDN, wl.SEG_VALUES.index("BUILDING"))[1]
    assert ng == ref.num_rows
    assert np.array_equal(sums, ref.columns[1].values[:10])
    assert np.array_equal(keys, ref.columns[0].values[:10])


def test_threaded_baselines_match_single_thread():
    """The all-cores CPU arm splits rows over threads and merges partial
    tables: same groups and counts, float sums within 1e-12 relative."""
    t = wl.scan_agg_table(rows=200_000)
    _, (s1, n1) = oracle.baseline_scan_agg(t, 9300 + EPOCH_JDN, 0.05, 0.07)
    _, (s4, n4) = oracle.baseline_scan_agg(t, 9300 + EPOCH_JDN, 0.05, 0.07, threads=4)
    assert n1 == n4 and abs(s1 - s4) <= 1e-12 * abs(s1)
    g = wl.group_by_table(rows=200_000)
    args = (10471 + EPOCH_JDN, _ranks(wl.RF_VALUES), _ranks(wl.LS_VALUES))
    _, r1 = oracle.baseline_group_by(g, *args)
    _, r4 = oracle.baseline_group_by(g, *args, threads=4)
    assert r1.shape == r4.shape
    assert np.array_equal(r1[:, [0, 1, 9]], r4[:, [0, 1, 9]])
    assert np.all(np.abs(r1 - r4) <= 1e-12 * np.maximum(np.abs(r1), 1e-300))
    b, p = wl.join_tables(build_rows=20_000, probe_rows=80_000)
    seg = wl.SEG_VALUES.index("BUILDING")
    ng1, k1, x1 = oracle.baseline_join_group(b, p, 9204 + EPOCH_JDN, seg)[1]
    ng4, k4, x4 = oracle.baseline_join_group(b, p, 9204 + EPOCH_JDN, seg, threads=4)[1]
    assert ng1 == ng4 and np.array_equal(k1, k4)
    assert np.all(np.abs(x1 - x4) <= 1e-12 * np.abs(x1))
