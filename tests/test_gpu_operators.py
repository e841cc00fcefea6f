"""GPU parity of the per-operator entry points (kdb_scan_select, kdb_hash_*,
kdb_agg_*, kdb_index_*, kdb_skinner_execute), all through the C ABI.

Selections and joins are index work and must match exactly: selection
vectors against numpy's evaluation of the same predicate (three-valued
logic with NULLs), probe pairs against a numpy sort-merge join of the same
keys, in the reference's order (probe row, then build insertion order).
Group-by results are compared with the CPU oracle running the equivalent
GROUP_BY_AGGREGATE plan: keys, counts, MIN/MAX and integer sums exactly,
float64 sums and averages within 1e-12 relative.
"""

import numpy as np
import pytest

from kushdb_b200 import workloads as wl
from kushdb_b200.data import HostColumn, HostTable, catalog_of
from kushdb_b200.plan import (AggregateExpression, And, ColRef, Count, GroupByAggregateOperator, Leq, Lt,
                              LiteralExpression, Literal, Geq, OperatorSchema, OutputOperator, ScanOperator,
                              Type, VirtualColumnRefExpression, VirtColRef, IsNull, Not, Or, Eq)
from parity import compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from kushdb_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()


def _oracle(*tables):
    from oracle import Oracle
    o = Oracle()
    for t in tables:
        o.register_table(t)
    return o


def V(t, idx, nullable=False):
    return VirtualColumnRefExpression(t, nullable, idx)


# ---------------------------------------------------------------------------
# scan-select
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("rows", [0, 1, 1023, 1024, 1025, 77_777, 1_000_000])
def test_scan_select_matches_numpy(engine, rows):
    from kushdb_b200.operators import scan_select
    t = wl.scan_agg_table(rows=rows, name=f"ops_sales_{rows}")
    engine.register_table(t)
    from kushdb_b200.plan import EPOCH_JDN
    f = And([Lt(V(Type.Date(), 0), LiteralExpression(Type.Date(), 9300 + EPOCH_JDN)),
             Geq(V(Type.Real(), 1), Literal(0.05)), Leq(V(Type.Real(), 1), Literal(0.07))])
    sv = scan_select(engine, t.name, ["s_date", "s_discount"], f)
    d = t.columns["s_date"].values
    disc = t.columns["s_discount"].values
    want = np.nonzero((d < 9300 + EPOCH_JDN) & (disc >= 0.05) & (disc <= 0.07))[0]
    got = sv.rows()
    assert len(sv) == len(want)
    np.testing.assert_array_equal(got, want)


def test_scan_select_three_valued_logic(engine):
    """NULL inputs: a comparison with NULL is NULL, NULL AND FALSE is FALSE,
    NULL OR TRUE is TRUE; only TRUE rows qualify."""
    from kushdb_b200.operators import scan_select
    rng = np.random.default_rng(5)
    n = 50_000
    a = rng.integers(0, 100, n).astype(np.int32)
    b = rng.integers(0, 100, n).astype(np.int32)
    an = (rng.random(n) < 0.2).astype(np.int8)
    bn = (rng.random(n) < 0.3).astype(np.int8)
    t = HostTable("ops_nulls")
    t.add(HostColumn("a", Type.Int(), values=a, nulls=an))
    t.add(HostColumn("b", Type.Int(), values=b, nulls=bn))
    engine.register_table(t)
    # (a < 40 OR b >= 70) AND NOT (b IS NULL)
    f = And([Or([Lt(V(Type.Int(), 0, True), Literal(40)), Geq(V(Type.Int(), 1, True), Literal(70))]),
             Not(IsNull(V(Type.Int(), 1, True)))])
    got = scan_select(engine, t.name, ["a", "b"], f).rows()
    a_lt = np.where(an == 1, -1, (a < 40).astype(int))   # -1 = NULL
    b_ge = np.where(bn == 1, -1, (b >= 70).astype(int))
    orv = np.where((a_lt == 1) | (b_ge == 1), 1, np.where((a_lt == -1) | (b_ge == -1), -1, 0))
    want = np.nonzero((orv == 1) & (bn == 0))[0]
    np.testing.assert_array_equal(got, want)


def test_scan_select_nothing_and_everything(engine):
    from kushdb_b200.operators import scan_select
    t = wl.scan_agg_table(rows=3000, name="ops_sales_all")
    engine.register_table(t)
    assert len(scan_select(engine, t.name, ["s_price"], Lt(V(Type.Real(), 0), Literal(0.0)))) == 0
    np.testing.assert_array_equal(
        scan_select(engine, t.name, ["s_price"], Geq(V(Type.Real(), 0), Literal(0.0))).rows(), np.arange(3000))


# ---------------------------------------------------------------------------
# hash build / probe
# ---------------------------------------------------------------------------

def _join_pairs(bkeys, bnull, bsel, pkeys, pnull, psel):
    """numpy sort-merge join: (probe row, build row) ascending."""
    brows = np.arange(len(bkeys)) if bsel is None else bsel
    prows = np.arange(len(pkeys)) if psel is None else psel
    if bnull is not None:
        brows = brows[bnull[brows] == 0]
    if pnull is not None:
        prows = prows[pnull[prows] == 0]
    bk = bkeys[brows].astype(np.int64)
    order = np.lexsort((brows, bk))
    bk, brows = bk[order], brows[order]
    pk = pkeys[prows].astype(np.int64)
    lo = np.searchsorted(bk, pk, "left")
    hi = np.searchsorted(bk, pk, "right")
    cnt = hi - lo
    p_out = np.repeat(prows, cnt)
    starts = np.repeat(lo, cnt)
    offs = np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    b_out = brows[starts + offs]
    order = np.lexsort((b_out, p_out))
    return p_out[order].astype(np.int32), b_out[order].astype(np.int32)


def _key_table(name, keys, nulls=None, dtype=np.int32, tname="INT"):
    t = HostTable(name)
    t.add(HostColumn("k", Type(tname), values=np.asarray(keys, dtype), nulls=nulls))
    t.add(HostColumn("v", Type.Int(), values=np.arange(len(keys), dtype=np.int32)))
    return t


# (262,000 build rows over 64 partitions straddle the size at which a
# probe-side sub-table still fits a shared-memory table buffer; with 16
# partitions none fits and they are probed in HBM)
@pytest.mark.parametrize("fanout", [1, 16, 64, 1024, 0])
@pytest.mark.parametrize("nb,np_,dup", [(1, 1, 1), (1000, 5000, 1), (150_000, 600_000, 1), (40_000, 200_000, 4),
                                        (262_000, 600_000, 1)])
def test_hash_join_matches_numpy(engine, fanout, nb, np_, dup):
    from kushdb_b200.operators import HashTable
    rng = np.random.default_rng(nb + np_)
    bkeys = rng.integers(0, max(nb // dup, 1), nb).astype(np.int32)
    bnull = (rng.random(nb) < 0.05).astype(np.int8)
    pkeys = rng.integers(-10, max(nb // dup, 1) + 10, np_).astype(np.int32)
    pnull = (rng.random(np_) < 0.05).astype(np.int8)
    b = _key_table(f"ops_b_{nb}_{dup}", bkeys, bnull)
    p = _key_table(f"ops_p_{np_}_{dup}", pkeys, pnull)
    engine.register_table(b)
    engine.register_table(p)
    ht = HashTable(engine, b.name, "k", load_factor=0.5, fanout=fanout)
    got_p, got_b = ht.probe(p.name, "k")
    want_p, want_b = _join_pairs(bkeys, bnull, None, pkeys, pnull, None)
    np.testing.assert_array_equal(got_p, want_p)
    np.testing.assert_array_equal(got_b, want_b)
    # unordered probes return the same pairs
    up, ub = ht.probe(p.name, "k", ordered=False)
    o = np.lexsort((ub, up))
    np.testing.assert_array_equal(up[o], want_p)
    np.testing.assert_array_equal(ub[o], want_b)


def test_hash_join_with_selections_and_bigint(engine):
    from kushdb_b200.operators import HashTable, scan_select
    rng = np.random.default_rng(11)
    nb, np_ = 60_000, 250_000
    bkeys = (rng.integers(0, 30_000, nb) * 1_000_003_001).astype(np.int64)  # beyond 32 bits
    pkeys = (rng.integers(0, 32_000, np_) * 1_000_003_001).astype(np.int64)
    b = _key_table("ops_big_b", bkeys, dtype=np.int64, tname="BIGINT")
    p = _key_table("ops_big_p", pkeys, dtype=np.int64, tname="BIGINT")
    engine.register_table(b)
    engine.register_table(p)
    bs = scan_select(engine, b.name, ["v"], Lt(V(Type.Int(), 0), Literal(40_000)))
    ps = scan_select(engine, p.name, ["v"], Geq(V(Type.Int(), 0), Literal(1000)))
    for fanout in (1, 256):
        ht = HashTable(engine, b.name, "k", sel=bs, fanout=fanout)
        got_p, got_b = ht.probe(p.name, "k", sel=ps)
        want_p, want_b = _join_pairs(bkeys, None, bs.rows(), pkeys, None, ps.rows())
        np.testing.assert_array_equal(got_p, want_p)
        np.testing.assert_array_equal(got_b, want_b)


def test_hash_join_empty_sides(engine):
    from kushdb_b200.operators import HashTable, scan_select
    b = _key_table("ops_e_b", np.arange(100))
    p = _key_table("ops_e_p", np.arange(50))
    engine.register_table(b)
    engine.register_table(p)
    none_b = scan_select(engine, b.name, ["v"], Lt(V(Type.Int(), 0), Literal(0)))
    for fanout in (1, 64):
        ht = HashTable(engine, b.name, "k", sel=none_b, fanout=fanout)
        assert len(ht.probe(p.name, "k")[0]) == 0
        ht2 = HashTable(engine, b.name, "k", fanout=fanout)
        none_p = scan_select(engine, p.name, ["v"], Lt(V(Type.Int(), 0), Literal(0)))
        assert len(ht2.probe(p.name, "k", sel=none_p)[0]) == 0


def test_partitioned_join_beyond_l2(engine):
    """A 30M-row build side (a 512 MiB table at load factor 0.5, four times
    L2): the automatic fan-out partitions it; every probe row finds its key."""
    from kushdb_b200.operators import HashTable
    nb, np_ = 30_000_000, 20_000_000
    rng = np.random.default_rng(3)
    bkeys = rng.permutation(nb).astype(np.int32) + 1
    pkeys = rng.integers(1, nb + 1, np_).astype(np.int32)
    pkeys[::97] = -5  # misses
    b = _key_table("ops_big_build", bkeys)
    p = _key_table("ops_big_probe", pkeys)
    engine.register_table(b)
    engine.register_table(p)
    ht = HashTable(engine, b.name, "k", fanout=0)
    fanout, slots, nbytes = ht.info()
    assert fanout > 1 and nbytes > 126 * 2 ** 20
    got_p, got_b = ht.probe(p.name, "k")
    hit = pkeys != -5
    assert len(got_p) == int(hit.sum())
    np.testing.assert_array_equal(got_p, np.nonzero(hit)[0])
    # build row of key k: inverse permutation
    inv = np.empty(nb, np.int64)
    inv[bkeys - 1] = np.arange(nb)
    np.testing.assert_array_equal(got_b, inv[pkeys[hit] - 1])
    b.columns.clear()
    engine.drop_table(b.name)
    engine.drop_table(p.name)


# ---------------------------------------------------------------------------
# group-by aggregation
# ---------------------------------------------------------------------------

def _agg_plan(table, keys, aggs):
    db = catalog_of([table])
    rel = db[table.name]
    cols = list(dict.fromkeys(list(keys) + [c for _, c in aggs if c is not None]))
    scan_s = OperatorSchema()
    scan_s.AddGeneratedColumns(rel, cols)
    scan = ScanOperator(scan_s, rel)
    gk = [ColRef(scan, k) for k in keys]
    ae = [AggregateExpression(n, ColRef(scan, c)) if c is not None else Count() for n, c in aggs]
    g = OperatorSchema()
    for i, k in enumerate(keys):
        g.AddDerivedColumn(k, VirtColRef(gk[i], i))
    for i, a in enumerate(ae):
        g.AddDerivedColumn(f"agg{i}", VirtColRef(a, len(keys) + i))
    return OutputOperator(GroupByAggregateOperator(g, scan, gk, ae))


def _agg_table(name, n, ngroups, zipf=0.0, seed=1, nulls=True):
    rng = np.random.default_rng(seed)
    if zipf:
        k1 = wl.zipf_keys(seed, n, ngroups, zipf).astype(np.int32)
    else:
        k1 = rng.integers(0, ngroups, n).astype(np.int32)
    t = HostTable(name)
    t.add(HostColumn("k1", Type.Int(), values=k1))
    t.add(HostColumn("k2", Type.SmallInt(), values=rng.integers(0, 3, n).astype(np.int16),
                     nulls=(rng.random(n) < 0.1).astype(np.int8) if nulls else None))
    t.add(HostColumn("price", Type.Real(), values=900 + rng.random(n) * 104100,
                     nulls=(rng.random(n) < 0.05).astype(np.int8) if nulls else None))
    t.add(HostColumn("qty", Type.Int(), values=rng.integers(1, 51, n).astype(np.int32),
                     nulls=(rng.random(n) < 0.05).astype(np.int8) if nulls else None))
    t.add(HostColumn("big", Type.BigInt(), values=rng.integers(-2 ** 40, 2 ** 40, n).astype(np.int64)))
    return t


AGGS = [("SUM", "price"), ("SUM", "qty"), ("MIN", "price"), ("MAX", "qty"), ("AVG", "price"),
        ("COUNT", "qty"), ("COUNT", None), ("MAX", "big")]


@pytest.mark.parametrize("pre", [True, False])
@pytest.mark.parametrize("n,ngroups,zipf", [(1, 1, 0.0), (5000, 7, 0.0), (200_000, 1000, 1.1),
                                            (400_000, 100_000, 1.1), (300_000, 50_000, 0.0)])
def test_group_by_matches_oracle(engine, pre, n, ngroups, zipf):
    from kushdb_b200.operators import AggTable
    t = _agg_table(f"ops_agg_{n}_{ngroups}", n, ngroups, zipf)
    engine.register_table(t)
    a = AggTable(engine, t.name, ["k1", "k2"], AGGS, pre_aggregate=pre)
    a.update()
    got = a.finalize()
    want = _oracle(t).execute(_agg_plan(t, ["k1", "k2"], AGGS))
    assert compare(got, want) == ""


def test_group_by_updates_accumulate_in_insertion_order(engine):
    """Two updates over disjoint selections equal one update over all rows,
    and the groups come out in first-insertion order across the updates."""
    from kushdb_b200.operators import AggTable, scan_select
    t = _agg_table("ops_agg_two", 100_000, 300, seed=4)
    engine.register_table(t)
    lo = scan_select(engine, t.name, ["qty"], Lt(V(Type.Int(), 0, True), Literal(25)))
    hi = scan_select(engine, t.name, ["qty"], Geq(V(Type.Int(), 0, True), Literal(25)))
    a = AggTable(engine, t.name, ["k1"], AGGS)
    a.update(lo)
    a.update(hi)
    got = a.finalize()
    # the same rows in the same order: the oracle over lo's rows, then hi's
    order = np.concatenate([lo.rows(), hi.rows()])
    t2 = HostTable("ops_agg_two_ordered")
    for c in t.columns.values():
        t2.add(HostColumn(c.name, c.type, values=c.values[order],
                          nulls=None if c.nulls is None else c.nulls[order]))
    want = _oracle(t2).execute(_agg_plan(t2, ["k1"], AGGS))
    assert compare(got, want) == ""


def test_group_by_capacity_error(engine):
    from kushdb_b200.engine import KdbError
    from kushdb_b200.operators import AggTable
    t = _agg_table("ops_agg_cap", 10_000, 5000, nulls=False)
    engine.register_table(t)
    a = AggTable(engine, t.name, ["k1"], [("COUNT", None)], max_groups=100)
    with pytest.raises(KdbError) as e:
        a.update()
    assert e.value.code == -4


# ---------------------------------------------------------------------------
# column indexes
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("n,nkeys", [(0, 1), (1, 1), (10_000, 37), (1_000_000, 200_000)])
def test_index_build_matches_numpy(engine, n, nkeys):
    from kushdb_b200.operators import ColumnIndex
    rng = np.random.default_rng(n)
    keys = rng.integers(-nkeys, nkeys, n).astype(np.int32)
    nulls = (rng.random(n) < 0.1).astype(np.int8)
    t = _key_table(f"ops_idx_{n}", keys, nulls)
    engine.register_table(t)
    idx = ColumnIndex.build(engine, t.name, "k")
    valid = nulls == 0
    want_keys = np.unique(keys[valid])
    np.testing.assert_array_equal(idx.keys(), want_keys)
    assert idx.num_rows() == int(valid.sum())
    for k in list(want_keys[:20]) + list(want_keys[-20:]) + [nkeys + 5]:
        np.testing.assert_array_equal(idx.get(k), np.nonzero(valid & (keys == k))[0])


# ---------------------------------------------------------------------------
# Skinner operator
# ---------------------------------------------------------------------------

def test_skinner_operator_matches_plan(engine):
    from kushdb_b200.operators import skinner_execute
    tables, tokens = wl.skinner_tables("star", 5, min_rows=2000, max_rows=8000, zipf_s=1.5, seed=21,
                                       prefix="ops_sk_")
    for t in tables:
        engine.register_table(t)
    plan = wl.skinner_plan(tables, tokens, "star")
    # the SKINNER_JOIN operator under the plan's aggregate / output
    op = plan
    while op.__class__.__name__ != "SkinnerJoinOperator":
        op = op.Child()
    want = _oracle(*tables).execute(OutputOperator(op))
    for policy, seed in (("uct", 0), ("random", 3)):
        got = skinner_execute(engine, op, policy=policy, budget_per_episode=500, seed=seed)
        assert compare(got, want, ordered=False) == ""


# ---------------------------------------------------------------------------
# sort of a table's rows (kdb_sort)
# ---------------------------------------------------------------------------


def _sorted_rows(cols, keys, asc, rows):
    """Python restatement of the ORDER BY order: NULL compares above every
    value (compile/proxy/evaluate.cc:339-351), so it comes after every value
    ascending and before every value descending; a stable sort keeps tied
    rows in input order (Python's reverse=True sort is stable too)."""
    out = list(rows)
    for k, a in reversed(list(zip(keys, asc))):
        vals, nulls = cols[k]
        out.sort(key=lambda r: (1, 0) if nulls[r] else (0, vals[r]), reverse=not a)
    return out


@pytest.mark.parametrize("keys,asc", [(["i"], [True]), (["i"], [False]), (["r", "i"], [False, True]),
                                      (["e", "s", "b"], [True, False, True]), (["big"], [False]),
                                      (["e"], [False])])
@pytest.mark.parametrize("with_sel", [False, True])
def test_sort_rows_matches_order_by_semantics(engine, keys, asc, with_sel):
    from kushdb_b200.operators import scan_select, sort_rows
    from kushdb_b200.plan import EnumRegistry
    EnumRegistry.register(83, ["pear", "apple", "fig", "kiwi"])
    rng = np.random.default_rng(len(keys) * 7 + int(with_sel))
    n = 20_000
    t = HostTable("sort_rows_t")
    t.add(HostColumn("i", Type.Int(), values=rng.integers(-50, 50, n).astype(np.int32),
                     nulls=(rng.random(n) < 0.1).astype(np.int8)))
    t.add(HostColumn("r", Type.Real(), values=rng.integers(-20, 20, n).astype(np.float64) / 4.0,
                     nulls=(rng.random(n) < 0.1).astype(np.int8)))
    t.add(HostColumn("e", Type.Enum(83), values=rng.integers(0, 4, n).astype(np.int32)))
    t.add(HostColumn("s", Type.SmallInt(), values=rng.integers(-3, 3, n).astype(np.int16)))
    t.add(HostColumn("b", Type.Boolean(), values=(rng.random(n) < 0.5).astype(np.int8)))
    t.add(HostColumn("big", Type.BigInt(), values=rng.integers(-(1 << 40), 1 << 40, n).astype(np.int64)))
    t.add(HostColumn("v", Type.Int(), values=np.arange(n, dtype=np.int32)))
    engine.register_table(t)
    names = ["pear", "apple", "fig", "kiwi"]
    cols = {}
    for c in ("i", "r", "s", "b", "big"):
        hc = t.columns[c]
        cols[c] = (hc.values, hc.nulls if hc.nulls is not None else np.zeros(n, np.int8))
    cols["e"] = ([names[x] for x in t.columns["e"].values], np.zeros(n, np.int8))
    rows = list(range(n))
    sel = None
    if with_sel:
        sel = scan_select(engine, t.name, ["v"], Geq(V(Type.Int(), 0), Literal(5000)))
        rows = list(range(5000, n))
    got = sort_rows(engine, t.name, keys, asc, sel=sel).rows()
    assert list(got) == _sorted_rows(cols, keys, asc, rows)
    engine.drop_table(t.name)
