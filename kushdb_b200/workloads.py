"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference quotes TPC-H / JOB shapes (benchmark/tpch1/queries/q06.cc,
q01.cc, q03.cc; benchmark/job/query_runner.cc); their datasets are not
available, so these seeded generators stand in for them with the stated
sizes and value distributions.  Dates are Julian day numbers (days since
1970-01-01 + 2440588, runtime/date.cc:10-25), discount/tax are k/100.

* ``scan_agg``  -- plain scan-select + ungrouped aggregate (1M rows):
  SUM(price*discount), COUNT(*) WHERE date < 9300 AND discount in [0.05, 0.07]
* ``group_by``  -- Q1-shape group-by (6M rows): 2 enum keys, 8 aggregates,
  filter date <= 10471, ORDER BY both keys
* ``join_group``-- Q3-shape hash join + group-by: build 1.5M rows filtered on
  date < 9204 and one segment, probe 6M rows (uniform or Zipf s=1.0 FK),
  GROUP BY build key, SUM(price*(1-discount)), ORDER BY sum DESC
"""

from __future__ import annotations

from typing import Dict, Tuple

import numpy as np

from .data import HostColumn, HostTable, catalog_of
from .plan import (EPOCH_JDN, Add, AggregateOperator, And, Avg, ColRef, ColRefE, Count, Eq, Geq,
                   GroupByAggregateOperator, HashJoinOperator, Leq, Literal, LiteralExpression, Lt,
                   Mul, OperatorSchema, OrderByOperator, OutputOperator, ScanOperator,
                   ScanSelectOperator, Sub, Sum, Type, VirtColRef, EnumRegistry)

MASK64 = (1 << 64) - 1

RF_ENUM_ID, LS_ENUM_ID, SEG_ENUM_ID = 100, 101, 102
RF_VALUES = ["A", "N", "R"]
LS_VALUES = ["F", "O"]
SEG_VALUES = ["AUTOMOBILE", "BUILDING", "FURNITURE", "HOUSEHOLD", "MACHINERY"]


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n splitmix64 outputs for a stream seeded with `seed` (vectorised)."""
    idx = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed & MASK64) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed: int, n: int) -> np.ndarray:
    return (splitmix64(seed, n) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def uniform_int(seed: int, n: int, lo: int, hi_inclusive: int) -> np.ndarray:
    span = hi_inclusive - lo + 1
    return (lo + (splitmix64(seed, n) % np.uint64(span)).astype(np.int64))


def register_enums() -> None:
    EnumRegistry.register(RF_ENUM_ID, RF_VALUES)
    EnumRegistry.register(LS_ENUM_ID, LS_VALUES)
    EnumRegistry.register(SEG_ENUM_ID, SEG_VALUES)


def _price(seed, n):
    return 900.0 + uniform01(seed, n) * 104100.0


def _hundredths(seed, n, hi):
    return uniform_int(seed, n, 0, hi).astype(np.float64) / 100.0


def _dates(seed, n):
    return (uniform_int(seed, n, 8035, 10591) + EPOCH_JDN).astype(np.int32)


# ---------------------------------------------------------------------------
# scan-select + ungrouped aggregate
# ---------------------------------------------------------------------------


def scan_agg_table(rows: int = 1_000_000, seed: int = 42, name: str = "sales") -> HostTable:
    t = HostTable(name)
    t.add(HostColumn("s_key", Type.Int(), values=uniform_int(seed + 1, rows, 0, 999_999).astype(np.int32)))
    t.add(HostColumn("s_price", Type.Real(), values=_price(seed + 2, rows)))
    t.add(HostColumn("s_discount", Type.Real(), values=_hundredths(seed + 3, rows, 10)))
    t.add(HostColumn("s_date", Type.Date(), values=_dates(seed + 4, rows)))
    return t


def scan_agg_plan(table: HostTable, date_lt: int = 9300, disc_lo: float = 0.05,
                  disc_hi: float = 0.07) -> OutputOperator:
    db = catalog_of([table])
    rel = db[table.name]
    scan = OperatorSchema()
    scan.AddGeneratedColumns(rel, ["s_date", "s_discount", "s_price"])
    filters = [Lt(VirtColRef(scan, "s_date"), LiteralExpression(Type.Date(), date_lt + EPOCH_JDN)),
               Geq(VirtColRef(scan, "s_discount"), Literal(disc_lo)),
               Leq(VirtColRef(scan, "s_discount"), Literal(disc_hi))]
    out = OperatorSchema()
    out.AddVirtualPassthroughColumns(scan, ["s_price", "s_discount"])
    sel = ScanSelectOperator(out, scan, rel, filters)
    revenue = Sum(Mul(ColRef(sel, "s_price"), ColRef(sel, "s_discount")))
    cnt = Count()
    schema = OperatorSchema()
    schema.AddDerivedColumn("revenue", VirtColRef(revenue, 0))
    schema.AddDerivedColumn("count", VirtColRef(cnt, 1))
    return OutputOperator(AggregateOperator(schema, sel, [revenue, cnt]))


SCAN_AGG_BYTES_PER_ROW = 4 + 8 + 8  # date + discount + price

# ---------------------------------------------------------------------------
# Q1-shape group-by
# ---------------------------------------------------------------------------

# the 4 populated (returnflag, linestatus) groups of the Q1 shape
GROUPS = [("A", "F"), ("N", "F"), ("N", "O"), ("R", "F")]


def group_by_table(rows: int = 6_000_000, seed: int = 7, name: str = "lineitem_q1") -> HostTable:
    register_enums()
    g = uniform_int(seed + 1, rows, 0, len(GROUPS) - 1)
    rf = np.array([RF_VALUES.index(a) for a, _ in GROUPS], np.int32)[g]
    ls = np.array([LS_VALUES.index(b) for _, b in GROUPS], np.int32)[g]
    t = HostTable(name)
    t.add(HostColumn("l_shipdate", Type.Date(), values=_dates(seed + 2, rows)))
    t.add(HostColumn("l_returnflag", Type.Enum(RF_ENUM_ID), values=rf))
    t.add(HostColumn("l_linestatus", Type.Enum(LS_ENUM_ID), values=ls))
    t.add(HostColumn("l_quantity", Type.Real(), values=uniform_int(seed + 3, rows, 1, 50).astype(np.float64)))
    t.add(HostColumn("l_extendedprice", Type.Real(), values=_price(seed + 4, rows)))
    t.add(HostColumn("l_discount", Type.Real(), values=_hundredths(seed + 5, rows, 10)))
    t.add(HostColumn("l_tax", Type.Real(), values=_hundredths(seed + 6, rows, 8)))
    return t


def group_by_plan(table: HostTable, date_leq: int = 10471) -> OutputOperator:
    db = catalog_of([table])
    rel = db[table.name]
    scan = OperatorSchema()
    cols = ["l_returnflag", "l_linestatus", "l_quantity", "l_extendedprice", "l_discount", "l_tax",
            "l_shipdate"]
    scan.AddGeneratedColumns(rel, cols)
    leq = Leq(VirtColRef(scan, "l_shipdate"), LiteralExpression(Type.Date(), date_leq + EPOCH_JDN))
    out = OperatorSchema()
    out.AddVirtualPassthroughColumns(scan, cols[:-1])
    sel = ScanSelectOperator(out, scan, rel, [leq])
    rf, ls = ColRefE(sel, "l_returnflag"), ColRefE(sel, "l_linestatus")
    aggs = [Sum(ColRef(sel, "l_quantity")), Sum(ColRef(sel, "l_extendedprice")),
            Sum(Mul(ColRef(sel, "l_extendedprice"), Sub(Literal(1.0), ColRef(sel, "l_discount")))),
            Sum(Mul(Mul(ColRef(sel, "l_extendedprice"), Sub(Literal(1.0), ColRef(sel, "l_discount"))),
                    Add(Literal(1.0), ColRef(sel, "l_tax")))),
            Avg(ColRef(sel, "l_quantity")), Avg(ColRef(sel, "l_extendedprice")),
            Avg(ColRef(sel, "l_discount")), Count()]
    g = OperatorSchema()
    g.AddDerivedColumn("l_returnflag", VirtColRef(rf, 0))
    g.AddDerivedColumn("l_linestatus", VirtColRef(ls, 1))
    for i, n in enumerate(["sum_qty", "sum_base_price", "sum_disc_price", "sum_charge", "avg_qty",
                           "avg_price", "avg_disc", "count_order"]):
        g.AddDerivedColumn(n, VirtColRef(aggs[i], i + 2))
    agg = GroupByAggregateOperator(g, sel, [rf, ls], aggs)
    o = OperatorSchema()
    o.AddPassthroughColumns(agg)
    return OutputOperator(OrderByOperator(o, agg, [ColRef(agg, "l_returnflag"), ColRef(agg, "l_linestatus")],
                                          [True, True]))


GROUP_BY_BYTES_PER_ROW = 4 + 4 + 4 + 8 * 4  # date + 2 enums + qty/price/disc/tax

# ---------------------------------------------------------------------------
# Q3-shape hash join + group-by
# ---------------------------------------------------------------------------


def zipf_keys(seed: int, n: int, nkeys: int, s: float = 1.0) -> np.ndarray:
    """Inverse-CDF Zipf(s) over ranks 1..nkeys, ranks mapped to keys by a
    seeded permutation so popularity is independent of key order."""
    w = 1.0 / np.arange(1, nkeys + 1, dtype=np.float64) ** s
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    ranks = np.searchsorted(cdf, uniform01(seed, n), side="right")
    ranks = np.minimum(ranks, nkeys - 1)
    perm = np.argsort(splitmix64(seed + 99, nkeys))
    return (perm[ranks] + 1).astype(np.int32)


def join_tables(build_rows: int = 1_500_000, probe_rows: int = 6_000_000, zipf: bool = False,
                seed: int = 11) -> Tuple[HostTable, HostTable]:
    register_enums()
    b = HostTable("customer_q3")
    b.add(HostColumn("c_custkey", Type.Int(), values=np.arange(1, build_rows + 1, dtype=np.int32)))
    b.add(HostColumn("c_date", Type.Date(), values=_dates(seed + 1, build_rows)))
    b.add(HostColumn("c_segment", Type.Enum(SEG_ENUM_ID),
                     values=uniform_int(seed + 2, build_rows, 0, len(SEG_VALUES) - 1).astype(np.int32)))
    p = HostTable("orders_q3")
    fk = zipf_keys(seed + 3, probe_rows, build_rows) if zipf else \
        uniform_int(seed + 3, probe_rows, 1, build_rows).astype(np.int32)
    p.add(HostColumn("o_custkey", Type.Int(), values=fk))
    p.add(HostColumn("o_price", Type.Real(), values=_price(seed + 4, probe_rows)))
    p.add(HostColumn("o_discount", Type.Real(), values=_hundredths(seed + 5, probe_rows, 10)))
    return b, p


def join_plan(build: HostTable, probe: HostTable, date_lt: int = 9204,
              segment: str = "BUILDING") -> OutputOperator:
    db = catalog_of([build, probe])
    brel, prel = db[build.name], db[probe.name]
    bs = OperatorSchema()
    bs.AddGeneratedColumns(brel, ["c_custkey", "c_date", "c_segment"])
    bf = [Lt(VirtColRef(bs, "c_date"), LiteralExpression(Type.Date(), date_lt + EPOCH_JDN)),
          Eq(VirtColRef(bs, "c_segment"), Literal(segment))]
    bout = OperatorSchema()
    bout.AddVirtualPassthroughColumns(bs, ["c_custkey"])
    bsel = ScanSelectOperator(bout, bs, brel, bf)
    ps = OperatorSchema()
    ps.AddGeneratedColumns(prel, ["o_custkey", "o_price", "o_discount"])
    pscan = ScanOperator(ps, prel)
    js = OperatorSchema()
    js.AddPassthroughColumns(bsel, ["c_custkey"], 0)
    js.AddPassthroughColumns(pscan, ["o_price", "o_discount"], 1)
    join = HashJoinOperator(js, bsel, pscan, [ColRef(bsel, "c_custkey", 0)], [ColRef(pscan, "o_custkey", 1)])
    key = ColRefE(join, "c_custkey")
    revenue = Sum(Mul(ColRef(join, "o_price"), Sub(Literal(1.0), ColRef(join, "o_discount"))))
    gs = OperatorSchema()
    gs.AddDerivedColumn("c_custkey", VirtColRef(key, 0))
    gs.AddDerivedColumn("revenue", VirtColRef(revenue, 1))
    agg = GroupByAggregateOperator(gs, join, [key], [revenue])
    os_ = OperatorSchema()
    os_.AddPassthroughColumns(agg)
    return OutputOperator(OrderByOperator(os_, agg, [ColRef(agg, "revenue")], [False]))


def join_bytes(build_rows: int, probe_rows: int, groups: int) -> int:
    # build side read (key, date, segment) + probe read (fk, price, discount)
    # + group table writes (key + sum)
    return build_rows * 12 + probe_rows * 20 + groups * 16


WORKLOADS: Dict[str, str] = {
    "scan_agg": "plain scan-select + ungrouped aggregate",
    "group_by": "Q1-shape group-by, 2 enum keys, 8 aggregates, ORDER BY keys",
    "join_group": "Q3-shape hash join + group-by + ORDER BY sum DESC",
}


# ---------------------------------------------------------------------------
# Skinner multiway join (JOB-style): 6-8 tables, star or chain
# ---------------------------------------------------------------------------

PRINTABLE = np.frombuffer(b"abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ0123456789 _-", np.uint8)


def random_text(seed: int, n: int, token: str, frac: float, lo: int = 8, hi: int = 40) -> HostColumn:
    """n random printable strings of length [lo, hi]; a seeded `frac` of them
    get the 3-char `token` planted (random 3-grams alone almost never match)."""
    lens = uniform_int(seed, n, lo, hi)
    off = np.zeros(n + 1, np.int64)
    off[1:] = np.cumsum(lens)
    chars = PRINTABLE[splitmix64(seed + 1, int(off[-1])) % np.uint64(len(PRINTABLE))].copy()
    plant = uniform01(seed + 2, n) < frac
    where = uniform_int(seed + 3, n, 0, 1 << 30)
    tok = np.frombuffer(token.encode(), np.uint8)
    for r in np.nonzero(plant)[0]:
        L = int(lens[r])
        p = int(off[r]) + int(where[r] % (L - len(tok) + 1))
        chars[p:p + len(tok)] = tok
    return HostColumn("", Type.Text(), offsets=off, chars=chars)


def skinner_tables(shape: str = "star", n_tables: int = 6, min_rows: int = 10_000, max_rows: int = 3_000_000,
                   zipf_s: float = 0.0, seed: int = 5, prefix: str = "j"):
    """Tables for a multiway join.  star: table 0 is the fact table with a
    foreign key into each other table's primary key; chain: table i+1 has a
    foreign key into table i.  Every table has an int32 primary key, and a
    text column with a planted token on a 2-10% share of rows."""
    rng_sizes = np.exp(np.log(min_rows) + uniform01(seed, n_tables) * (np.log(max_rows) - np.log(min_rows)))
    sizes = [int(x) for x in rng_sizes]
    if shape == "star":  # the fact table is the largest
        sizes.sort(reverse=True)
    tables = []
    tokens = []
    for i in range(n_tables):
        n = sizes[i]
        t = HostTable(f"{prefix}{i}")
        t.add(HostColumn("pk", Type.Int(), values=np.arange(n, dtype=np.int32)))
        tok = "".join(chr(c) for c in PRINTABLE[splitmix64(seed + 100 + i, 3) % np.uint64(26)])
        frac = 0.02 + 0.08 * float(uniform01(seed + 200 + i, 1)[0])
        txt = random_text(seed + 300 + i, n, tok, frac)
        txt.name = "note"
        t.add(txt)
        tables.append(t)
        tokens.append(tok)
    def fk(seed_, n, target_rows):
        if zipf_s > 0:
            return (zipf_keys(seed_, n, target_rows, zipf_s) - 1).astype(np.int32)
        return uniform_int(seed_, n, 0, target_rows - 1).astype(np.int32)
    if shape == "star":
        for i in range(1, n_tables):
            tables[0].add(HostColumn(f"fk{i}", Type.Int(), values=fk(seed + 400 + i, sizes[0], sizes[i])))
    else:
        for i in range(1, n_tables):
            tables[i].add(HostColumn("fk", Type.Int(), values=fk(seed + 400 + i, sizes[i], sizes[i - 1])))
    return tables, tokens


def skinner_plan(tables, tokens, shape: str = "star", like_tables=(1, 2)):
    """SkinnerJoin of ScanSelect children (LIKE '%tok%' -> CONTAINS on the
    listed tables) with equality join predicates, under an aggregate
    COUNT(*), MIN(pk of table 0)."""
    from .plan import (AggregateOperator, Contains, Min, ScanSelectOperator as SSO, SkinnerJoinOperator)
    db = catalog_of(tables)
    children = []
    for i, t in enumerate(tables):
        rel = db[t.name]
        cols = [c for c in t.columns if c != "note"]
        scan = OperatorSchema()
        scan.AddGeneratedColumns(rel, cols + (["note"] if i in like_tables else []))
        filters = [Contains(VirtColRef(scan, "note"), Literal(tokens[i]))] if i in like_tables else []
        out = OperatorSchema()
        out.AddVirtualPassthroughColumns(scan, cols)
        children.append(SSO(out, scan, rel, filters))
    conds = []
    if shape == "star":
        for i in range(1, len(tables)):
            conds.append(Eq(ColRef(children[0], f"fk{i}", 0), ColRef(children[i], "pk", i)))
    else:
        for i in range(1, len(tables)):
            conds.append(Eq(ColRef(children[i], "fk", i), ColRef(children[i - 1], "pk", i - 1)))
    js = OperatorSchema()
    js.AddPassthroughColumns(children[0], ["pk"], 0)
    join = SkinnerJoinOperator(js, children, conds)
    cnt = Count()
    mn = Min(ColRef(join, "pk"))
    s = OperatorSchema()
    s.AddDerivedColumn("count", VirtColRef(cnt, 0))
    s.AddDerivedColumn("min_pk", VirtColRef(mn, 1))
    return OutputOperator(AggregateOperator(s, join, [cnt, mn]))


# ---------------------------------------------------------------------------
# Batched form: many uneven join + group-by queries of one template
# ---------------------------------------------------------------------------


def batch_tables(n_queries: int = 256, min_fact: int = 10_000, max_fact: int = 6_000_000, seed: int = 21,
                 prefix: str = "bq"):
    """Per query: a dimension table (1/4 of the fact rows; unique int32 key,
    date, segment) and a fact table (foreign key uniform over the dimension
    keys, price, discount); fact rows log-uniform in [min_fact, max_fact].
    The predicate constants give a dimension selectivity uniform in
    [1%, 90%].  Returns [(dim, fact, date_lt_jdn, seg)]."""
    out = []
    sizes = np.exp(np.log(min_fact) + uniform01(seed, n_queries) * (np.log(max_fact) - np.log(min_fact)))
    sel = 0.01 + 0.89 * uniform01(seed + 1, n_queries)
    for q in range(n_queries):
        nf = int(sizes[q])
        nd = max(1, nf // 4)
        s = seed * 1000 + 17 * q
        d = HostTable(f"{prefix}_dim{q}")
        d.add(HostColumn("d_key", Type.Int(), values=(np.arange(nd, dtype=np.int64) * 7 + q).astype(np.int32)))
        d.add(HostColumn("d_date", Type.Date(), values=_dates(s + 1, nd)))
        d.add(HostColumn("d_seg", Type.Int(), values=np.zeros(nd, np.int32)))
        f = HostTable(f"{prefix}_fact{q}")
        fk_idx = uniform_int(s + 2, nf, 0, nd - 1)
        f.add(HostColumn("f_fk", Type.Int(), values=(fk_idx * 7 + q).astype(np.int32)))
        f.add(HostColumn("f_price", Type.Real(), values=_price(s + 3, nf)))
        f.add(HostColumn("f_disc", Type.Real(), values=_hundredths(s + 4, nf, 10)))
        date_lt = EPOCH_JDN + 8035 + int(round(float(sel[q]) * (10591 - 8035 + 1)))
        out.append((d, f, date_lt, 0))
    return out


def batch_plan(dim: HostTable, fact: HostTable, date_lt_jdn: int, seg: int) -> OutputOperator:
    """The plain form of one batched query: HashJoin(ScanSelect(dim),
    Scan(fact)) -> GROUP BY dim key, SUM(price * (1 - discount))."""
    db = catalog_of([dim, fact])
    drel, frel = db[dim.name], db[fact.name]
    ds = OperatorSchema()
    ds.AddGeneratedColumns(drel, ["d_key", "d_date", "d_seg"])
    filt = [Lt(VirtColRef(ds, "d_date"), LiteralExpression(Type.Date(), date_lt_jdn)),
            Eq(VirtColRef(ds, "d_seg"), Literal(int(seg)))]
    dout = OperatorSchema()
    dout.AddVirtualPassthroughColumns(ds, ["d_key"])
    dsel = ScanSelectOperator(dout, ds, drel, filt)
    fs = OperatorSchema()
    fs.AddGeneratedColumns(frel, ["f_fk", "f_price", "f_disc"])
    fscan = ScanOperator(fs, frel)
    js = OperatorSchema()
    js.AddPassthroughColumns(dsel, ["d_key"], 0)
    js.AddPassthroughColumns(fscan, ["f_price", "f_disc"], 1)
    join = HashJoinOperator(js, dsel, fscan, [ColRef(dsel, "d_key", 0)], [ColRef(fscan, "f_fk", 1)])
    key = ColRefE(join, "d_key")
    rev = Sum(Mul(ColRef(join, "f_price"), Sub(Literal(1.0), ColRef(join, "f_disc"))))
    gs = OperatorSchema()
    gs.AddDerivedColumn("d_key", VirtColRef(key, 0))
    gs.AddDerivedColumn("revenue", VirtColRef(rev, 1))
    return OutputOperator(GroupByAggregateOperator(gs, join, [key], [rev]))


def batch_query_desc(dim: HostTable, fact: HostTable, date_lt_jdn: int, seg: int) -> dict:
    return {"dim_table": dim.name, "dim_key": "d_key", "dim_date": "d_date", "dim_seg": "d_seg",
            "fact_table": fact.name, "fact_fk": "f_fk", "fact_price": "f_price", "fact_disc": "f_disc",
            "date_lt": int(date_lt_jdn), "seg": int(seg)}
