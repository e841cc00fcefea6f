"""Join keys stored in the table slot (32-bit key types) against probe keys
of a wider type: the stored key is compared sign-extended, so negative keys
match and probe values that agree only in their low 32 bits do not.  Also a
build side with duplicate and NULL keys, through the filter in front of the
table."""

import numpy as np
import pytest

from kushdb_b200.data import HostColumn, HostTable, catalog_of
from kushdb_b200.plan import ColRef, HashJoinOperator, OperatorSchema, OutputOperator, ScanOperator, Type
from parity import compare

pytestmark = pytest.mark.gpu


def _join(b, p, bkey, pkey):
    d = catalog_of([b, p])
    bs = OperatorSchema()
    bs.AddGeneratedColumns(d[b.name], [bkey, "tag"])
    ps = OperatorSchema()
    ps.AddGeneratedColumns(d[p.name], [pkey, "val"])
    bscan, pscan = ScanOperator(bs, d[b.name]), ScanOperator(ps, d[p.name])
    js = OperatorSchema()
    js.AddPassthroughColumns(bscan, [bkey, "tag"], 0)
    js.AddPassthroughColumns(pscan, [pkey, "val"], 1)
    return OutputOperator(HashJoinOperator(js, bscan, pscan, [ColRef(bscan, bkey, 0)], [ColRef(pscan, pkey, 1)]))


@pytest.fixture(scope="module")
def engine():
    from kushdb_b200.engine import Engine
    e = Engine(0)
    e.set_prepared_queries(False)
    yield e
    e.close()


def _run(engine, *tables, plan):
    from oracle import Oracle
    o = Oracle()
    for t in tables:
        try:
            engine.drop_table(t.name)
        except Exception:
            pass
        engine.register_table(t)
        o.register_table(t)
    text = plan.to_json()
    return engine.execute(text), o.execute(text)


def test_int_build_bigint_probe(engine):
    bk = np.array([-5, -1, 0, 1, 3, 7, 7, 2147483647, -2147483648], dtype=np.int32)
    b = HostTable("keys_b")
    b.add(HostColumn("k", Type.Int(), values=bk))
    b.add(HostColumn("tag", Type.Int(), values=np.arange(len(bk), dtype=np.int32)))
    pk = np.array([-5, 3, 7, 7 + (1 << 32), 3 - (1 << 32), 2147483647, -2147483648, 1 << 40, -1, 11],
                  dtype=np.int64)
    p = HostTable("keys_p")
    p.add(HostColumn("k64", Type.BigInt(), values=pk))
    p.add(HostColumn("val", Type.Int(), values=np.arange(len(pk), dtype=np.int32) * 10))
    got, want = _run(engine, b, p, plan=_join(b, p, "k", "k64"))
    assert want.num_rows == 7  # -5, 3, 7 (two build rows), INT_MAX, INT_MIN, -1
    assert compare(got, want, ordered=False) == ""


@pytest.mark.parametrize("kind", ["int", "date", "smallint"])
def test_duplicates_and_nulls(engine, kind):
    rng = np.random.default_rng(5)
    n_b, n_p = 50_000, 200_000
    t = {"int": (Type.Int(), np.int32), "date": (Type.Date(), np.int32), "smallint": (Type.SmallInt(), np.int16)}[kind]
    bk = rng.integers(-3000, 3000, n_b).astype(t[1])
    b = HostTable("dup_b")
    b.add(HostColumn("k", t[0], values=bk, nulls=(rng.random(n_b) < 0.05).astype(np.int8)))
    b.add(HostColumn("tag", Type.Int(), values=np.arange(n_b, dtype=np.int32)))
    p = HostTable("dup_p")
    p.add(HostColumn("k2", t[0], values=rng.integers(-6000, 6000, n_p).astype(t[1]),
                     nulls=(rng.random(n_p) < 0.05).astype(np.int8)))
    p.add(HostColumn("val", Type.Int(), values=np.arange(n_p, dtype=np.int32)))
    got, want = _run(engine, b, p, plan=_join(b, p, "k", "k2"))
    assert want.num_rows > 0
    assert compare(got, want, ordered=False) == ""
