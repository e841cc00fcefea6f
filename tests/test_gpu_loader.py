"""The reference's own data files through the C ABI on the GPU: the people,
people_enum and info tables are read from their raw .kdb / _null.kdb /
.kdbenum files (kdb_column_open_kdb, kdb_enum_open_kdbenum; TEXT decoded on
the device) and every golden case runs on them with the reference's expected
output; the .kdbindex files equal the device-built indexes of the same
columns."""

import os

import numpy as np
import pytest

import reference_plans as rp

pytestmark = pytest.mark.gpu

KDB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kdb")

FILES = {
    "people": [("id", "INT", "people_id"), ("name", "TEXT", "people_name")],
    "people_enum": [("id", "INT", "people_id"), ("name", "ENUM:0", "people_name_enum")],
    "info": [("id", "INT", "info_id"), ("cheated", "BOOLEAN", "info_cheated"), ("date", "DATE", "info_date"),
             ("zscore", "REAL", "info_zscore"), ("num1", "SMALLINT", "info_num1"), ("num2", "BIGINT", "info_num2")],
}


@pytest.fixture(scope="module")
def engine():
    from kushdb_b200.engine import Engine
    e = Engine(0)
    e.open_kdbenum(0, os.path.join(KDB, "people_name_enum.kdbenum"))
    for table, cols in FILES.items():
        for col, typ, stem in cols:
            e.open_kdb(table, col, typ, os.path.join(KDB, stem + ".kdb"), os.path.join(KDB, stem + "_null.kdb"))
    for name, t in rp.golden_tables().items():
        if name not in FILES:
            e.register_table(t)
    yield e
    e.close()


def test_text_decoded_on_device_matches_fixture(engine):
    """Every row's name, decoded on the device from the .kdb image, against
    the fixture, matched by id (a scan's rows come out in no particular
    order)."""
    from kushdb_b200.data import catalog_of
    from kushdb_b200.plan import OperatorSchema, OutputOperator, ScanOperator
    t = rp.golden_tables()["people"]
    ids = t.columns["id"].values
    names = t.columns["name"].strings()
    nulls = t.columns["name"].nulls
    want = {int(i): (None if z else n) for i, n, z in zip(ids, names, nulls)}
    rel = catalog_of([t])["people"]
    s = OperatorSchema()
    s.AddGeneratedColumns(rel, ["id", "name"])
    res = engine.execute(OutputOperator(ScanOperator(s, rel)))
    got = {}
    for r in range(res.num_rows):
        i, n = res.row(r)
        got[int(i)] = n
    assert res.num_rows == len(want) == len(got)
    assert got == want


@pytest.mark.parametrize("case", [c for c in rp.CASES if not c.name.startswith("tpch/")],
                         ids=lambda c: c.name)
def test_golden_case_on_files_read_from_disk(engine, case):
    res = engine.execute(case.build())
    err = rp.check(case, res.lines, [c.type for c in res.columns], rel=rp.GPU_REL)
    assert err == "", err


@pytest.mark.parametrize("table,col,stem,typ", [("people", "id", "people_id", "INT"), ("info", "date", "info_date", "DATE"),
                                                ("info", "num2", "info_num2", "BIGINT"),
                                                ("people_enum", "name", "people_name_enum", "ENUM:0")])
def test_kdbindex_equals_device_index(engine, table, col, stem, typ):
    from kushdb_b200.operators import ColumnIndex
    a = ColumnIndex.open_kdbindex(engine, os.path.join(KDB, stem + ".kdbindex"), typ)
    b = ColumnIndex.build(engine, table, col)
    np.testing.assert_array_equal(a.keys(), b.keys())
    assert a.num_rows() == b.num_rows()
    for k in a.keys():
        np.testing.assert_array_equal(a.get(k), b.get(k))
