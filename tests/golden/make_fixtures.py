"""Generate the golden fixtures under tests/golden/ from the reference's test data.

Reads the reference's end-to-end test inputs (``end_to_end_test/data/*.kdb``,
``*_null.kdb``, ``*.kdbenum``) and expected outputs
(``end_to_end_test/<operator>/*_expected.tbl``) and writes:

* ``tests/golden/tables/<table>.npz`` -- the columns the parity tests scan
  (text columns as int64 offsets + bytes, null flags as int8);
* ``tests/golden/enums.json`` -- enum dictionaries (key -> string);
* ``tests/golden/expected/<operator>/<name>.tbl`` -- the expected tables;
* ``tests/golden/kdb/`` -- the raw reference files (``.kdb``, ``_null.kdb``,
  ``.kdbenum``, ``.kdbindex``) of the small tables in RAW_KDB, byte for byte,
  for the tests of the file readers (kdb_column_open_kdb,
  kdb_enum_open_kdbenum, kdb_index_open_kdbindex).

File formats read (reference):
* fixed-width ``.kdb``: raw little-endian values (runtime/column_data.cc:121-172);
* TEXT ``.kdb``: ``StringMetadata{int32 cardinality; {int32 len; uint64 off}[]}``
  followed by NUL-terminated bytes (runtime/column_data.h:45-57, writer
  runtime/column_data.cc:175-229);
* ``.kdbenum``: ``EnumData{u64 entry_offset; u64 mask; u64 array[]}`` then
  ``EnumEntry{u64 str_offset; u32 str_len; u32 value}`` per key
  (runtime/enum.cc:19-115).

Run once in a container that has the reference checked out:
    python tests/golden/make_fixtures.py /path/to/reference
"""

import json
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# stems whose raw reference files are copied into tests/golden/kdb/
RAW_KDB = ["people_id", "people_name", "people_name_enum", "info_id", "info_cheated", "info_date",
           "info_zscore", "info_num1", "info_num2"]

WIDTH = {"SMALLINT": np.int16, "INT": np.int32, "BIGINT": np.int64, "REAL": np.float64,
         "DATE": np.int32, "BOOLEAN": np.int8, "ENUM": np.int32}

# table -> list of (column, type, data file stem, has null file)
TABLES = {
    "region": [("r_regionkey", "INT", "r_regionkey", False), ("r_name", "TEXT", "r_name", False)],
    "people": [("id", "INT", "people_id", True), ("name", "TEXT", "people_name", True)],
    "people_enum": [("id", "INT", "people_id", True),
                    ("name", "ENUM:people_name_enum", "people_name_enum", True)],
    "info": [("id", "INT", "info_id", True), ("cheated", "BOOLEAN", "info_cheated", True),
             ("date", "DATE", "info_date", True), ("zscore", "REAL", "info_zscore", True),
             ("num1", "SMALLINT", "info_num1", True), ("num2", "BIGINT", "info_num2", True)],
    "lineitem": [("l_orderkey", "INT", "l_orderkey", False),
                 ("l_partkey", "INT", "l_partkey", False),
                 ("l_suppkey", "INT", "l_suppkey", False),
                 ("l_linenumber", "INT", "l_linenumber", False),
                 ("l_quantity", "REAL", "l_quantity", False),
                 ("l_extendedprice", "REAL", "l_extendedprice", False),
                 ("l_discount", "REAL", "l_discount", False),
                 ("l_tax", "REAL", "l_tax", False),
                 ("l_returnflag", "TEXT", "l_returnflag", False),
                 ("l_linestatus", "TEXT", "l_linestatus", False),
                 ("l_shipdate", "DATE", "l_shipdate", False),
                 ("l_commitdate", "DATE", "l_commitdate", False),
                 ("l_receiptdate", "DATE", "l_receiptdate", False)],
    # dictionary-encoded variant used by the reference's EnumSchema()
    # (end_to_end_test/schema.h:259-): same rows, enum flag/status columns
    "lineitem_enum": [("l_shipdate", "DATE", "l_shipdate", False),
                      ("l_returnflag", "ENUM:l_returnflag_enum", "l_returnflag_enum", False),
                      ("l_linestatus", "ENUM:l_linestatus_enum", "l_linestatus_enum", False)],
    "nation": [("n_nationkey", "INT", "n_nationkey", False),
               ("n_regionkey", "INT", "n_regionkey", False)],
    "orders": [("o_orderkey", "INT", "o_orderkey", False), ("o_custkey", "INT", "o_custkey", False),
               ("o_orderdate", "DATE", "o_orderdate", False),
               ("o_shippriority", "INT", "o_shippriority", False),
               ("o_totalprice", "REAL", "o_totalprice", False)],
    "customer": [("c_custkey", "INT", "c_custkey", False), ("c_nationkey", "INT", "c_nationkey", False),
                 ("c_mktsegment", "TEXT", "c_mktsegment", False),
                 ("c_acctbal", "REAL", "c_acctbal", False)],
}

EXPECTED_DIRS = ["tpch", "hash_join", "group_by_aggregate", "aggregate", "scan_select",
                 "select", "order_by", "skinner_join", "simd_scan_select", "cross_product"]
TPCH_KEEP = {"q01_expected.tbl", "q03_expected.tbl", "q06_expected.tbl"}


def read_text(path):
    raw = np.fromfile(path, dtype=np.uint8)
    card = int(raw[:4].view(np.int32)[0])
    slots = raw[8:8 + 16 * card].view(np.dtype([("len", "<i4"), ("pad", "<i4"), ("off", "<u8")]))
    lens = slots["len"].astype(np.int64)
    offs = slots["off"].astype(np.int64)
    out_off = np.zeros(card + 1, dtype=np.int64)
    out_off[1:] = np.cumsum(lens)
    chars = bytearray()
    for o, n in zip(offs, lens):
        chars += raw[o:o + n].tobytes()
    return out_off, np.frombuffer(bytes(chars), dtype=np.uint8)


def read_enum(path):
    raw = np.fromfile(path, dtype=np.uint8)
    entry_offset = int(raw[:8].view(np.uint64)[0])
    entries = []
    pos = entry_offset
    first_str = None
    while first_str is None or pos < first_str:
        str_off, str_len, value = np.frombuffer(raw[pos:pos + 16].tobytes(), dtype=np.dtype(
            [("o", "<u8"), ("l", "<u4"), ("v", "<u4")]))[0]
        if first_str is None:
            first_str = int(str_off)
        entries.append((int(value), raw[int(str_off):int(str_off) + int(str_len)].tobytes().decode()))
        pos += 16
    entries.sort()
    assert [v for v, _ in entries] == list(range(len(entries)))
    return [s for _, s in entries]


def main(ref):
    data = os.path.join(ref, "end_to_end_test", "data")
    out_tables = os.path.join(HERE, "tables")
    os.makedirs(out_tables, exist_ok=True)
    enums = {}
    enum_ids = {}
    schema = {}
    for table, cols in TABLES.items():
        arrays = {}
        schema[table] = []
        for name, typ, stem, has_null in cols:
            if typ.startswith("ENUM:"):
                enum_name = typ.split(":", 1)[1]
                if enum_name not in enum_ids:
                    enum_ids[enum_name] = len(enum_ids)
                    enums[enum_ids[enum_name]] = read_enum(os.path.join(data, enum_name + ".kdbenum"))
                typ = f"ENUM:{enum_ids[enum_name]}"
                arrays[name] = np.fromfile(os.path.join(data, stem + ".kdb"), dtype=np.int32)
            elif typ == "TEXT":
                off, chars = read_text(os.path.join(data, stem + ".kdb"))
                arrays[name + "__off"] = off
                arrays[name + "__chars"] = chars
            else:
                arrays[name] = np.fromfile(os.path.join(data, stem + ".kdb"), dtype=WIDTH[typ])
            if has_null:
                arrays[name + "__null"] = np.fromfile(os.path.join(data, stem + "_null.kdb"),
                                                      dtype=np.int8)
            schema[table].append({"name": name, "type": typ, "nullable": has_null})
        np.savez_compressed(os.path.join(out_tables, table + ".npz"), **arrays)
    with open(os.path.join(HERE, "schema.json"), "w") as f:
        json.dump(schema, f, indent=1)
    with open(os.path.join(HERE, "enums.json"), "w") as f:
        json.dump({str(k): v for k, v in enums.items()}, f)
    raw = os.path.join(HERE, "kdb")
    os.makedirs(raw, exist_ok=True)
    for stem in RAW_KDB:
        for suffix in (".kdb", "_null.kdb", ".kdbenum", ".kdbindex"):
            src = os.path.join(data, stem + suffix)
            if os.path.exists(src):
                shutil.copyfile(src, os.path.join(raw, stem + suffix))
    for d in EXPECTED_DIRS:
        src = os.path.join(ref, "end_to_end_test", d)
        dst = os.path.join(HERE, "expected", d)
        os.makedirs(dst, exist_ok=True)
        for fn in sorted(os.listdir(src)):
            if not fn.endswith("_expected.tbl"):
                continue
            if d == "tpch" and fn not in TPCH_KEEP:
                continue
            shutil.copyfile(os.path.join(src, fn), os.path.join(dst, fn))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("KDB_REFERENCE_DIR", "/root/reference"))
