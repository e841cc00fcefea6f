"""The reference file readers on the host, without a GPU (compile-only
context): .kdbindex posting lists parsed from the reference's own files
match the posting lists of the .kdb columns they index, and corrupt or
truncated .kdb / .kdbenum / .kdbindex files are rejected with
KDB_ERR_INVALID before anything is read out of bounds."""

import os
import struct

import numpy as np
import pytest

from kushdb_b200.engine import Engine, KdbError

KDB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kdb")
ERR_INVALID = -1


@pytest.fixture(scope="module")
def dry():
    e = Engine(-1)
    yield e
    e.close()


def _postings(values, nulls):
    out = {}
    for r, (k, n) in enumerate(zip(values.tolist(), nulls.tolist())):
        if not n:
            out.setdefault(k, []).append(r)
    return out


@pytest.mark.parametrize("stem,type_str,dtype", [
    ("people_id", "INT", np.int32), ("info_id", "INT", np.int32), ("info_date", "DATE", np.int32),
    ("info_num1", "SMALLINT", np.int16), ("info_num2", "BIGINT", np.int64), ("info_cheated", "BOOLEAN", np.int8),
    ("people_name_enum", "ENUM:0", np.int32)])
def test_kdbindex_matches_its_column(dry, stem, type_str, dtype):
    """NULL rows are not in the reference's index, exactly as kdb_index_build
    leaves them out."""
    from kushdb_b200.operators import ColumnIndex
    vals = np.fromfile(os.path.join(KDB, stem + ".kdb"), dtype)
    nulls = np.fromfile(os.path.join(KDB, stem + "_null.kdb"), np.int8)
    want = _postings(vals, nulls)
    idx = ColumnIndex.open_kdbindex(dry, os.path.join(KDB, stem + ".kdbindex"), type_str)
    assert idx.num_keys() == len(want)
    assert idx.num_rows() == sum(len(v) for v in want.values())
    np.testing.assert_array_equal(idx.keys(), np.array(sorted(want), np.int64))
    for k, rows in want.items():
        np.testing.assert_array_equal(idx.get(k), np.array(rows, np.int32))
    assert len(idx.get(max(want) + 1)) == 0


def _write(tmp_path, name, data: bytes):
    p = tmp_path / name
    p.write_bytes(data)
    return str(p)


def _text_file(strings, card=None, slots=None):
    card = len(strings) if card is None else card
    meta = struct.pack("<iI", card, 0)
    off = 8 + 16 * len(strings)
    body = b""
    for i, s in enumerate(strings):
        o = off + len(body) if slots is None else slots[i]
        meta += struct.pack("<iIQ", len(s), 0, o)
        body += s + b"\0"
    return meta + body


def test_text_file_reads(dry, tmp_path):
    p = _write(tmp_path, "ok.kdb", _text_file([b"alpha", b"", b"gamma"]))
    dry.open_kdb("t_ok", "s", "TEXT", p)


@pytest.mark.parametrize("case", ["short", "negative_card", "card_past_end", "slot_past_end", "slot_in_meta",
                                  "negative_len"])
def test_corrupt_text_file_is_rejected(dry, tmp_path, case):
    good = _text_file([b"alpha", b"beta"])
    if case == "short":
        data = good[:5]
    elif case == "negative_card":
        data = struct.pack("<i", -3) + good[4:]
    elif case == "card_past_end":
        data = struct.pack("<i", 1000) + good[4:]
    elif case == "slot_past_end":
        data = _text_file([b"alpha", b"beta"], slots=[40, 10_000])
    elif case == "slot_in_meta":
        data = _text_file([b"alpha", b"beta"], slots=[0, 40])
    else:
        data = bytearray(good)
        struct.pack_into("<i", data, 8, -7)
        data = bytes(data)
    p = _write(tmp_path, case + ".kdb", data)
    with pytest.raises(KdbError) as e:
        dry.open_kdb("t_bad_" + case, "s", "TEXT", p)
    assert e.value.code == ERR_INVALID


def test_fixed_width_file_of_wrong_length_is_rejected(dry, tmp_path):
    p = _write(tmp_path, "odd.kdb", b"\0" * 10)
    with pytest.raises(KdbError) as e:
        dry.open_kdb("t_odd", "x", "INT", p)
    assert e.value.code == ERR_INVALID
    n = _write(tmp_path, "odd_null.kdb", b"\0" * 3)
    p2 = _write(tmp_path, "ok.kdb", b"\0" * 8)
    with pytest.raises(KdbError):
        dry.open_kdb("t_odd2", "x", "INT", p2, n)


def test_reference_kdbenum_reads(dry):
    dry.open_kdbenum(7, os.path.join(KDB, "people_name_enum.kdbenum"))


@pytest.mark.parametrize("case", ["short", "bad_offset", "entry_past_end", "string_past_end", "key_out_of_order"])
def test_corrupt_kdbenum_is_rejected(dry, tmp_path, case):
    raw = bytearray(open(os.path.join(KDB, "people_name_enum.kdbenum"), "rb").read())
    entry = struct.unpack_from("<Q", raw, 0)[0]
    if case == "short":
        raw = raw[:12]
    elif case == "bad_offset":
        struct.pack_into("<Q", raw, 0, len(raw) + 100)
    elif case == "entry_past_end":
        struct.pack_into("<Q", raw, entry, len(raw) * 4)
    elif case == "string_past_end":
        struct.pack_into("<I", raw, entry + 16 + 8, 1 << 30)
    else:
        struct.pack_into("<I", raw, entry + 16 + 12, 5)
    p = _write(tmp_path, case + ".kdbenum", bytes(raw))
    with pytest.raises(KdbError) as e:
        dry.open_kdbenum(9, p)
    assert e.value.code == ERR_INVALID


@pytest.mark.parametrize("case", ["short", "mask", "cycle", "posting_past_end", "chain_in_header"])
def test_corrupt_kdbindex_is_rejected(dry, tmp_path, case):
    from kushdb_b200.operators import ColumnIndex
    raw = bytearray(open(os.path.join(KDB, "info_id.kdbindex"), "rb").read())
    mask = struct.unpack_from("<Q", raw, 0)[0]
    first = next(struct.unpack_from("<Q", raw, 8 + 8 * b)[0] for b in range(mask + 1)
                 if struct.unpack_from("<Q", raw, 8 + 8 * b)[0])
    if case == "short":
        raw = raw[:20]
    elif case == "mask":
        struct.pack_into("<Q", raw, 0, 1 << 40)
    elif case == "cycle":
        struct.pack_into("<Q", raw, first + 16, first)  # next -> itself
    elif case == "posting_past_end":
        struct.pack_into("<Q", raw, first + 8, 1 << 40)
    else:
        struct.pack_into("<Q", raw, first + 16, 8)
    p = _write(tmp_path, case + ".kdbindex", bytes(raw))
    with pytest.raises(KdbError) as e:
        ColumnIndex.open_kdbindex(dry, p, "INT")
    assert e.value.code == ERR_INVALID
