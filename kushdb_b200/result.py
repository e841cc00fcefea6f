"""Query results read back through the C ABI into numpy columns.

Both the GPU engine (``kdb_result_*``) and the CPU oracle (``kdbo_result_*``)
export the same accessor set; ``Result.from_handle`` reads either one.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from .data import parse_type
from .plan import Type


@dataclass
class ResultColumn:
    type: Type
    values: object          # np.ndarray (int64 / float64) or list[str] for TEXT
    nulls: np.ndarray       # int8


class Result:
    """A query result.  Columns and the printer-format lines are read from
    the C result handle on first access; the handle is freed with the
    object."""

    def __init__(self, columns: List[ResultColumn] = None, lines: List[str] = None):
        self._columns = columns
        self._lines = lines
        self._src = None

    @property
    def columns(self) -> List[ResultColumn]:
        if self._columns is None:
            self._columns = self._read_columns()
        return self._columns

    @property
    def lines(self) -> List[str]:
        if self._lines is None:
            self._lines = self._read_lines()
        return self._lines

    @property
    def num_rows(self) -> int:
        if self._src is not None and self._columns is None:
            lib, prefix, _ctx, h = self._src
            return int(getattr(lib, prefix + "result_num_rows")(h))
        return len(self.columns[0].nulls) if self.columns else 0

    def row(self, r: int):
        return [None if c.nulls[r] else c.values[r] for c in self.columns]

    @staticmethod
    def from_handle(lib, prefix: str, ctx, handle, owner=None) -> "Result":
        """Takes ownership of `handle`.  `owner` is the engine that made it:
        the printer-format lines need its enum dictionaries, so they are read
        only while it is open (the columns stay readable after it closed)."""
        res = Result()
        res._owner = owner
        res._src = (lib, prefix, ctx, ctypes.c_void_p(handle.value if hasattr(handle, "value") else handle))
        return res

    def close(self):
        if self._src is not None:
            lib, prefix, _ctx, h = self._src
            getattr(lib, prefix + "result_free")(h)
            self._src = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _read_columns(self) -> List[ResultColumn]:
        lib, prefix, _ctx, handle = self._src
        f = lambda n: getattr(lib, prefix + n)  # noqa: E731
        nrows = f("result_num_rows")(handle)
        ncols = f("result_num_cols")(handle)
        cols = []
        buf = ctypes.create_string_buffer(64)
        for c in range(ncols):
            if f("result_col_type")(handle, c, buf, 64) != 0:
                raise RuntimeError("bad result column")
            t = parse_type(buf.value.decode())
            nulls = np.zeros(nrows, np.int8)
            f("result_get_nulls")(handle, c, nulls.ctypes.data_as(ctypes.c_void_p))
            if t.type_id == "REAL":
                vals = np.zeros(nrows, np.float64)
                f("result_get_f64")(handle, c, vals.ctypes.data_as(ctypes.c_void_p))
            elif t.type_id == "TEXT":
                vals = []
                tb = ctypes.create_string_buffer(256)
                for r in range(nrows):
                    n = f("result_get_text")(handle, c, r, tb, 256)
                    if n > 256:
                        tb2 = ctypes.create_string_buffer(int(n))
                        f("result_get_text")(handle, c, r, tb2, n)
                        vals.append(tb2.raw[:n].decode())
                    else:
                        vals.append(tb.raw[:n].decode())
            else:
                vals = np.zeros(nrows, np.int64)
                f("result_get_i64")(handle, c, vals.ctypes.data_as(ctypes.c_void_p))
            cols.append(ResultColumn(t, vals, nulls))
        return cols

    def _read_lines(self) -> List[str]:
        lib, prefix, ctx, handle = self._src
        owner = getattr(self, "_owner", None)
        if owner is not None and getattr(owner, "ctx", None) is None:
            raise RuntimeError("result lines are formatted with the engine's enum dictionaries: "
                               "read them before closing the engine")
        f = lambda n: getattr(lib, prefix + n)  # noqa: E731
        need = f("result_format")(ctx, handle, None, 0)
        tbuf = ctypes.create_string_buffer(int(need))
        f("result_format")(ctx, handle, tbuf, need)
        lines = tbuf.value.decode().split("\n")
        if lines and lines[-1] == "":
            lines.pop()
        return lines


def declare_result_api(lib, prefix: str) -> None:
    """Set ctypes signatures for the shared result accessors."""
    P, I32, I64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    sig = {
        "result_num_rows": (I64, [P]),
        "result_num_cols": (I32, [P]),
        "result_col_type": (ctypes.c_int, [P, I32, ctypes.c_char_p, I32]),
        "result_get_i64": (ctypes.c_int, [P, I32, P]),
        "result_get_f64": (ctypes.c_int, [P, I32, P]),
        "result_get_nulls": (ctypes.c_int, [P, I32, P]),
        "result_get_text": (I64, [P, I32, I64, ctypes.c_char_p, I64]),
        "result_format": (I64, [P, P, ctypes.c_char_p, I64]),
        "result_free": (None, [P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, prefix + name)
        fn.restype = res
        fn.argtypes = args


def compare_tbl(expected: List[str], output: List[str], types: List[Type],
                threshold: float = 1e-5, rel: float = 0.0) -> Optional[str]:
    """CHECK_EQ_TBL (util/test_util.h:82-175): ordered, REAL within an absolute
    threshold, TEXT/ENUM with surrounding quotes stripped, others exact.
    `rel` > 0 also accepts a REAL within that relative distance (a parallel
    summation order moves a sum of magnitude 1e9 by more than 1e-5).
    Returns None when equal, else a description of the first difference."""
    if len(expected) != len(output):
        return f"Differing table sizes: {len(expected)} vs {len(output)}"

    def split(s):
        parts = s.split("|")
        if parts and parts[-1] == "":
            parts.pop()
        return parts

    for i, (e, o) in enumerate(zip(expected, output)):
        se, so = split(e), split(o)
        if len(se) != len(types) or len(so) != len(types):
            return f"row {i}: column count {len(se)}/{len(so)} vs {len(types)}"
        for j, t in enumerate(types):
            ev, ov = se[j], so[j]
            if ev == "":
                if ov != "":
                    return f"({i},{j}) expected NULL got {ov!r}"
                continue
            if t.type_id == "REAL":
                d = abs(float(ev) - float(ov))
                if d >= threshold and d > rel * abs(float(ev)):
                    return f"({i},{j}) {ev} vs {ov}"
            elif t.type_id in ("TEXT", "ENUM"):
                if len(ev) >= 2 and ev[0] == '"' and ev[-1] == '"':
                    ev = ev[1:-1]
                if ev != ov:
                    return f"({i},{j}) {ev!r} vs {ov!r}"
            elif ev != ov:
                return f"({i},{j}) {ev!r} vs {ov!r}"
    return None
