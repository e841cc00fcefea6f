"""Per-operator API over the C ABI (include/kdb_b200.h, per-operator boundary).

Mirrors the reference runtime structures that its generated code drives one
at a time -- ``runtime::HashTable`` (runtime/hash_table.h:22-38),
``runtime::AggregateHashTable`` with the proxy aggregators
(runtime/aggregate_hash_table.h:28-49, compile/proxy/aggregator.cc),
``MemoryColumnIndex`` / ``ColumnIndex`` (runtime/memory_column_index.cc,
runtime/column_index.cc), ``ScanSelectTranslator`` (scan_select_translator.cc:
92-156) and ``ExecutePermutableSkinnerJoin`` (skinner_join_executor.h:16-25) --
over tables resident in an :class:`~kushdb_b200.engine.Engine`.  Every call
runs hand-written or generated sm_100a kernels; there is no CPU path.
"""

from __future__ import annotations

import ctypes
import json
from typing import Optional, Sequence, Tuple

import numpy as np

from .engine import Engine
from .result import Result

AGG = {"SUM": 0, "MIN": 1, "MAX": 2, "AVG": 3, "COUNT": 4}


def _names(names: Sequence[str]):
    arr = (ctypes.c_char_p * max(len(names), 1))()
    for i, n in enumerate(names):
        arr[i] = n.encode()
    return arr


class SelVec:
    """Ascending row ids of one table (a device selection vector)."""

    def __init__(self, engine: Engine, handle):
        self.engine, self.h = engine, handle

    def __len__(self):
        return int(self.engine.lib.kdb_selvec_size(self.h))

    def rows(self) -> np.ndarray:
        n = len(self)
        out = np.empty(n, np.int32)
        rc = self.engine.lib.kdb_selvec_get(self.h, out.ctypes.data_as(ctypes.c_void_p), n)
        if rc < 0:
            raise RuntimeError(f"kdb_selvec_get failed ({rc})")
        return out

    def close(self):
        if self.h:
            self.engine.lib.kdb_selvec_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def scan_select(engine: Engine, table: str, columns: Sequence[str], filter_expr) -> SelVec:
    """Rows of `table` whose filter (a plan expression over `columns`, bound by
    position through VirtColRef / ColRef indices) is TRUE."""
    engine.register_enums()
    text = json.dumps(filter_expr.to_dict() if hasattr(filter_expr, "to_dict") else filter_expr)
    h = ctypes.c_void_p()
    engine._check(engine.lib.kdb_scan_select(engine.ctx, table.encode(), _names(columns), len(columns),
                                             text.encode(), ctypes.byref(h)))
    return SelVec(engine, h)


def sort_rows(engine: Engine, table: str, keys: Sequence[str], asc: Sequence[bool],
              sel: Optional[SelVec] = None) -> SelVec:
    """Rows of `table` (or of `sel`) in ORDER BY order of `keys` (kdb_sort):
    NULL after values ascending, before them descending; ties keep the
    input order."""
    if len(keys) != len(asc) or not keys:
        raise ValueError("one direction per key")
    engine.register_enums()
    dirs = (ctypes.c_int8 * len(asc))(*[1 if a else 0 for a in asc])
    h = ctypes.c_void_p()
    engine._check(engine.lib.kdb_sort(engine.ctx, table.encode(), _names(keys), dirs, len(keys),
                                      sel.h if sel is not None else None, ctypes.byref(h)))
    return SelVec(engine, h)


class HashTable:
    """A device join table over one integer key column."""

    def __init__(self, engine: Engine, table: str, key: str, sel: Optional[SelVec] = None,
                 load_factor: float = 0.5, fanout: int = 0):
        self.engine = engine
        self.h = ctypes.c_void_p()
        engine._check(engine.lib.kdb_hash_build(engine.ctx, table.encode(), key.encode(),
                                                sel.h if sel is not None else None, load_factor, fanout,
                                                ctypes.byref(self.h)))

    def info(self) -> Tuple[int, int, int]:
        """(fanout, slots, bytes)"""
        f, s, b = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
        self.engine.lib.kdb_hash_info(self.h, ctypes.byref(f), ctypes.byref(s), ctypes.byref(b))
        return f.value, s.value, b.value

    def probe(self, table: str, key: str, sel: Optional[SelVec] = None, ordered: bool = True):
        """(probe rows, build rows) of every pair of equal keys."""
        p = ctypes.c_void_p()
        lib = self.engine.lib
        self.engine._check(lib.kdb_hash_probe(self.engine.ctx, self.h, table.encode(), key.encode(),
                                              sel.h if sel is not None else None, 1 if ordered else 0,
                                              ctypes.byref(p)))
        try:
            n = lib.kdb_pairs_size(p)
            a, b = np.empty(n, np.int32), np.empty(n, np.int32)
            if lib.kdb_pairs_get(p, a.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p), n) < 0:
                raise RuntimeError("kdb_pairs_get failed")
            return a, b
        finally:
            lib.kdb_pairs_free(p)

    def close(self):
        if self.h:
            self.engine.lib.kdb_hash_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class KdbAggSpec(ctypes.Structure):
    _fields_ = [("agg", ctypes.c_int32), ("column", ctypes.c_char_p)]


class AggTable:
    """A device group-by table: keys are columns of `table`, aggregates are
    (name, column or None) pairs, name in SUM/MIN/MAX/AVG/COUNT."""

    def __init__(self, engine: Engine, table: str, keys: Sequence[str], aggs: Sequence[Tuple[str, Optional[str]]],
                 max_groups: int = 0, pre_aggregate: bool = True):
        self.engine = engine
        specs = (KdbAggSpec * len(aggs))()
        self._keep = []
        for i, (name, col) in enumerate(aggs):
            specs[i].agg = AGG[name]
            b = col.encode() if col is not None else None
            self._keep.append(b)
            specs[i].column = b
        self.h = ctypes.c_void_p()
        engine._check(engine.lib.kdb_agg_create(engine.ctx, table.encode(), _names(keys), len(keys),
                                                ctypes.cast(specs, ctypes.c_void_p), len(aggs), max_groups,
                                                ctypes.byref(self.h)))
        engine.lib.kdb_agg_set_pre_aggregation(self.h, 1 if pre_aggregate else 0)

    def update(self, sel: Optional[SelVec] = None) -> None:
        self.engine._check(self.engine.lib.kdb_agg_update(self.engine.ctx, self.h, sel.h if sel is not None else None))

    def finalize(self) -> Result:
        h = ctypes.c_void_p()
        self.engine._check(self.engine.lib.kdb_agg_finalize(self.engine.ctx, self.h, ctypes.byref(h)))
        return Result.from_handle(self.engine.lib, "kdb_", self.engine.ctx, h, owner=self.engine)

    def close(self):
        if self.h:
            self.engine.lib.kdb_agg_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ColumnIndex:
    """key -> ascending row ids, built on the device or read from a .kdbindex."""

    def __init__(self, engine: Engine, handle):
        self.engine, self.h = engine, handle

    @classmethod
    def build(cls, engine: Engine, table: str, column: str) -> "ColumnIndex":
        h = ctypes.c_void_p()
        engine._check(engine.lib.kdb_index_build(engine.ctx, table.encode(), column.encode(), ctypes.byref(h)))
        return cls(engine, h)

    @classmethod
    def open_kdbindex(cls, engine: Engine, path: str, type_str: str) -> "ColumnIndex":
        h = ctypes.c_void_p()
        engine._check(engine.lib.kdb_index_open_kdbindex(engine.ctx, path.encode(), type_str.encode(),
                                                         ctypes.byref(h)))
        return cls(engine, h)

    def num_keys(self) -> int:
        return int(self.engine.lib.kdb_index_num_keys(self.h))

    def num_rows(self) -> int:
        return int(self.engine.lib.kdb_index_num_rows(self.h))

    def keys(self) -> np.ndarray:
        n = self.num_keys()
        out = np.empty(n, np.int64)
        self.engine.lib.kdb_index_keys(self.h, out.ctypes.data_as(ctypes.c_void_p), n)
        return out

    def get(self, key: int) -> np.ndarray:
        n = self.engine.lib.kdb_index_get(self.h, int(key), None, 0)
        if n < 0:
            raise RuntimeError(f"kdb_index_get failed ({n})")
        out = np.empty(n, np.int32)
        if n:
            self.engine.lib.kdb_index_get(self.h, int(key), out.ctypes.data_as(ctypes.c_void_p), n)
        return out

    def close(self):
        if self.h:
            self.engine.lib.kdb_index_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def skinner_execute(engine: Engine, skinner_op, policy: str = "uct", budget_per_episode: int = 1 << 20,
                    seed: int = 0) -> Result:
    """Runs one SKINNER_JOIN operator (children: scans) on its own."""
    engine.register_enums()
    pol = {"uct": 0, "prior": 1, "random": 2}[policy]
    text = json.dumps(skinner_op.to_dict())
    h = ctypes.c_void_p()
    engine._check(engine.lib.kdb_skinner_execute(engine.ctx, text.encode(), pol, budget_per_episode, seed,
                                                 ctypes.byref(h)))
    return Result.from_handle(engine.lib, "kdb_", engine.ctx, h, owner=engine)
