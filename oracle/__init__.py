"""CPU oracle (TEST INFRASTRUCTURE ONLY): ctypes binding of liboracle.so.

Used by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` to check and time against the GPU engine; the product path never
imports it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Dict

import numpy as np

from kushdb_b200.data import HostTable
from kushdb_b200.plan import EnumRegistry, Operator
from kushdb_b200.result import Result, declare_result_api

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libkdbref.so")

_lib = None


def build(ref: bool = False) -> None:
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.check_call(["make", "-s", "-C", HERE] + targets)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P, I32, I64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
        L.kdbo_create.restype = P
        L.kdbo_destroy.argtypes = [P]
        L.kdbo_last_error.restype = ctypes.c_char_p
        L.kdbo_last_error.argtypes = [P]
        L.kdbo_register_column.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                           P, I64, P]
        L.kdbo_register_text_column.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p, P, P, I64, P]
        L.kdbo_register_enum.argtypes = [P, I32, P, P, I32]
        L.kdbo_set_skinner_options.argtypes = [P, I32, I32]
        L.kdbo_execute.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(P)]
        L.kdbo_last_exec_seconds.restype = ctypes.c_double
        L.kdbo_last_exec_seconds.argtypes = [P]
        declare_result_api(L, "kdbo_")
        D = ctypes.c_double
        L.kdbo_baseline_scan_agg.restype = D
        L.kdbo_baseline_scan_agg.argtypes = [P, P, P, I64, I32, D, D, P, P, P]
        L.kdbo_baseline_group_by.restype = D
        L.kdbo_baseline_group_by.argtypes = [P, P, P, P, P, P, P, I64, I32, P, P, P, I32, P]
        L.kdbo_baseline_join_group.restype = D
        L.kdbo_baseline_join_group.argtypes = [P, P, P, I64, I32, I32, P, P, P, I64, I32, P, P, P]
        L.kdbo_baseline_scan_agg_mt.restype = D
        L.kdbo_baseline_scan_agg_mt.argtypes = [P, P, P, I64, I32, D, D, P, P, P, I32]
        L.kdbo_baseline_group_by_mt.restype = D
        L.kdbo_baseline_group_by_mt.argtypes = [P, P, P, P, P, P, P, I64, I32, P, P, P, I32, P, I32]
        L.kdbo_baseline_join_group_mt.restype = D
        L.kdbo_baseline_join_group_mt.argtypes = [P, P, P, I64, I32, I32, P, P, P, I64, I32, P, P, P, I32]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Oracle:
    """One oracle context: registered tables + enum dictionaries."""

    def __init__(self):
        self.lib = lib()
        self.ctx = self.lib.kdbo_create()
        self._keep = []
        self._enums_sent = set()

    def close(self):
        if self.ctx:
            self.lib.kdbo_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.kdbo_last_error(self.ctx).decode())

    def register_enums(self) -> None:
        for k, vals in EnumRegistry.all().items():
            enc = [v.encode() for v in vals]
            off = np.zeros(len(enc) + 1, np.int64)
            off[1:] = np.cumsum([len(b) for b in enc])
            chars = np.frombuffer(b"".join(enc) or b"\0", np.uint8)
            self._check(self.lib.kdbo_register_enum(self.ctx, k, _ptr(off), _ptr(chars), len(enc)))

    def register_table(self, table: HostTable, name: str = None) -> None:
        name = (name or table.name).encode()
        for c in table.columns.values():
            nulls = None if c.nulls is None else np.ascontiguousarray(c.nulls, np.int8)
            if c.type.type_id == "TEXT":
                off = np.ascontiguousarray(c.offsets, np.int64)
                chars = np.ascontiguousarray(c.chars, np.uint8)
                if chars.size == 0:
                    chars = np.zeros(1, np.uint8)
                self._check(self.lib.kdbo_register_text_column(
                    self.ctx, name, c.name.encode(), _ptr(off), _ptr(chars), len(off) - 1, _ptr(nulls)))
            else:
                v = np.ascontiguousarray(c.values)
                self._check(self.lib.kdbo_register_column(
                    self.ctx, name, c.name.encode(), c.type.to_json().encode(), _ptr(v), len(v),
                    _ptr(nulls)))

    def set_skinner_options(self, budget: int = 10000, seed: int = 0):
        self.lib.kdbo_set_skinner_options(self.ctx, budget, seed)

    def execute(self, plan) -> Result:
        text = plan.to_json() if isinstance(plan, Operator) else plan
        self.register_enums()
        h = ctypes.c_void_p()
        self._check(self.lib.kdbo_execute(self.ctx, text.encode(), ctypes.byref(h)))
        return Result.from_handle(self.lib, "kdbo_", self.ctx, h)

    def last_exec_seconds(self) -> float:
        return self.lib.kdbo_last_exec_seconds(self.ctx)


def oracle_for(tables: Dict[str, HostTable]) -> Oracle:
    o = Oracle()
    for t in tables.values():
        o.register_table(t)
    return o


# ---------------------------------------------------------------------------
# Compiled CPU baseline loops (oracle/baseline.cc): the benchmark plans as the
# reference's generated code runs them, one thread.  Each returns
# (seconds, result).
# ---------------------------------------------------------------------------


def host_threads() -> int:
    """Host cores this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def baseline_scan_agg(table, date_lt_jdn: int, lo: float, hi: float, threads: int = 1):
    L = lib()
    c = table.columns
    date = np.ascontiguousarray(c["s_date"].values)
    disc = np.ascontiguousarray(c["s_discount"].values)
    price = np.ascontiguousarray(c["s_price"].values)
    s, n, e = ctypes.c_double(), ctypes.c_int64(), ctypes.c_int8()
    args = [_ptr(date), _ptr(disc), _ptr(price), len(date), date_lt_jdn, lo, hi,
            ctypes.byref(s), ctypes.byref(n), ctypes.byref(e)]
    secs = L.kdbo_baseline_scan_agg(*args) if threads <= 1 else L.kdbo_baseline_scan_agg_mt(*args, threads)
    return secs, (None if e.value else s.value, None if e.value else n.value)


def baseline_group_by(table, date_leq_jdn: int, rank_rf, rank_ls, threads: int = 1):
    L = lib()
    c = table.columns
    arrs = [np.ascontiguousarray(c[k].values) for k in
            ["l_shipdate", "l_returnflag", "l_linestatus", "l_quantity", "l_extendedprice", "l_discount", "l_tax"]]
    rr = np.ascontiguousarray(rank_rf, np.int32)
    rl = np.ascontiguousarray(rank_ls, np.int32)
    out = np.zeros((64, 10), np.float64)
    ng = ctypes.c_int32()
    args = [*[_ptr(a) for a in arrs], len(arrs[0]), date_leq_jdn, _ptr(rr), _ptr(rl), _ptr(out), 64,
            ctypes.byref(ng)]
    secs = L.kdbo_baseline_group_by(*args) if threads <= 1 else L.kdbo_baseline_group_by_mt(*args, threads)
    return secs, out[:min(ng.value, 64)]


def baseline_join_group(build, probe, date_lt_jdn: int, seg: int, top: int = 10, threads: int = 1):
    L = lib()
    b, p = build.columns, probe.columns
    ck, cd, cs = (np.ascontiguousarray(b[k].values) for k in ["c_custkey", "c_date", "c_segment"])
    ok, op, od = (np.ascontiguousarray(p[k].values) for k in ["o_custkey", "o_price", "o_discount"])
    keys = np.zeros(top, np.int32)
    sums = np.zeros(top, np.float64)
    ng = ctypes.c_int32()
    args = [_ptr(ck), _ptr(cd), _ptr(cs), len(ck), date_lt_jdn, seg, _ptr(ok), _ptr(op), _ptr(od), len(ok), top,
            _ptr(keys), _ptr(sums), ctypes.byref(ng)]
    secs = L.kdbo_baseline_join_group(*args) if threads <= 1 else L.kdbo_baseline_join_group_mt(*args, threads)
    return secs, (ng.value, keys, sums)
