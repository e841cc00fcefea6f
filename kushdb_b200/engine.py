"""Python host API over the C ABI (include/kdb_b200.h).

``Engine`` owns one ``kdb_ctx``: tables registered with it stay resident in
HBM (runtime::ColumnData replaced by device columns) and plans built with
``kushdb_b200.plan`` run as generated sm_100a pipelines.  There is no CPU
fallback: without the compiled library or a GPU the calls raise.
"""

from __future__ import annotations

import ctypes
import os
from typing import Dict, Optional

import numpy as np

from .data import HostTable
from .plan import EnumRegistry, Operator
from .result import Result, declare_result_api

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkdb_b200.so")

# every symbol include/kdb_b200.h declares
EXPORTS = [
    "kdb_ctx_create", "kdb_ctx_destroy", "kdb_last_error", "kdb_ctx_kernel_launches",
    "kdb_ctx_column_bytes", "kdb_ctx_stream", "kdb_ctx_set_profiling", "kdb_last_query_kernels", "kdb_table_add_column", "kdb_table_add_text_column",
    "kdb_column_open_kdb", "kdb_table_drop", "kdb_table_num_rows", "kdb_enum_register",
    "kdb_enum_open_kdbenum", "kdb_query_execute", "kdb_last_query_device_ms",
    "kdb_result_num_rows", "kdb_result_num_cols", "kdb_result_col_type", "kdb_result_get_i64",
    "kdb_result_get_f64", "kdb_result_get_nulls", "kdb_result_get_text", "kdb_result_format",
    "kdb_result_free", "kdb_sort_pairs", "kdb_ctx_set_skinner", "kdb_last_skinner_episodes",
    "kdb_batch_create", "kdb_batch_configure", "kdb_batch_tune", "kdb_batch_config", "kdb_batch_run",
    "kdb_batch_run_timed", "kdb_batch_result", "kdb_batch_free", "kdb_sort_pairs_noalloc",
    "kdb_server_start", "kdb_server_submit", "kdb_server_poll", "kdb_server_stats", "kdb_server_stop",
    "kdb_last_skinner_work", "kdb_last_skinner_batches", "kdb_mlp_num_features", "kdb_mlp_num_params", "kdb_mlp_create",
    "kdb_mlp_last_error", "kdb_mlp_set_params", "kdb_mlp_get_params", "kdb_mlp_forward", "kdb_mlp_gradient",
    "kdb_mlp_train_step", "kdb_mlp_free", "kdb_ctx_set_skinner_policy", "kdb_last_skinner_samples",
    "kdb_ctx_set_prepared_queries",
    "kdb_scan_select", "kdb_sort", "kdb_selvec_size", "kdb_selvec_get", "kdb_selvec_device_rows", "kdb_selvec_free",
    "kdb_hash_build", "kdb_hash_info", "kdb_hash_probe", "kdb_hash_free", "kdb_pairs_size", "kdb_pairs_get",
    "kdb_pairs_free", "kdb_agg_create", "kdb_agg_set_pre_aggregation", "kdb_agg_update", "kdb_agg_finalize",
    "kdb_agg_free", "kdb_index_build", "kdb_index_open_kdbindex", "kdb_index_num_keys", "kdb_index_num_rows",
    "kdb_index_keys", "kdb_index_get", "kdb_index_free", "kdb_skinner_execute",
    "kdb_query_execute_host", "kdb_ctx_set_ingest", "kdb_ctx_set_option", "kdb_ctx_get_option",
]

_lib = None


class KdbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def load_library(path: str = LIB_PATH):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python kushdb_b200/build.py` (no CPU fallback)")
    L = ctypes.CDLL(path)
    P, I32, I64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    L.kdb_ctx_create.argtypes = [ctypes.c_int, ctypes.POINTER(P)]
    L.kdb_ctx_destroy.argtypes = [P]
    L.kdb_last_error.restype = ctypes.c_char_p
    L.kdb_last_error.argtypes = [P]
    L.kdb_ctx_kernel_launches.restype = I64
    L.kdb_ctx_kernel_launches.argtypes = [P]
    L.kdb_ctx_column_bytes.restype = I64
    L.kdb_ctx_column_bytes.argtypes = [P]
    L.kdb_ctx_stream.restype = P
    L.kdb_ctx_stream.argtypes = [P]
    L.kdb_ctx_set_profiling.argtypes = [P, ctypes.c_int]
    L.kdb_last_query_kernels.restype = I64
    L.kdb_last_query_kernels.argtypes = [P, ctypes.c_char_p, I64]
    L.kdb_table_add_column.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, P, I64, P]
    L.kdb_table_add_text_column.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p, P, P, I64, P]
    L.kdb_column_open_kdb.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                      ctypes.c_char_p, ctypes.c_char_p]
    L.kdb_table_drop.argtypes = [P, ctypes.c_char_p]
    L.kdb_table_num_rows.restype = I64
    L.kdb_table_num_rows.argtypes = [P, ctypes.c_char_p]
    L.kdb_enum_register.argtypes = [P, I32, P, P, I32]
    L.kdb_enum_open_kdbenum.argtypes = [P, I32, ctypes.c_char_p]
    L.kdb_query_execute.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(P)]
    L.kdb_last_query_device_ms.restype = ctypes.c_double
    L.kdb_last_query_device_ms.argtypes = [P]
    L.kdb_sort_pairs.argtypes = [P, P, P, I64, I32]
    L.kdb_ctx_set_skinner.argtypes = [P, I64, ctypes.c_uint32]
    L.kdb_batch_create.argtypes = [P, P, I32, ctypes.POINTER(P)]
    L.kdb_batch_configure.argtypes = [P, I32, ctypes.c_double, I32]
    L.kdb_batch_tune.argtypes = [P, I32, ctypes.c_char_p, I64]
    L.kdb_batch_config.argtypes = [P, P, P, P]
    L.kdb_batch_run.argtypes = [P]
    L.kdb_batch_run_timed.restype = ctypes.c_double
    L.kdb_batch_run_timed.argtypes = [P, I32]
    L.kdb_batch_result.restype = I64
    L.kdb_batch_result.argtypes = [P, I32, P, P, I64]
    L.kdb_batch_free.argtypes = [P]
    L.kdb_last_skinner_episodes.restype = I64
    L.kdb_last_skinner_episodes.argtypes = [P]
    L.kdb_sort_pairs_noalloc.argtypes = [P, P, I64, I32, P]
    L.kdb_server_start.argtypes = [P, I32, I64, ctypes.POINTER(P)]
    L.kdb_server_submit.restype = I64
    L.kdb_server_submit.argtypes = [P, ctypes.c_char_p]
    L.kdb_server_poll.argtypes = [P, I64, I64, ctypes.POINTER(P)]
    L.kdb_server_stats.restype = I64
    L.kdb_server_stats.argtypes = [P, ctypes.c_char_p, I64]
    L.kdb_server_stop.argtypes = [P]
    L.kdb_ctx_set_prepared_queries.argtypes = [P, I32]
    L.kdb_last_skinner_work.restype = I64
    L.kdb_last_skinner_work.argtypes = [P]
    L.kdb_last_skinner_batches.restype = I64
    L.kdb_last_skinner_batches.argtypes = [P]
    L.kdb_mlp_num_features.restype = I32
    L.kdb_mlp_num_features.argtypes = []
    L.kdb_mlp_num_params.restype = I64
    L.kdb_mlp_num_params.argtypes = []
    L.kdb_mlp_create.argtypes = [P, ctypes.c_uint32, ctypes.POINTER(P)]
    L.kdb_mlp_last_error.restype = ctypes.c_char_p
    L.kdb_mlp_last_error.argtypes = [P]
    L.kdb_mlp_set_params.argtypes = [P, P, I64]
    L.kdb_mlp_get_params.argtypes = [P, P, I64]
    L.kdb_mlp_forward.argtypes = [P, P, I64, P]
    L.kdb_mlp_gradient.argtypes = [P, P, P, I64, P, ctypes.POINTER(ctypes.c_double)]
    L.kdb_mlp_train_step.argtypes = [P, P, P, I64, ctypes.c_float, ctypes.POINTER(ctypes.c_double)]
    L.kdb_mlp_free.argtypes = [P]
    L.kdb_ctx_set_skinner_policy.argtypes = [P, I32, P, I32]
    L.kdb_last_skinner_samples.restype = I64
    L.kdb_last_skinner_samples.argtypes = [P, P, P, I64]
    # per-operator boundary
    CP = ctypes.c_char_p
    L.kdb_scan_select.argtypes = [P, CP, P, I32, CP, ctypes.POINTER(P)]
    L.kdb_sort.argtypes = [P, CP, P, P, I32, P, ctypes.POINTER(P)]
    L.kdb_selvec_size.restype = I64
    L.kdb_selvec_size.argtypes = [P]
    L.kdb_selvec_get.restype = I64
    L.kdb_selvec_get.argtypes = [P, P, I64]
    L.kdb_selvec_device_rows.restype = P
    L.kdb_selvec_device_rows.argtypes = [P]
    L.kdb_selvec_free.argtypes = [P]
    L.kdb_hash_build.argtypes = [P, CP, CP, P, ctypes.c_double, I32, ctypes.POINTER(P)]
    L.kdb_hash_info.argtypes = [P, P, P, P]
    L.kdb_hash_probe.argtypes = [P, P, CP, CP, P, I32, ctypes.POINTER(P)]
    L.kdb_hash_free.argtypes = [P]
    L.kdb_pairs_size.restype = I64
    L.kdb_pairs_size.argtypes = [P]
    L.kdb_pairs_get.restype = I64
    L.kdb_pairs_get.argtypes = [P, P, P, I64]
    L.kdb_pairs_free.argtypes = [P]
    L.kdb_agg_create.argtypes = [P, CP, P, I32, P, I32, I64, ctypes.POINTER(P)]
    L.kdb_agg_set_pre_aggregation.argtypes = [P, I32]
    L.kdb_agg_update.argtypes = [P, P, P]
    L.kdb_agg_finalize.argtypes = [P, P, ctypes.POINTER(P)]
    L.kdb_agg_free.argtypes = [P]
    L.kdb_index_build.argtypes = [P, CP, CP, ctypes.POINTER(P)]
    L.kdb_index_open_kdbindex.argtypes = [P, CP, CP, ctypes.POINTER(P)]
    L.kdb_index_num_keys.restype = I64
    L.kdb_index_num_keys.argtypes = [P]
    L.kdb_index_num_rows.restype = I64
    L.kdb_index_num_rows.argtypes = [P]
    L.kdb_index_keys.restype = I64
    L.kdb_index_keys.argtypes = [P, P, I64]
    L.kdb_index_get.restype = I64
    L.kdb_index_get.argtypes = [P, I64, P, I64]
    L.kdb_index_free.argtypes = [P]
    L.kdb_skinner_execute.argtypes = [P, CP, I32, I64, ctypes.c_uint32, ctypes.POINTER(P)]
    L.kdb_query_execute_host.argtypes = [P, CP, P, I32, ctypes.POINTER(P)]
    L.kdb_ctx_set_ingest.argtypes = [P, I64, I32]
    L.kdb_ctx_set_option.argtypes = [P, CP, CP]
    L.kdb_ctx_get_option.restype = I64
    L.kdb_ctx_get_option.argtypes = [P, CP, ctypes.c_char_p, I64]
    declare_result_api(L, "kdb_")
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class HostColumnSpec(ctypes.Structure):
    """kdb_host_column"""
    _fields_ = [("table", ctypes.c_char_p), ("column", ctypes.c_char_p), ("type", ctypes.c_char_p),
                ("data", ctypes.c_void_p), ("n", ctypes.c_int64), ("nulls", ctypes.c_void_p)]


class Engine:
    """One device context.  ``device=-1`` makes a compile-only context: every
    pipeline is generated and compiled by NVRTC but nothing runs (no GPU
    needed); results are then empty."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.kdb_ctx_create(device, ctypes.byref(h))
        if rc != 0:
            raise KdbError(rc, f"kdb_ctx_create({device}) failed (no CUDA device?)")
        self.ctx = h
        self.device = device
        self._enums_sent: Dict[int, int] = {}

    def close(self):
        if self.ctx:
            self.lib.kdb_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != 0:
            raise KdbError(rc, self.lib.kdb_last_error(self.ctx).decode())

    def register_enums(self) -> None:
        for k, vals in EnumRegistry.all().items():
            key = tuple(vals)
            if self._enums_sent.get(k) == key:
                continue
            self._enums_sent[k] = key
            enc = [v.encode() for v in vals]
            off = np.zeros(len(enc) + 1, np.int64)
            off[1:] = np.cumsum([len(b) for b in enc])
            chars = np.frombuffer(b"".join(enc) or b"\0", np.uint8)
            self._check(self.lib.kdb_enum_register(self.ctx, k, _ptr(off), _ptr(chars), len(enc)))

    def register_table(self, table: HostTable, name: Optional[str] = None) -> None:
        name = (name or table.name).encode()
        for c in table.columns.values():
            nulls = None if c.nulls is None else np.ascontiguousarray(c.nulls, np.int8)
            if c.type.type_id == "TEXT":
                off = np.ascontiguousarray(c.offsets, np.int64)
                chars = np.ascontiguousarray(c.chars, np.uint8)
                if chars.size == 0:
                    chars = np.zeros(1, np.uint8)
                self._check(self.lib.kdb_table_add_text_column(
                    self.ctx, name, c.name.encode(), _ptr(off), _ptr(chars), len(off) - 1, _ptr(nulls)))
            else:
                v = np.ascontiguousarray(c.values)
                self._check(self.lib.kdb_table_add_column(
                    self.ctx, name, c.name.encode(), c.type.to_json().encode(), _ptr(v), len(v),
                    _ptr(nulls)))

    def execute_host(self, plan, tables, fetch: bool = True):
        """End to end from host memory: brings every fixed-width column of
        `tables` into HBM (chunked copies on several streams, all in flight
        together) and runs the plan over them (kdb_query_execute_host)."""
        text = plan.to_json() if isinstance(plan, Operator) else plan
        if isinstance(text, str):
            text = text.encode()
        self.register_enums()
        specs, keep = [], []
        for t in tables:
            for c in t.columns.values():
                if c.type.type_id == "TEXT":
                    raise ValueError("execute_host takes fixed-width columns")
                v = np.ascontiguousarray(c.values)
                nl = None if c.nulls is None else np.ascontiguousarray(c.nulls, np.int8)
                names = (t.name.encode(), c.name.encode(), c.type.to_json().encode())
                keep.append((v, nl, names))
                specs.append((names, v, nl))
        arr = (HostColumnSpec * max(len(specs), 1))()
        for i, (names, v, nl) in enumerate(specs):
            arr[i].table, arr[i].column, arr[i].type = names
            arr[i].data = v.ctypes.data_as(ctypes.c_void_p)
            arr[i].n = len(v)
            arr[i].nulls = None if nl is None else nl.ctypes.data_as(ctypes.c_void_p)
        h = ctypes.c_void_p()
        self._check(self.lib.kdb_query_execute_host(self.ctx, text, ctypes.cast(arr, ctypes.c_void_p), len(specs),
                                                    ctypes.byref(h)))
        del keep
        if not fetch:
            n = self.lib.kdb_result_num_rows(h)
            self.lib.kdb_result_free(h)
            return n
        return Result.from_handle(self.lib, "kdb_", self.ctx, h, owner=self)

    def open_kdb(self, table: str, column: str, type_str: str, path: str, null_path: str = "") -> None:
        """Reads a reference .kdb column file (and its _null.kdb) into HBM."""
        self._check(self.lib.kdb_column_open_kdb(self.ctx, table.encode(), column.encode(), type_str.encode(),
                                                 path.encode(), null_path.encode()))

    def open_kdbenum(self, enum_id: int, path: str) -> None:
        """Reads a reference .kdbenum dictionary."""
        self._check(self.lib.kdb_enum_open_kdbenum(self.ctx, enum_id, path.encode()))

    def set_option(self, name: str, value: Optional[str] = "1") -> None:
        """Sets (value None: removes) a KDB_* code-generation switch."""
        self._check(self.lib.kdb_ctx_set_option(self.ctx, name.encode(),
                                                None if value is None else str(value).encode()))

    def get_option(self, name: str) -> Optional[str]:
        n = self.lib.kdb_ctx_get_option(self.ctx, name.encode(), None, 0)
        if n <= 0:
            return None
        buf = ctypes.create_string_buffer(n)
        self.lib.kdb_ctx_get_option(self.ctx, name.encode(), buf, n)
        return buf.value.decode()

    def set_ingest(self, chunk_bytes: int = 64 << 20, streams: int = 2) -> None:
        self._check(self.lib.kdb_ctx_set_ingest(self.ctx, chunk_bytes, streams))

    def drop_table(self, name: str) -> None:
        self._check(self.lib.kdb_table_drop(self.ctx, name.encode()))

    def execute(self, plan, fetch: bool = True):
        """Runs the plan; returns a Result (fetch=True) or the row count."""
        text = plan.to_json() if isinstance(plan, Operator) else plan
        if isinstance(text, str):
            text = text.encode()
        self.register_enums()
        h = ctypes.c_void_p()
        self._check(self.lib.kdb_query_execute(self.ctx, text, ctypes.byref(h)))
        if not fetch:
            n = self.lib.kdb_result_num_rows(h)
            self.lib.kdb_result_free(h)
            return n
        return Result.from_handle(self.lib, "kdb_", self.ctx, h, owner=self)

    def set_prepared_queries(self, on: bool) -> None:
        """Replay repeated plans as recorded CUDA graphs (default on)."""
        self._check(self.lib.kdb_ctx_set_prepared_queries(self.ctx, 1 if on else 0))

    def last_device_ms(self) -> float:
        return self.lib.kdb_last_query_device_ms(self.ctx)

    def kernel_launches(self) -> int:
        return self.lib.kdb_ctx_kernel_launches(self.ctx)

    def sort_pairs(self, d_keys: int, d_vals: int, n: int, key_bits: int = 64) -> None:
        """Stable device sort of n (uint64 key, uint32 value) pairs in place."""
        self._check(self.lib.kdb_sort_pairs(self.ctx, ctypes.c_void_p(d_keys), ctypes.c_void_p(d_vals), n, key_bits))

    def set_skinner(self, budget_per_episode: int = 1 << 20, seed: int = 0) -> None:
        """Skinner join episode budget (tuples examined) and UCT seed."""
        self._check(self.lib.kdb_ctx_set_skinner(self.ctx, budget_per_episode, seed))

    def last_skinner_episodes(self) -> int:
        return self.lib.kdb_last_skinner_episodes(self.ctx)

    def last_skinner_batches(self) -> int:
        return int(self.lib.kdb_last_skinner_batches(self.ctx))

    def last_skinner_work(self) -> int:
        """Tuples examined by all episodes of the last Skinner join."""
        return self.lib.kdb_last_skinner_work(self.ctx)

    def set_skinner_policy(self, policy: str = "uct", prior: "JoinPriorModel" = None, log: bool = False) -> None:
        """Join-order search: "uct" (the reference's), "prior" (UCT seeded by
        a learned JoinPriorModel), "random" (random connected orders, for
        collecting training samples); `log` records (features, reward) of
        every episode step."""
        code = {"uct": 0, "prior": 1, "random": 2}[policy]
        self._check(self.lib.kdb_ctx_set_skinner_policy(self.ctx, code, prior.h if prior else None,
                                                         1 if log else 0))
        self._prior = prior

    def last_skinner_samples(self):
        """(features [n, 64] float32, rewards [n] float32) of the last Skinner
        join run with logging on."""
        n = self.lib.kdb_last_skinner_samples(self.ctx, None, None, 0)
        d = self.lib.kdb_mlp_num_features()
        x = np.zeros((n, d), np.float32)
        r = np.zeros(n, np.float32)
        if n:
            self.lib.kdb_last_skinner_samples(self.ctx, _ptr(x), _ptr(r), n)
        return x, r

    def stream_handle(self) -> int:
        return self.lib.kdb_ctx_stream(self.ctx) or 0

    def set_profiling(self, on: bool) -> None:
        self._check(self.lib.kdb_ctx_set_profiling(self.ctx, 1 if on else 0))

    def last_kernels(self):
        import json
        n = self.lib.kdb_last_query_kernels(self.ctx, None, 0)
        buf = ctypes.create_string_buffer(int(n))
        self.lib.kdb_last_query_kernels(self.ctx, buf, n)
        return json.loads(buf.value.decode())


def sort_pairs_noalloc(d_keys: int, d_vals: int, n: int, key_bits: int = 64, stream: int = 0) -> int:
    """kdb_sort_pairs_noalloc: the device sort with no device allocation
    (scratch is a static array of KDB_SORT_NOALLOC_MAX_PAIRS pairs).  Queued on
    `stream` of the current device; returns the C status code (0 = ok,
    -4 = more pairs than the static scratch holds)."""
    lib = load_library()
    return lib.kdb_sort_pairs_noalloc(ctypes.c_void_p(d_keys), ctypes.c_void_p(d_vals), n, key_bits,
                                      ctypes.c_void_p(stream) if stream else None)


class BatchQuery(ctypes.Structure):
    """kdb_batch_query: one query of the batched join + group-by template."""
    _fields_ = [("dim_table", ctypes.c_char_p), ("dim_key", ctypes.c_char_p), ("dim_date", ctypes.c_char_p),
                ("dim_seg", ctypes.c_char_p), ("fact_table", ctypes.c_char_p), ("fact_fk", ctypes.c_char_p),
                ("fact_price", ctypes.c_char_p), ("fact_disc", ctypes.c_char_p), ("date_lt", ctypes.c_int32),
                ("seg", ctypes.c_int32)]


class Batch:
    """Many join + group-by template queries run as one captured CUDA graph
    (kdb_batch_*)."""

    def __init__(self, engine: Engine, queries):
        self.engine = engine
        self.lib = engine.lib
        arr = (BatchQuery * len(queries))()
        self._keep = []
        for i, q in enumerate(queries):
            enc = {k: (v.encode() if isinstance(v, str) else v) for k, v in q.items()}
            self._keep.append(enc)
            arr[i] = BatchQuery(**enc)
        h = ctypes.c_void_p()
        engine._check(self.lib.kdb_batch_create(engine.ctx, ctypes.cast(arr, ctypes.c_void_p), len(queries),
                                                ctypes.byref(h)))
        self.h = h
        self.n = len(queries)

    def configure(self, block: int = 256, load_factor: float = 0.5, fanout: int = 1) -> None:
        self.engine._check(self.lib.kdb_batch_configure(self.h, block, load_factor, fanout))

    def tune(self, reps: int = 3):
        import json
        buf = ctypes.create_string_buffer(1 << 16)
        self.engine._check(self.lib.kdb_batch_tune(self.h, reps, buf, 1 << 16))
        return json.loads(buf.value.decode())

    def config(self):
        b, lf, f = ctypes.c_int32(), ctypes.c_double(), ctypes.c_int32()
        self.lib.kdb_batch_config(self.h, ctypes.byref(b), ctypes.byref(lf), ctypes.byref(f))
        return {"block": b.value, "load_factor": lf.value, "fanout": f.value}

    def run(self) -> None:
        self.engine._check(self.lib.kdb_batch_run(self.h))

    def run_timed(self, reps: int = 10) -> float:
        return self.lib.kdb_batch_run_timed(self.h, reps)

    def result(self, q: int):
        n = self.lib.kdb_batch_result(self.h, q, None, None, 0)
        if n < 0:
            raise KdbError(int(n), self.lib.kdb_last_error(self.engine.ctx).decode())
        keys = np.zeros(n, np.int32)
        sums = np.zeros(n, np.float64)
        self.lib.kdb_batch_result(self.h, q, _ptr(keys), _ptr(sums), n)
        return keys, sums

    def close(self):
        if self.h:
            self.lib.kdb_batch_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Request loop over an engine's resident tables (kdb_server_*): `slots`
    worker threads with their own CUDA streams run queued plans concurrently
    as slots and the device-memory budget allow."""

    def __init__(self, engine: Engine, slots: int = 4, hbm_budget_bytes: int = 8 << 30):
        self.engine = engine
        self.lib = engine.lib
        engine.register_enums()
        h = ctypes.c_void_p()
        engine._check(self.lib.kdb_server_start(engine.ctx, slots, hbm_budget_bytes, ctypes.byref(h)))
        self.h = h

    def submit(self, plan) -> int:
        text = plan.to_json() if isinstance(plan, Operator) else plan
        if isinstance(text, str):
            text = text.encode()
        self.engine.register_enums()
        t = self.lib.kdb_server_submit(self.h, text)
        if t < 0:
            raise KdbError(int(t), self.lib.kdb_last_error(self.engine.ctx).decode())
        return int(t)

    def poll(self, ticket: int, wait_ms: int = 0):
        """The ticket's Result once done, else None; raises if it failed."""
        h = ctypes.c_void_p()
        rc = self.lib.kdb_server_poll(self.h, ticket, wait_ms, ctypes.byref(h))
        if rc == 1:
            return None
        self.engine._check(rc)
        return Result.from_handle(self.lib, "kdb_", self.engine.ctx, h, owner=self.engine)

    def wait(self, ticket: int, timeout_s: float = 600.0):
        import time
        end = time.monotonic() + timeout_s
        while True:
            r = self.poll(ticket, 100)
            if r is not None:
                return r
            if time.monotonic() > end:
                raise TimeoutError(f"request {ticket} not done after {timeout_s} s")

    def stats(self):
        import json
        n = self.lib.kdb_server_stats(self.h, None, 0)
        buf = ctypes.create_string_buffer(int(n))
        self.lib.kdb_server_stats(self.h, buf, n)
        return json.loads(buf.value.decode())

    def close(self):
        if self.h:
            self.lib.kdb_server_stop(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class JoinPriorModel:
    """The learned join-order prior (kdb_mlp_*): a 64-128-128-128-1 ReLU MLP
    whose forward, backward and Adam kernels run on the engine's GPU."""

    MAX_ROWS = 4096

    def __init__(self, engine: Engine, seed: int = 0):
        self.engine = engine
        self.lib = engine.lib
        h = ctypes.c_void_p()
        engine._check(self.lib.kdb_mlp_create(engine.ctx, seed, ctypes.byref(h)))
        self.h = h
        self.num_features = int(self.lib.kdb_mlp_num_features())
        self.num_params = int(self.lib.kdb_mlp_num_params())

    def _check(self, rc):
        if rc != 0:
            raise KdbError(rc, self.lib.kdb_mlp_last_error(self.h).decode())

    def params(self) -> np.ndarray:
        p = np.zeros(self.num_params, np.float32)
        self._check(self.lib.kdb_mlp_get_params(self.h, _ptr(p), self.num_params))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        self._check(self.lib.kdb_mlp_set_params(self.h, _ptr(p), p.size))

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        out = []
        for i in range(0, len(x), self.MAX_ROWS):
            xb = np.ascontiguousarray(x[i:i + self.MAX_ROWS])
            y = np.zeros(len(xb), np.float32)
            self._check(self.lib.kdb_mlp_forward(self.h, _ptr(xb), len(xb), _ptr(y)))
            out.append(y)
        return np.concatenate(out) if out else np.zeros(0, np.float32)

    def gradient(self, x, t):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(self.num_params, np.float32)
        loss = ctypes.c_double()
        self._check(self.lib.kdb_mlp_gradient(self.h, _ptr(x), _ptr(t), len(x), _ptr(g), ctypes.byref(loss)))
        return g, loss.value

    def train_step(self, x, t, lr: float = 1e-3) -> float:
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        loss = ctypes.c_double()
        self._check(self.lib.kdb_mlp_train_step(self.h, _ptr(x), _ptr(t), len(x), lr, ctypes.byref(loss)))
        return loss.value

    def close(self):
        if self.h:
            self.lib.kdb_mlp_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
