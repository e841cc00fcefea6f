"""Host-side column data: the tables a query scans, before they go to HBM.

``HostColumn`` holds one ``runtime::ColumnData`` column
(runtime/column_data.h:20-57) as numpy arrays: fixed-width values in the
type's physical width (int8 BOOLEAN, int16 SMALLINT, int32 INT/DATE/ENUM,
int64 BIGINT, f64 REAL), TEXT as int64 offsets + bytes, and optional int8
NULL flags (the reference keeps those in a separate BOOLEAN ``_null.kdb``).
"""

from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from .plan import Database, EnumRegistry, Type

NP_DTYPE = {"SMALLINT": np.int16, "INT": np.int32, "BIGINT": np.int64, "REAL": np.float64,
            "DATE": np.int32, "BOOLEAN": np.int8, "ENUM": np.int32}


def parse_type(s: str) -> Type:
    if s.startswith("ENUM:"):
        return Type.Enum(int(s[5:]))
    return Type(s)


@dataclass
class HostColumn:
    name: str
    type: Type
    values: Optional[np.ndarray] = None      # fixed-width
    offsets: Optional[np.ndarray] = None     # TEXT: int64[n+1]
    chars: Optional[np.ndarray] = None       # TEXT: uint8 bytes
    nulls: Optional[np.ndarray] = None       # int8[n], 1 = NULL

    def __len__(self):
        if self.type.type_id == "TEXT":
            return len(self.offsets) - 1
        return len(self.values)

    @property
    def nullable(self) -> bool:
        return self.nulls is not None

    @staticmethod
    def from_strings(name: str, strings: Sequence[str], nulls=None) -> "HostColumn":
        enc = [s.encode() for s in strings]
        off = np.zeros(len(enc) + 1, dtype=np.int64)
        off[1:] = np.cumsum([len(b) for b in enc])
        chars = np.frombuffer(b"".join(enc), dtype=np.uint8) if enc else np.zeros(0, np.uint8)
        return HostColumn(name, Type.Text(), offsets=off, chars=chars,
                          nulls=None if nulls is None else np.asarray(nulls, np.int8))

    def strings(self) -> List[str]:
        b = self.chars.tobytes()
        return [b[self.offsets[i]:self.offsets[i + 1]].decode() for i in range(len(self))]


@dataclass
class HostTable:
    name: str
    columns: Dict[str, HostColumn] = field(default_factory=dict)

    def add(self, col: HostColumn) -> "HostTable":
        self.columns[col.name] = col
        return self

    @property
    def rows(self) -> int:
        return len(next(iter(self.columns.values()))) if self.columns else 0

    def nbytes(self) -> int:
        n = 0
        for c in self.columns.values():
            if c.values is not None:
                n += c.values.nbytes
            if c.offsets is not None:
                n += c.offsets.nbytes + c.chars.nbytes
            if c.nulls is not None:
                n += c.nulls.nbytes
        return n


def catalog_of(tables: Sequence[HostTable]) -> Database:
    """A catalog::Database describing host tables (paths left empty)."""
    db = Database()
    for t in tables:
        ct = db.Insert(t.name)
        for c in t.columns.values():
            ct.Insert(c.name, c.type, null_path="null" if c.nullable else "")
    return db


# ---------------------------------------------------------------------------
# Reference file formats
# ---------------------------------------------------------------------------


def read_kdb(path: str, type_: Type, null_path: str = "") -> HostColumn:
    """Read a reference ``.kdb`` column file (runtime/column_data.cc:121-229)."""
    name = os.path.basename(path)
    if type_.type_id == "TEXT":
        raw = np.fromfile(path, dtype=np.uint8)
        card = int(raw[:4].view(np.int32)[0])
        slots = raw[8:8 + 16 * card].view(np.dtype([("len", "<i4"), ("pad", "<i4"), ("off", "<u8")]))
        lens = slots["len"].astype(np.int64)
        offs = slots["off"].astype(np.int64)
        off = np.zeros(card + 1, np.int64)
        off[1:] = np.cumsum(lens)
        chars = np.concatenate([raw[o:o + n] for o, n in zip(offs, lens)]) if card else np.zeros(0, np.uint8)
        col = HostColumn(name, type_, offsets=off, chars=chars)
    else:
        col = HostColumn(name, type_, values=np.fromfile(path, dtype=NP_DTYPE[type_.type_id]))
    if null_path:
        col.nulls = np.fromfile(null_path, dtype=np.int8)
    return col


def load_golden(golden_dir: str) -> Dict[str, HostTable]:
    """Load the committed golden fixtures (tests/golden/) and register enums."""
    with open(os.path.join(golden_dir, "schema.json")) as f:
        schema = json.load(f)
    with open(os.path.join(golden_dir, "enums.json")) as f:
        for k, v in json.load(f).items():
            EnumRegistry.register(int(k), v)
    tables = {}
    for tname, cols in schema.items():
        z = np.load(os.path.join(golden_dir, "tables", tname + ".npz"))
        t = HostTable(tname)
        for c in cols:
            typ = parse_type(c["type"])
            nulls = z[c["name"] + "__null"] if c["nullable"] else None
            if typ.type_id == "TEXT":
                t.add(HostColumn(c["name"], typ, offsets=z[c["name"] + "__off"],
                                 chars=z[c["name"] + "__chars"], nulls=nulls))
            else:
                t.add(HostColumn(c["name"], typ, values=z[c["name"]], nulls=nulls))
        tables[tname] = t
    return tables
