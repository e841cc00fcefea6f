"""Plan operator / expression trees for the KushDB hot path, built in Python.

This module mirrors the reference's operator API so that plans read like the
reference's own tests:

* ``catalog::Type`` / ``catalog::TypeId``            (catalog/sql_type.h:7-85)
* ``plan::OperatorSchema`` and its Add*Columns        (plan/operator/operator_schema.cc:38-128)
* ``plan::ScanOperator``, ``ScanSelectOperator``, ``SelectOperator``,
  ``HashJoinOperator``, ``GroupByAggregateOperator``, ``AggregateOperator``,
  ``OrderByOperator``, ``SkinnerJoinOperator``, ``OutputOperator``
                                                       (plan/operator/*.h)
* expressions: ``ColumnRefExpression``, ``VirtualColumnRefExpression``,
  ``LiteralExpression``, ``BinaryArithmeticExpression``,
  ``UnaryArithmeticExpression``, ``AggregateExpression``, ``CaseExpression``,
  ``IntToFloatConversionExpression``, ``ExtractExpression``,
  ``EnumInExpression``, ``RegexpMatchingExpression`` (plan/expression/*.h)
* the builder DSL ``ColRef``, ``VirtColRef``, ``Literal``, ``Eq`` ... ``Count``
                                                       (util/builder.h:33-300)

A finished tree is serialised to JSON (``to_json``) and handed to either
engine through the C ABI (``kdb_query_execute``).  Type inference follows
``CalculateBinaryType`` (plan/expression/arithmetic_expression.cc:11-78) and
``CalculateAggTypeId`` (plan/expression/aggregate_expression.cc:17-53).
"""

from __future__ import annotations

import json
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Union

# ----------------------------------------------------------------------------
# catalog::Type
# ----------------------------------------------------------------------------

INT_MIN, INT_MAX = -2**31, 2**31 - 1

TYPE_IDS = ("SMALLINT", "INT", "BIGINT", "REAL", "DATE", "TEXT", "BOOLEAN", "ENUM")


@dataclass(frozen=True)
class Type:
    """catalog::Type (catalog/sql_type.h:18-85)."""

    type_id: str
    enum_id: int = 0

    def __post_init__(self):
        if self.type_id not in TYPE_IDS:
            raise ValueError(f"unknown type id {self.type_id}")

    def to_json(self) -> str:
        return f"ENUM:{self.enum_id}" if self.type_id == "ENUM" else self.type_id

    @staticmethod
    def SmallInt():
        return Type("SMALLINT")

    @staticmethod
    def Int():
        return Type("INT")

    @staticmethod
    def BigInt():
        return Type("BIGINT")

    @staticmethod
    def Real():
        return Type("REAL")

    @staticmethod
    def Date():
        return Type("DATE")

    @staticmethod
    def Text():
        return Type("TEXT")

    @staticmethod
    def Boolean():
        return Type("BOOLEAN")

    @staticmethod
    def Enum(enum_id: int):
        return Type("ENUM", enum_id)


# ----------------------------------------------------------------------------
# Dates: Julian day numbers (runtime/date.cc:10-25)
# ----------------------------------------------------------------------------


def build_date(year: int, month: int, day: int) -> int:
    """runtime::Date::BuildDate (runtime/date.cc:10-25): civil date -> JDN."""
    if month > 2:
        month += 1
        year += 4800
    else:
        month += 13
        year += 4799
    century = year // 100
    julian = year * 365 - 32167
    julian += year // 4 - century + century // 4
    julian += 7834 * month // 256 + day
    return julian


def split_date(jd: int):
    """runtime::Date::SplitDate (runtime/date.cc:29-44): JDN -> (y, m, d)."""
    julian = (jd + 32044) & 0xFFFFFFFF
    quad = julian // 146097
    extra = ((julian - quad * 146097) * 4 + 3) & 0xFFFFFFFF
    julian += 60 + quad * 3 + extra // 146097
    quad = julian // 1461
    julian -= quad * 1461
    y = julian * 4 // 1461
    julian = ((julian + 305) % 365 if y != 0 else (julian + 306) % 366) + 123
    y += quad * 4
    year = y - 4800
    quad = julian * 2141 // 65536
    day = julian - 7834 * quad // 256
    month = (quad + 10) % 12 + 1
    return year, month, day


EPOCH_JDN = build_date(1970, 1, 1)  # 2440588


# ----------------------------------------------------------------------------
# Enum dictionaries (runtime::Enum::EnumManager, runtime/enum.cc:133-182)
# ----------------------------------------------------------------------------


class EnumRegistry:
    """Process-wide id -> list-of-strings dictionaries.

    The reference resolves an enum literal's string to its integer key when the
    plan is built (plan/expression/literal_expression.cc:57-61); plans built
    here do the same through this registry.
    """

    _dicts: Dict[int, List[str]] = {}

    @classmethod
    def register(cls, enum_id: int, values: Sequence[str]) -> None:
        cls._dicts[enum_id] = list(values)

    @classmethod
    def values(cls, enum_id: int) -> List[str]:
        return cls._dicts[enum_id]

    @classmethod
    def key(cls, enum_id: int, value: str) -> int:
        try:
            return cls._dicts[enum_id].index(value)
        except (KeyError, ValueError):
            # GetValue returns -1 for unknown strings (runtime/enum.cc:165-182)
            return -1

    @classmethod
    def all(cls) -> Dict[int, List[str]]:
        return dict(cls._dicts)


# ----------------------------------------------------------------------------
# Catalog (catalog/catalog.h:14-59)
# ----------------------------------------------------------------------------


class Column:
    def __init__(self, name: str, type_: Type, path: str = "", null_path: str = "",
                 index_path: str = ""):
        self.name = name
        self.type = type_
        self.path = path
        self.null_path = null_path
        self.index_path = index_path

    def Nullable(self) -> bool:
        return bool(self.null_path)

    def GetType(self) -> Type:
        return self.type

    def Name(self) -> str:
        return self.name


class Table:
    def __init__(self, name: str):
        self.name = name
        self._cols: Dict[str, Column] = {}
        self._order: List[str] = []

    def Insert(self, name: str, type_: Type, path: str = "", null_path: str = "",
               index_path: str = "") -> Column:
        col = Column(name, type_, path, null_path, index_path)
        self._cols[name] = col
        self._order.append(name)
        return col

    def __getitem__(self, name: str) -> Column:
        return self._cols[name]

    def Columns(self) -> List[Column]:
        return [self._cols[n] for n in self._order]

    def Name(self) -> str:
        return self.name


class Database:
    def __init__(self):
        self._tables: Dict[str, Table] = {}

    def Insert(self, name: str) -> Table:
        t = Table(name)
        self._tables[name] = t
        return t

    def __getitem__(self, name: str) -> Table:
        return self._tables[name]

    def __contains__(self, name: str) -> bool:
        return name in self._tables

    def tables(self) -> List[Table]:
        return list(self._tables.values())


# ----------------------------------------------------------------------------
# Expressions (plan/expression/*)
# ----------------------------------------------------------------------------


class Expression:
    def __init__(self, type_: Type, nullable: bool):
        self.type = type_
        self.nullable = nullable

    def Type(self) -> Type:
        return self.type

    def Nullable(self) -> bool:
        return self.nullable

    def to_dict(self) -> dict:  # pragma: no cover - abstract
        raise NotImplementedError


class ColumnRefExpression(Expression):
    """plan/expression/column_ref_expression.h: (child_idx, column_idx)."""

    def __init__(self, type_: Type, nullable: bool, child_idx: int, column_idx: int):
        super().__init__(type_, nullable)
        self.child_idx = child_idx
        self.column_idx = column_idx

    def to_dict(self):
        return {"e": "colref", "type": self.type.to_json(), "nullable": self.nullable,
                "child": self.child_idx, "idx": self.column_idx}


class VirtualColumnRefExpression(Expression):
    def __init__(self, type_: Type, nullable: bool, column_idx: int):
        super().__init__(type_, nullable)
        self.column_idx = column_idx

    def to_dict(self):
        return {"e": "vcolref", "type": self.type.to_json(), "nullable": self.nullable,
                "idx": self.column_idx}


class LiteralExpression(Expression):
    """plan/expression/literal_expression.h:15-49."""

    def __init__(self, type_: Type, value, null: bool = False):
        super().__init__(type_, null)
        self.value = value
        self.null = null

    def to_dict(self):
        v = self.value
        if self.type.type_id == "REAL":
            v = float(v)
        elif self.type.type_id == "BOOLEAN":
            v = bool(v)
        elif self.type.type_id == "TEXT":
            v = str(v)
        else:
            v = int(v)
        return {"e": "lit", "type": self.type.to_json(), "null": self.null, "v": v}


BINARY_OPS = ("ADD", "SUB", "MUL", "DIV", "EQ", "NEQ", "LT", "LEQ", "GT", "GEQ",
              "AND", "OR", "STARTS_WITH", "ENDS_WITH", "CONTAINS")
_BOOL_RESULT = {"AND", "OR", "EQ", "NEQ", "LT", "LEQ", "GT", "GEQ", "STARTS_WITH",
                "ENDS_WITH", "CONTAINS"}


def _binary_type(op: str, left: Type, right: Type) -> Type:
    """CalculateBinaryType (plan/expression/arithmetic_expression.cc:11-78)."""
    if left.type_id == "ENUM":
        if op in ("EQ", "NEQ"):
            if left != right:
                raise TypeError("Require same type arguments")
            return Type.Boolean()
        if op in ("LT", "LEQ", "GT", "GEQ", "STARTS_WITH", "ENDS_WITH", "CONTAINS"):
            if right.type_id != "TEXT" and left != right:
                raise TypeError("Require same type arguments")
            return Type.Boolean()
        raise TypeError("Invalid expr type")
    if right.type_id == "ENUM":
        raise TypeError("not supported yet")
    if left != right:
        raise TypeError(f"Require same type arguments ({left} vs {right})")
    if op in _BOOL_RESULT:
        return Type.Boolean()
    return left


class BinaryArithmeticExpression(Expression):
    def __init__(self, op: str, left: Expression, right: Expression):
        if op not in BINARY_OPS:
            raise ValueError(op)
        super().__init__(_binary_type(op, left.type, right.type),
                         left.nullable or right.nullable)
        self.op = op
        self.left = left
        self.right = right

    def to_dict(self):
        return {"e": "bin", "op": self.op, "type": self.type.to_json(),
                "nullable": self.nullable, "l": self.left.to_dict(),
                "r": self.right.to_dict()}


class UnaryArithmeticExpression(Expression):
    """NOT / IS_NULL (plan/expression/arithmetic_expression.cc:109-153)."""

    def __init__(self, op: str, child: Expression):
        if op == "NOT":
            if child.type.type_id != "BOOLEAN":
                raise TypeError("Not boolean child")
            nullable = child.nullable
        elif op == "IS_NULL":
            nullable = False
        else:
            raise ValueError(op)
        super().__init__(Type.Boolean(), nullable)
        self.op = op
        self.child = child

    def to_dict(self):
        return {"e": "un", "op": self.op, "type": "BOOLEAN", "nullable": self.nullable,
                "c": self.child.to_dict()}


AGG_TYPES = ("SUM", "MIN", "MAX", "AVG", "COUNT")


def _agg_type(agg: str, child: Type) -> Type:
    """CalculateAggTypeId (plan/expression/aggregate_expression.cc:17-53)."""
    t = child.type_id
    if agg == "SUM":
        if t in ("INT", "SMALLINT", "BIGINT", "REAL"):
            return child
        raise TypeError("Invalid input type for sum aggregate")
    if agg == "AVG":
        if t in ("INT", "SMALLINT", "BIGINT", "REAL"):
            return Type.Real()
        raise TypeError("Invalid input type for avg aggregate")
    if agg == "COUNT":
        return Type.BigInt()
    if t in ("INT", "SMALLINT", "BIGINT", "REAL", "DATE", "TEXT", "ENUM"):
        return child
    raise TypeError("Invalid input type for max/min aggregate")


class AggregateExpression(Expression):
    def __init__(self, agg: str, child: Expression):
        if agg not in AGG_TYPES:
            raise ValueError(agg)
        super().__init__(_agg_type(agg, child.type), agg != "COUNT")
        self.agg = agg
        self.child = child

    def AggType(self) -> str:
        return self.agg

    def to_dict(self):
        return {"e": "agg", "agg": self.agg, "type": self.type.to_json(),
                "nullable": self.nullable, "c": self.child.to_dict()}


class CaseExpression(Expression):
    def __init__(self, cond: Expression, then: Expression, otherwise: Expression):
        if then.type != otherwise.type:
            raise TypeError("case branches must have the same type")
        super().__init__(then.type, then.nullable or otherwise.nullable)
        self.cond, self.then, self.otherwise = cond, then, otherwise

    def to_dict(self):
        return {"e": "case", "type": self.type.to_json(), "nullable": self.nullable,
                "c": self.cond.to_dict(), "t": self.then.to_dict(),
                "f": self.otherwise.to_dict()}


class IntToFloatConversionExpression(Expression):
    def __init__(self, child: Expression):
        super().__init__(Type.Real(), child.nullable)
        self.child = child

    def to_dict(self):
        return {"e": "i2f", "type": "REAL", "nullable": self.nullable,
                "c": self.child.to_dict()}


class ExtractExpression(Expression):
    def __init__(self, child: Expression, what: str = "YEAR"):
        if child.type.type_id != "DATE":
            raise TypeError("extract requires a DATE")
        super().__init__(Type.Int(), child.nullable)
        self.child = child
        self.what = what

    def to_dict(self):
        return {"e": "extract", "what": self.what, "type": "INT",
                "nullable": self.nullable, "c": self.child.to_dict()}


class EnumInExpression(Expression):
    def __init__(self, child: Expression, values: Sequence[int]):
        if child.type.type_id != "ENUM":
            raise TypeError("enum IN requires an ENUM child")
        super().__init__(Type.Boolean(), False)
        self.child = child
        self.values = [int(v) for v in values]

    def to_dict(self):
        return {"e": "enum_in", "type": "BOOLEAN", "nullable": False,
                "c": self.child.to_dict(), "values": self.values}


class RegexpMatchingExpression(Expression):
    """SQL LIKE as the planner hands it over: an RE2 full-match pattern
    ``^...$`` (plan/expression/arithmetic_expression.h:69-83; the pattern
    text is ``RE2::pattern()``).  Only the planner's LIKE translation is
    accepted: escaped bytes, ``.`` (any byte but newline) and ``.*``.
    Never NULL; a NULL child is false (expression_translator.cc:277-297)."""

    def __init__(self, child: Expression, regex: str):
        if child.type.type_id not in ("TEXT", "ENUM"):
            raise TypeError("Invalid child type for LIKE. Expected text/enum.")
        super().__init__(Type.Boolean(), False)
        self.child = child
        self.regex = regex

    def to_dict(self):
        return {"e": "regex", "type": "BOOLEAN", "nullable": False,
                "c": self.child.to_dict(), "pattern": self.regex}


# ----------------------------------------------------------------------------
# OperatorSchema (plan/operator/operator_schema.cc)
# ----------------------------------------------------------------------------


class SchemaColumn:
    def __init__(self, name: str, expr: Expression):
        self.name = name
        self.expr = expr

    def Name(self):
        return self.name

    def Expr(self):
        return self.expr


class OperatorSchema:
    def __init__(self):
        self.columns: List[SchemaColumn] = []
        self._idx: Dict[str, int] = {}
        self.generated_from: Optional[Table] = None

    def Columns(self) -> List[SchemaColumn]:
        return self.columns

    def GetColumnIndex(self, name: str) -> int:
        if name not in self._idx:
            raise KeyError(f"Unknown column {name}")
        return self._idx[name]

    def AddDerivedColumn(self, name: str, expr: Expression) -> None:
        self._idx[name] = len(self.columns)
        self.columns.append(SchemaColumn(name, expr))

    def AddGeneratedColumns(self, table: Table, columns: Optional[Sequence[str]] = None):
        """operator_schema.cc:43-67: columns of a base table, refs (0, position)."""
        self.generated_from = table
        cols = table.Columns() if columns is None else [table[c] for c in columns]
        for c in cols:
            idx = len(self.columns)
            self._idx[c.name] = idx
            self.columns.append(SchemaColumn(
                c.name, ColumnRefExpression(c.type, c.Nullable(), 0, idx)))

    def AddPassthroughColumns(self, op: "Operator", columns: Optional[Union[Sequence[str], int]] = None,
                              child_idx: int = 0):
        """operator_schema.cc:69-95."""
        if isinstance(columns, int):
            child_idx, columns = columns, None
        schema = op.Schema()
        names = [c.name for c in schema.columns] if columns is None else list(columns)
        for name in names:
            idx = schema.GetColumnIndex(name)
            col = schema.columns[idx]
            self.AddDerivedColumn(name, ColumnRefExpression(
                col.expr.type, col.expr.nullable, child_idx, idx))

    def AddVirtualPassthroughColumns(self, schema: "OperatorSchema",
                                     columns: Optional[Sequence[str]] = None):
        """operator_schema.cc:97-120."""
        names = [c.name for c in schema.columns] if columns is None else list(columns)
        for name in names:
            idx = schema.GetColumnIndex(name)
            col = schema.columns[idx]
            self.AddDerivedColumn(name, VirtualColumnRefExpression(
                col.expr.type, col.expr.nullable, idx))

    def AddPassthroughColumn(self, op: "Operator", base_name: str, derived_name: str,
                             child_idx: int = 0):
        schema = op.Schema()
        idx = schema.GetColumnIndex(base_name)
        col = schema.columns[idx]
        self.AddDerivedColumn(derived_name, ColumnRefExpression(
            col.expr.type, col.expr.nullable, child_idx, idx))

    def to_list(self) -> list:
        return [{"name": c.name, "expr": c.expr.to_dict()} for c in self.columns]


# ----------------------------------------------------------------------------
# Operators (plan/operator/*)
# ----------------------------------------------------------------------------


class Operator:
    def __init__(self, schema: OperatorSchema, children: Sequence["Operator"] = ()):
        self.schema = schema
        self.children = list(children)

    def Schema(self) -> OperatorSchema:
        return self.schema

    def Children(self):
        return self.children

    def Child(self):
        return self.children[0]

    def to_dict(self) -> dict:  # pragma: no cover - abstract
        raise NotImplementedError

    def to_json(self) -> str:
        return json.dumps(self.to_dict(), separators=(",", ":"))


def _scan_columns(schema: OperatorSchema, relation: Table) -> list:
    out = []
    for c in schema.columns:
        cat = relation[c.name]
        out.append({"name": c.name, "type": cat.type.to_json(), "nullable": cat.Nullable()})
    return out


class ScanOperator(Operator):
    """plan/operator/scan_operator.h: every schema column is a catalog column."""

    def __init__(self, schema: OperatorSchema, relation: Table):
        super().__init__(schema)
        self.relation = relation

    def to_dict(self):
        return {"op": "SCAN", "relation": self.relation.name,
                "columns": _scan_columns(self.schema, self.relation),
                "output": self.schema.to_list()}


class ScanSelectOperator(Operator):
    """plan/operator/scan_select_operator.h:14-38."""

    def __init__(self, schema: OperatorSchema, scan_schema: OperatorSchema, relation: Table,
                 filters: Sequence[Expression]):
        super().__init__(schema)
        self.scan_schema = scan_schema
        self.relation = relation
        self.filters = list(filters)

    def ScanSchema(self):
        return self.scan_schema

    def to_dict(self):
        return {"op": "SCAN_SELECT", "relation": self.relation.name,
                "columns": _scan_columns(self.scan_schema, self.relation),
                "output": self.schema.to_list(),
                "filters": [f.to_dict() for f in self.filters]}


class SimdScanSelectOperator(ScanSelectOperator):
    """plan/operator/simd_scan_select_operator.h: same semantics as
    ScanSelect (the reference only changes how the CPU evaluates it)."""

    def to_dict(self):
        d = super().to_dict()
        d["op"] = "SIMD_SCAN_SELECT"
        return d


class SelectOperator(Operator):
    def __init__(self, schema: OperatorSchema, child: Operator, cond: Expression):
        super().__init__(schema, [child])
        self.cond = cond

    def to_dict(self):
        return {"op": "SELECT", "child": self.Child().to_dict(),
                "cond": self.cond.to_dict(), "output": self.schema.to_list()}


class HashJoinOperator(Operator):
    """plan/operator/hash_join_operator.h:12-34 (left child = build side)."""

    def __init__(self, schema: OperatorSchema, left: Operator, right: Operator,
                 left_keys: Sequence[ColumnRefExpression],
                 right_keys: Sequence[ColumnRefExpression]):
        super().__init__(schema, [left, right])
        self.left_keys = list(left_keys)
        self.right_keys = list(right_keys)

    def to_dict(self):
        return {"op": "HASH_JOIN", "left": self.children[0].to_dict(),
                "right": self.children[1].to_dict(),
                "left_keys": [k.to_dict() for k in self.left_keys],
                "right_keys": [k.to_dict() for k in self.right_keys],
                "output": self.schema.to_list()}


class CrossProductOperator(Operator):
    """plan/operator/cross_product_operator.h: left x right (two children),
    every right row paired with every left row."""

    def __init__(self, schema: OperatorSchema, children: Sequence[Operator]):
        if len(children) != 2:
            raise ValueError("CrossProduct takes two children")
        super().__init__(schema, list(children))

    def to_dict(self):
        return {"op": "CROSS_PRODUCT", "left": self.children[0].to_dict(),
                "right": self.children[1].to_dict(), "output": self.schema.to_list()}


class GroupByAggregateOperator(Operator):
    def __init__(self, schema: OperatorSchema, child: Operator,
                 group_by: Sequence[Expression], aggs: Sequence[AggregateExpression]):
        super().__init__(schema, [child])
        self.group_by = list(group_by)
        self.aggs = list(aggs)

    def to_dict(self):
        return {"op": "GROUP_BY_AGGREGATE", "child": self.Child().to_dict(),
                "group_by": [g.to_dict() for g in self.group_by],
                "aggs": [a.to_dict() for a in self.aggs],
                "output": self.schema.to_list()}


class AggregateOperator(Operator):
    def __init__(self, schema: OperatorSchema, child: Operator,
                 aggs: Sequence[AggregateExpression]):
        super().__init__(schema, [child])
        self.aggs = list(aggs)

    def to_dict(self):
        return {"op": "AGGREGATE", "child": self.Child().to_dict(),
                "aggs": [a.to_dict() for a in self.aggs],
                "output": self.schema.to_list()}


class OrderByOperator(Operator):
    def __init__(self, schema: OperatorSchema, child: Operator,
                 keys: Sequence[ColumnRefExpression], ascending: Sequence[bool]):
        super().__init__(schema, [child])
        self.keys = list(keys)
        self.ascending = [bool(a) for a in ascending]

    def to_dict(self):
        return {"op": "ORDER_BY", "child": self.Child().to_dict(),
                "keys": [k.to_dict() for k in self.keys], "asc": self.ascending,
                "output": self.schema.to_list()}


class SkinnerJoinOperator(Operator):
    """plan/operator/skinner_join_operator.h:12-33."""

    def __init__(self, schema: OperatorSchema, children: Sequence[Operator],
                 conditions: Sequence[Expression], prefix_order: Sequence[int] = ()):
        super().__init__(schema, children)
        self.conditions = list(conditions)
        self.prefix_order = list(prefix_order)

    def to_dict(self):
        return {"op": "SKINNER_JOIN", "children": [c.to_dict() for c in self.children],
                "conditions": [c.to_dict() for c in self.conditions],
                "prefix_order": self.prefix_order, "output": self.schema.to_list()}


class OutputOperator(Operator):
    def __init__(self, child: Operator):
        super().__init__(child.Schema(), [child])

    def to_dict(self):
        return {"op": "OUTPUT", "child": self.Child().to_dict()}


# ----------------------------------------------------------------------------
# util/builder.h
# ----------------------------------------------------------------------------


def ColRef(op: Operator, col: str, child_idx: int = 0) -> ColumnRefExpression:
    idx = op.Schema().GetColumnIndex(col)
    e = op.Schema().columns[idx].expr
    return ColumnRefExpression(e.type, e.nullable, child_idx, idx)


ColRefE = ColRef


def VirtColRef(expr_or_schema, idx_or_name) -> VirtualColumnRefExpression:
    if isinstance(expr_or_schema, OperatorSchema):
        idx = expr_or_schema.GetColumnIndex(idx_or_name)
        e = expr_or_schema.columns[idx].expr
        return VirtualColumnRefExpression(e.type, e.nullable, idx)
    e = expr_or_schema
    return VirtualColumnRefExpression(e.type, e.nullable, int(idx_or_name))


def Exp(e):
    return e


def Literal(*args) -> LiteralExpression:
    """Literal(v) / Literal(y, m, d) / Literal(enum_id, "str") (util/builder.h:74-90)."""
    if len(args) == 3:
        return LiteralExpression(Type.Date(), build_date(*args))
    if len(args) == 2:
        enum_id, s = args
        return LiteralExpression(Type.Enum(enum_id), EnumRegistry.key(enum_id, s))
    (v,) = args
    if isinstance(v, bool):
        return LiteralExpression(Type.Boolean(), v)
    if isinstance(v, int):
        return LiteralExpression(Type.Int(), v)
    if isinstance(v, float):
        return LiteralExpression(Type.Real(), v)
    if isinstance(v, str):
        return LiteralExpression(Type.Text(), v)
    raise TypeError(type(v))


def SmallIntLiteral(v: int):
    return LiteralExpression(Type.SmallInt(), v)


def BigIntLiteral(v: int):
    return LiteralExpression(Type.BigInt(), v)


def NullLiteral(t: Type):
    return LiteralExpression(t, 0, null=True)


def _enum_rewrite(op, e1, e2):
    # Eq / Neq against a TEXT literal on an ENUM column become an enum literal
    # (util/builder.h:92-135).
    if e1.type.type_id == "ENUM" and isinstance(e2, LiteralExpression) and e2.type.type_id == "TEXT":
        e2 = LiteralExpression(Type.Enum(e1.type.enum_id), EnumRegistry.key(e1.type.enum_id, e2.value))
    return BinaryArithmeticExpression(op, e1, e2)


def Eq(e1, e2):
    return _enum_rewrite("EQ", e1, e2)


def Neq(e1, e2):
    return _enum_rewrite("NEQ", e1, e2)


def Lt(e1, e2):
    return BinaryArithmeticExpression("LT", e1, e2)


def Leq(e1, e2):
    return BinaryArithmeticExpression("LEQ", e1, e2)


def Gt(e1, e2):
    return BinaryArithmeticExpression("GT", e1, e2)


def Geq(e1, e2):
    return BinaryArithmeticExpression("GEQ", e1, e2)


def StartsWith(e1, e2):
    return BinaryArithmeticExpression("STARTS_WITH", e1, e2)


def EndsWith(e1, e2):
    return BinaryArithmeticExpression("ENDS_WITH", e1, e2)


def Contains(e1, e2):
    return BinaryArithmeticExpression("CONTAINS", e1, e2)


_REGEX_SPECIAL = set(".+*?^$()[]{}|\\")


def LikeRegex(pattern: str) -> str:
    """The planner's LIKE -> RE2 translation (plan/planner.cc:283-318):
    ``_`` -> ``.``, ``%`` -> ``.*``, regex metacharacters escaped, anchored
    with ``^...$``."""
    out = ["^"]
    for c in pattern:
        if c in _REGEX_SPECIAL:
            out.append("\\" + c)
        elif c == "_":
            out.append(".")
        elif c == "%":
            out.append(".*")
        else:
            out.append(c)
    out.append("$")
    return "".join(out)


def Like(e, pattern: str):
    """``e LIKE pattern`` in its general (regex) form."""
    return RegexpMatchingExpression(e, LikeRegex(pattern))


def And(exprs: Sequence[Expression]):
    """Left-deep AND chain (util/builder.h And)."""
    out = BinaryArithmeticExpression("AND", exprs[0], exprs[1])
    for e in exprs[2:]:
        out = BinaryArithmeticExpression("AND", out, e)
    return out


def Or(exprs: Sequence[Expression]):
    out = BinaryArithmeticExpression("OR", exprs[0], exprs[1])
    for e in exprs[2:]:
        out = BinaryArithmeticExpression("OR", out, e)
    return out


def Add(e1, e2):
    return BinaryArithmeticExpression("ADD", e1, e2)


def Sub(e1, e2):
    return BinaryArithmeticExpression("SUB", e1, e2)


def Mul(e1, e2):
    return BinaryArithmeticExpression("MUL", e1, e2)


def Div(e1, e2):
    return BinaryArithmeticExpression("DIV", e1, e2)


def Not(e):
    return UnaryArithmeticExpression("NOT", e)


def IsNull(e):
    return UnaryArithmeticExpression("IS_NULL", e)


def Sum(e):
    return AggregateExpression("SUM", e)


def Avg(e):
    return AggregateExpression("AVG", e)


def Max(e):
    return AggregateExpression("MAX", e)


def Min(e):
    return AggregateExpression("MIN", e)


def Count(e: Optional[Expression] = None):
    """Count() counts rows via Literal(true) (util/builder.h:282-291)."""
    return AggregateExpression("COUNT", Literal(True) if e is None else e)


def Float(e):
    return IntToFloatConversionExpression(e)


def Case(cond, then, otherwise):
    return CaseExpression(cond, then, otherwise)


def Extract(e, what="YEAR"):
    return ExtractExpression(e, what)


def In(e, values: Sequence[Union[int, str]]):
    ids = [EnumRegistry.key(e.type.enum_id, v) if isinstance(v, str) else int(v) for v in values]
    return EnumInExpression(e, ids)


def MakeVector(*xs):
    return list(xs)
