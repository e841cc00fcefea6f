"""The KushDB-side plan serialiser (include/kdb_plan_json.h) against the
plan JSON of kushdb_b200/plan.py: the header is compiled with g++ against
the class subset in tests/kushplan/plan_subset.h (laid out under the
reference's include paths), the program builds the benchmark plans with the
C++ plan classes, and every JSON it prints must equal, as parsed JSON, the
one plan.py writes for the same plan.  The C++ output then parses in the
backend (compile-only context: every pipeline is generated and compiled)."""

import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from kushdb_b200 import workloads as wl
from kushdb_b200.data import HostColumn, HostTable, catalog_of
from kushdb_b200.plan import (CaseExpression, ColRef, EnumInExpression, ExtractExpression, Float, Gt, Like,
                              IntToFloatConversionExpression, Literal, OperatorSchema, OutputOperator, Or,
                              ScanOperator, SelectOperator, Type, UnaryArithmeticExpression)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KP = os.path.join(ROOT, "tests", "kushplan")

HEADERS = [
    "catalog/catalog.h", "catalog/sql_type.h", "runtime/date.h",
    "plan/expression/aggregate_expression.h", "plan/expression/arithmetic_expression.h",
    "plan/expression/case_expression.h", "plan/expression/column_ref_expression.h",
    "plan/expression/conversion_expression.h", "plan/expression/enum_in_expression.h",
    "plan/expression/expression_visitor.h", "plan/expression/extract_expression.h",
    "plan/expression/literal_expression.h", "plan/expression/virtual_column_ref_expression.h",
    "plan/operator/aggregate_operator.h", "plan/operator/cross_product_operator.h",
    "plan/operator/group_by_aggregate_operator.h", "plan/operator/hash_join_operator.h",
    "plan/operator/operator_visitor.h", "plan/operator/order_by_operator.h", "plan/operator/output_operator.h",
    "plan/operator/scan_operator.h", "plan/operator/scan_select_operator.h", "plan/operator/select_operator.h",
    "plan/operator/simd_scan_select_operator.h", "plan/operator/skinner_join_operator.h",
]


@pytest.fixture(scope="module")
def cpp_plans(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    inc = tmp_path_factory.mktemp("kushinc")
    for h in HEADERS:  # the reference's include paths, each forwarding to the subset
        p = inc / h
        p.parent.mkdir(parents=True, exist_ok=True)
        p.write_text(f'#include "{os.path.join(KP, "plan_subset.h")}"\n')
    exe = inc / "plan_json"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", str(inc), "-I",
                           os.path.join(ROOT, "include"), "-o", str(exe), os.path.join(KP, "plan_json_main.cc")])
    out = subprocess.check_output([str(exe)], text=True).strip().split("\n")
    assert len(out) == 5
    return out


def _tables():
    wl.register_enums()
    one = lambda t: np.zeros(1, t)  # noqa: E731
    sk = []
    for i in range(3):
        t = HostTable(f"sk{i}")
        t.add(HostColumn("pk", Type.Int(), values=one(np.int32)))
        t.add(HostColumn.from_strings("note", ["x"]))
        if i == 0:
            t.add(HostColumn("fk1", Type.Int(), values=one(np.int32)))
            t.add(HostColumn("fk2", Type.Int(), values=one(np.int32)))
        sk.append(t)
    misc = HostTable("misc")
    misc.add(HostColumn("d", Type.Date(), values=one(np.int32), nulls=one(np.int8)))
    misc.add(HostColumn("c", Type.Enum(wl.SEG_ENUM_ID), values=one(np.int32)))
    misc.add(HostColumn("v", Type.Real(), values=one(np.float64)))
    misc.add(HostColumn("n", Type.Int(), values=one(np.int32), nulls=one(np.int8)))
    return sk, misc


def _misc_plan(misc):
    rel = catalog_of([misc])["misc"]
    ss = OperatorSchema()
    ss.AddGeneratedColumns(rel, ["d", "c", "v", "n"])
    scan = ScanOperator(ss, rel)
    cond = Or([EnumInExpression(ColRef(scan, "c"), [0, 2]),
               UnaryArithmeticExpression("NOT", UnaryArithmeticExpression("IS_NULL", ColRef(scan, "n")))])
    out = OperatorSchema()
    out.AddDerivedColumn("y", ExtractExpression(ColRef(scan, "d")))
    out.AddDerivedColumn("w", CaseExpression(Gt(ColRef(scan, "v"), Literal(0.5)),
                                             IntToFloatConversionExpression(ColRef(scan, "n")), Literal(-1.25)))
    out.AddDerivedColumn("m", Like(ColRef(scan, "c"), "%(B)%_N%"))
    return OutputOperator(SelectOperator(out, scan, cond))


def test_cpp_serialiser_matches_python_plans(cpp_plans):
    sk, misc = _tables()
    py = [wl.scan_agg_plan(wl.scan_agg_table(rows=1)),
          wl.group_by_plan(wl.group_by_table(rows=1)),
          wl.join_plan(*wl.join_tables(build_rows=1, probe_rows=1)),
          wl.skinner_plan(sk, ["abc", "XYZ", "q!r"], "star"),
          _misc_plan(misc)]
    for i, (c, p) in enumerate(zip(cpp_plans, py)):
        assert json.loads(c) == json.loads(p.to_json()), f"plan {i}"


def test_cpp_serialised_plans_compile_in_the_backend(cpp_plans):
    from kushdb_b200.engine import Engine
    sk, misc = _tables()
    e = Engine(-1)
    for t in [wl.scan_agg_table(rows=100), wl.group_by_table(rows=100),
              *wl.join_tables(build_rows=100, probe_rows=100), *sk, misc]:
        e.register_table(t)
    for text in cpp_plans:
        e.execute(text)
    e.close()
