"""General LIKE (RegexpMatchingExpression): the planner's LIKE -> RE2
translation (plan/planner.cc:283-321) and the oracle's full-match evaluation
(expression_translator.cc:277-297, RE2::FullMatch) against Python's
``re.fullmatch`` of the same pattern ('.' excludes '\\n' in both), on TEXT
with NULLs, on an ENUM, with escaped metacharacters, newlines and empty
strings; and the patterns the backend rejects."""

import re

import numpy as np
import pytest

from kushdb_b200.data import HostColumn, HostTable, catalog_of
from kushdb_b200.plan import (ColRef, EnumRegistry, Like, LikeRegex, OperatorSchema, OutputOperator,
                              RegexpMatchingExpression, ScanOperator, SelectOperator, Type)

ALPHABET = list("ab.c%_(\n") + ["xy"]
PATTERNS = ["%", "", "a%", "%a", "%a%b%", "a_b", "_", "%.%", "%(%", "a%%b", "%\n%", "_%_", "%%_%%c",
            "ab.c", "%xy%xy%", "%_(_%"]


def _strings(rng, n):
    out = []
    for _ in range(n):
        k = int(rng.integers(0, 7))
        out.append("".join(ALPHABET[int(i)] for i in rng.integers(0, len(ALPHABET), k)))
    return out


def _plan(t, pattern, col="s"):
    rel = catalog_of([t])[t.name]
    ss = OperatorSchema()
    ss.AddGeneratedColumns(rel, [col])
    scan = ScanOperator(ss, rel)
    out = OperatorSchema()
    out.AddPassthroughColumns(scan, [col])
    return OutputOperator(SelectOperator(out, scan, Like(ColRef(scan, col), pattern)))


def test_like_regex_matches_the_planner_translation():
    assert LikeRegex("%BRASS") == "^.*BRASS$"
    assert LikeRegex("a_b%") == "^a.b.*$"
    assert LikeRegex("1+1=2?") == "^1\\+1=2\\?$"
    assert LikeRegex("[x](y){z}|$^.*\\") == "^\\[x\\]\\(y\\)\\{z\\}\\|\\$\\^\\.\\*\\\\$"


@pytest.mark.parametrize("pattern", PATTERNS)
def test_oracle_like_matches_python_re(pattern):
    from oracle import Oracle
    rng = np.random.default_rng(len(pattern) * 7 + 1)
    n = 3000
    strings = _strings(rng, n)
    nulls = (rng.random(n) < 0.1).astype(np.int8)
    t = HostTable("like_t")
    t.add(HostColumn.from_strings("s", strings, nulls=nulls))
    o = Oracle()
    o.register_table(t)
    got = sorted(o.execute(_plan(t, pattern).to_json()).columns[0].values)
    rx = re.compile(LikeRegex(pattern))
    want = sorted(s for s, z in zip(strings, nulls) if not z and rx.fullmatch(s))
    assert got == want
    o.close()


def test_oracle_like_on_enum():
    from oracle import Oracle
    EnumRegistry.register(77, ["RED WINE", "white wine", "ROSE", "red\nwine", ""])
    t = HostTable("like_enum")
    keys = np.array([0, 1, 2, 3, 4, 0, 2], np.int32)
    t.add(HostColumn("c", Type.Enum(77), values=keys))
    o = Oracle()
    o.register_table(t)
    # rows: RED WINE, white wine, ROSE, red\nwine, "", RED WINE, ROSE; "%" is
    # ".*", which stops at the newline
    for pattern, want in [("%WINE", 2), ("%wine%", 1), ("r%", 0), ("red_wine", 0), ("%", 6), ("", 1),
                          ("%ROSE%", 2), ("R__ WINE", 2)]:
        assert o.execute(_plan(t, pattern, "c").to_json()).num_rows == want, pattern
    o.close()


@pytest.mark.parametrize("regex", ["^a+$", "abc", "^a|b$", "^[ab]$", "^a\\", "^(a)$"])
def test_non_like_regex_is_rejected(regex):
    from kushdb_b200.engine import Engine, KdbError
    t = HostTable("like_rej")
    t.add(HostColumn.from_strings("s", ["a"]))
    rel = catalog_of([t])[t.name]
    ss = OperatorSchema()
    ss.AddGeneratedColumns(rel, ["s"])
    scan = ScanOperator(ss, rel)
    out = OperatorSchema()
    out.AddPassthroughColumns(scan, ["s"])
    plan = OutputOperator(SelectOperator(out, scan, RegexpMatchingExpression(ColRef(scan, "s"), regex)))
    e = Engine(-1)
    e.register_table(t)
    with pytest.raises(KdbError):
        e.execute(plan)
    e.close()


def test_like_pattern_compiles_in_the_backend():
    from kushdb_b200.engine import Engine
    t = HostTable("like_dry")
    t.add(HostColumn.from_strings("s", ["a", "b"], nulls=np.array([0, 1], np.int8)))
    e = Engine(-1)
    e.register_table(t)
    for pattern in PATTERNS + ["_" * 63]:
        e.execute(_plan(t, pattern))
    e.close()
