"""A result's printer lines are formatted with the engine's enum
dictionaries: after the engine is closed they raise a clear error instead of
reading a freed context, and the columns stay readable (compile-only engine,
no GPU)."""

import pytest

from kushdb_b200 import workloads as wl


def test_lines_after_close_raise_columns_stay_readable():
    from kushdb_b200.engine import Engine
    t = wl.group_by_table(rows=1000, name="lifetime_rows")
    e = Engine(-1)
    e.register_table(t)
    r = e.execute(wl.group_by_plan(t))
    assert isinstance(e.execute(wl.group_by_plan(t)).lines, list)
    e.close()
    assert len(r.columns) > 0
    with pytest.raises(RuntimeError, match="before closing the engine"):
        r.lines
