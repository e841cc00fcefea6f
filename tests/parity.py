"""Result comparison helpers for the parity tests.

Integer, date, enum, boolean and text columns must match exactly; float64
aggregates within a relative tolerance (the GPU sums in a different order
than the reference's sequential loop; both accumulate in FP64).
"""

import math

import numpy as np

REL_TOL = 1e-12


def _close(a: float, b: float, rel: float) -> bool:
    if a == b:
        return True
    if math.isnan(a) or math.isnan(b):
        return math.isnan(a) and math.isnan(b)
    return abs(a - b) <= rel * max(abs(a), abs(b), 1e-300)


def _rows(res):
    out = []
    for r in range(res.num_rows):
        out.append(tuple(res.row(r)))
    return out


def _sort_key(row, types):
    k = []
    for v, t in zip(row, types):
        if v is None:
            k.append((0, ""))
        elif t.type_id == "REAL":
            k.append((1, f"{v:.9e}"))
        else:
            k.append((1, str(v)))
    return k


def compare(gpu, ref, ordered: bool = True, rel: float = REL_TOL) -> str:
    """'' when equal within tolerance, else a description of the first
    difference."""
    if len(gpu.columns) != len(ref.columns):
        return f"column count {len(gpu.columns)} vs {len(ref.columns)}"
    types = [c.type for c in ref.columns]
    for i, (a, b) in enumerate(zip(gpu.columns, ref.columns)):
        if a.type != b.type:
            return f"column {i} type {a.type} vs {b.type}"
    if gpu.num_rows != ref.num_rows:
        return f"row count {gpu.num_rows} vs {ref.num_rows}"
    g, o = _rows(gpu), _rows(ref)
    if not ordered:
        g = sorted(g, key=lambda r: _sort_key(r, types))
        o = sorted(o, key=lambda r: _sort_key(r, types))
    for r, (x, y) in enumerate(zip(g, o)):
        for c, (a, b, t) in enumerate(zip(x, y, types)):
            if (a is None) != (b is None):
                return f"row {r} col {c}: {a!r} vs {b!r} (NULL mismatch)"
            if a is None:
                continue
            if t.type_id == "REAL":
                if not _close(float(a), float(b), rel):
                    return f"row {r} col {c}: {a!r} vs {b!r} (rel diff {abs(a-b)/max(abs(b),1e-300):.3e})"
            elif a != b:
                return f"row {r} col {c}: {a!r} vs {b!r}"
    return ""


def max_rel_diff(gpu, ref) -> float:
    worst = 0.0
    for a, b in zip(gpu.columns, ref.columns):
        if a.type.type_id != "REAL":
            continue
        av, bv = np.asarray(a.values, np.float64), np.asarray(b.values, np.float64)
        m = np.maximum(np.abs(bv), 1e-300)
        if len(av):
            worst = max(worst, float(np.max(np.abs(av - bv) / m)))
    return worst
