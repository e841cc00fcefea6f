"""Oracle restatements against the reference's unit tests and runtime.

* runtime/date_test.cc: BuildDate / SplitDate known answers;
* runtime::Vector::Sort tie order (runtime/vector.cc:45-110), checked against
  the reference's own sort compiled from source when oracle/_ref is built.
"""

import ctypes
import os

import numpy as np
import pytest

from kushdb_b200.plan import EPOCH_JDN, build_date, split_date
import oracle


def test_date_known_answers():
    # 1970-01-01 is JDN 2440588; round trips over a wide range of dates
    assert EPOCH_JDN == 2440588
    assert build_date(2000, 1, 1) == 2451545
    for jd in range(2415021, 2488070, 97):
        y, m, d = split_date(jd)
        assert build_date(y, m, d) == jd


@pytest.mark.skipif(not os.path.exists(oracle.REF_LIB_PATH), reason="reference runtime not built")
def test_dates_match_reference_runtime():
    ref = ctypes.CDLL(oracle.REF_LIB_PATH)
    y, m, d = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    for (yy, mm, dd) in [(1992, 1, 2), (1998, 12, 1), (1995, 3, 30), (2021, 1, 29), (1200, 12, 31)]:
        assert ref.kdbref_build_date(yy, mm, dd) == build_date(yy, mm, dd)
    for jd in range(2400000, 2500000, 331):
        ref.kdbref_split_date(jd, ctypes.byref(y), ctypes.byref(m), ctypes.byref(d))
        assert (y.value, m.value, d.value) == split_date(jd)


def _merge_sort_restated(pairs):
    # the oracle's merge (oracle.cc MergeSort): take left only if left < right
    def rec(v):
        if len(v) <= 1:
            return v
        m = (len(v) - 1) // 2 + 1
        a, b = rec(v[:m]), rec(v[m:])
        out, i, j = [], 0, 0
        while i < len(a) and j < len(b):
            if a[i][0] < b[j][0]:
                out.append(a[i]); i += 1
            else:
                out.append(b[j]); j += 1
        return out + a[i:] + b[j:]
    return rec(list(pairs))


@pytest.mark.skipif(not os.path.exists(oracle.REF_LIB_PATH), reason="reference runtime not built")
@pytest.mark.parametrize("n", [1, 2, 7, 64, 1000])
def test_sort_tie_order_matches_reference(n):
    ref = ctypes.CDLL(oracle.REF_LIB_PATH)
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 5, n).astype(np.int32)
    pairs = np.stack([keys, np.arange(n, dtype=np.int32)], 1).copy()
    ref.kdbref_sort_pairs(pairs.ctypes.data_as(ctypes.c_void_p), n)
    want = _merge_sort_restated([(int(k), i) for i, k in enumerate(keys)])
    assert [tuple(p) for p in pairs.tolist()] == [tuple(p) for p in want]
