"""The allocation-free sort entry point (kdb_sort_pairs_noalloc).

Callers that cannot allocate device memory while they sort -- host callbacks
where CUDA allocation calls are not allowed, engines that budget all HBM
through their own allocator -- use this entry
point: its scratch is a static device array, so it never calls cudaMalloc.
This test runs it through the C ABI and checks it against the allocating
entry point (kdb_sort_pairs) on the same inputs, twice in a row, so stale
contents of the shared static scratch would show.  It lives in its own file,
collected last, and works alone in a fresh process as well as after the other
tests.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KDB_ERR_CAPACITY = -4
MAX_PAIRS = 1 << 20


def _pairs(rng, n, hi):
    keys = rng.integers(0, hi, n, dtype=np.int64).astype(np.uint64)
    vals = rng.permutation(n).astype(np.uint32)
    return keys, vals


@pytest.mark.parametrize("n,bits,hi", [(MAX_PAIRS, 64, 1 << 62), (300_001, 24, 1 << 24), (1500, 64, 50)])
def test_noalloc_sort_matches_allocating_sort_twice(n, bits, hi):
    import torch
    from kushdb_b200.engine import Engine, sort_pairs_noalloc

    rng = np.random.default_rng(n)
    stream = torch.cuda.current_stream().cuda_stream
    with Engine(0) as engine:
        for call in range(2):  # two calls in a row share the static scratch
            keys, vals = _pairs(rng, n, hi)
            ka = torch.from_numpy(keys.view(np.int64)).cuda()
            va = torch.from_numpy(vals.view(np.int32)).cuda()
            kb, vb = ka.clone(), va.clone()
            torch.cuda.synchronize()
            engine.sort_pairs(ka.data_ptr(), va.data_ptr(), n, bits)
            rc = sort_pairs_noalloc(kb.data_ptr(), vb.data_ptr(), n, bits, stream)
            assert rc == 0, rc
            torch.cuda.synchronize()
            assert torch.equal(ka, kb), f"keys differ on call {call}"
            assert torch.equal(va, vb), f"values differ on call {call}"
            mask = np.uint64((1 << bits) - 1) if bits < 64 else np.uint64(0xFFFFFFFFFFFFFFFF)
            order = np.argsort(keys & mask, kind="stable")
            assert np.array_equal(vb.cpu().numpy().view(np.uint32), vals[order])


def test_noalloc_sort_rejects_more_pairs_than_its_scratch():
    import torch
    from kushdb_b200.engine import sort_pairs_noalloc

    n = MAX_PAIRS + 1
    k = torch.zeros(n, dtype=torch.int64, device="cuda")
    v = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert sort_pairs_noalloc(k.data_ptr(), v.data_ptr(), n, 64, 0) == KDB_ERR_CAPACITY
