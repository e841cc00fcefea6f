"""Device sort entry point (kdb_sort_pairs): stable radix sort of (key,
value) pairs, checked against numpy's stable argsort."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from kushdb_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("n,bits,hi", [(1, 64, 10), (7, 64, 3), (2048, 64, 1 << 40), (2049, 64, 100),
                                       (5000, 64, 1 << 63), (40_000, 64, 1 << 40), (100_000, 64, 1 << 62),
                                       (300_000, 20, 1 << 20), (1 << 20, 64, 7)])
def test_sort_pairs_matches_stable_argsort(engine, n, bits, hi):
    import torch
    rng = np.random.default_rng(n + bits)
    keys = rng.integers(0, hi, n, dtype=np.int64).astype(np.uint64)
    vals = np.arange(n, dtype=np.uint32)
    dk = torch.from_numpy(keys.view(np.int64)).cuda()
    dv = torch.from_numpy(vals.view(np.int32)).cuda()
    torch.cuda.synchronize()
    engine.sort_pairs(dk.data_ptr(), dv.data_ptr(), n, bits)
    got_k = dk.cpu().numpy().view(np.uint64)
    got_v = dv.cpu().numpy().view(np.uint32)
    mask = np.uint64((1 << bits) - 1) if bits < 64 else np.uint64(0xFFFFFFFFFFFFFFFF)
    order = np.argsort(keys & mask, kind="stable")
    assert np.array_equal(got_v, vals[order])
    assert np.array_equal(got_k, keys[order])
