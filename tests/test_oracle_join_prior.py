"""The join-order prior's CPU oracle (numpy MLP) against central finite
differences, so that it can be trusted as the checker of the CUDA
backward kernel."""

import numpy as np

from oracle import join_prior as jp


def _loss(p, x, t):
    return float(np.mean((jp.forward(p, x)[0] - t) ** 2))


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.1, jp.num_params())
    x = rng.normal(0, 1, (7, jp.N_IN))
    t = rng.normal(0, 1, 7)
    g, loss = jp.gradient(p, x, t)
    assert abs(loss - _loss(p, x, t)) < 1e-12
    # a few entries of every parameter block
    idx = [0, 77, 8191, 8192 + 3, 8320 + 5000, 24704 + 9, 24832 + 16000, 41216 + 100, 41344 + 50, 41472]
    for i in idx:
        e = np.zeros_like(p)
        e[i] = 1e-6
        fd = (_loss(p + e, x, t) - _loss(p - e, x, t)) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, g[i], fd)


def test_layout_size():
    assert jp.num_params() == 41473
