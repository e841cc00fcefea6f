"""Learned join-order prior: the CUDA forward / backward kernels against the
numpy oracle (fp32 on the GPU vs float64: forward within 1e-4 relative,
gradients within 1e-4 of the largest gradient entry plus 1e-3 relative), a
training run that fits, results unchanged under every policy, and the
prior's gain over plain UCT on held-out multiway joins."""

import numpy as np
import pytest

from kushdb_b200 import workloads as wl
from oracle import join_prior as jp
from parity import compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from kushdb_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()


def _random_model(engine, seed=3):
    from kushdb_b200.engine import JoinPriorModel
    m = JoinPriorModel(engine, seed=seed)
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.08, m.num_params).astype(np.float32)
    m.set_params(p)
    return m, p


def test_forward_matches_oracle(engine):
    m, p = _random_model(engine)
    x = np.random.default_rng(1).normal(0, 1, (333, m.num_features)).astype(np.float32)
    y = m.forward(x)
    ref, _ = jp.forward(p, x)
    assert np.all(np.abs(y - ref) <= 1e-4 * (1 + np.abs(ref)))
    assert np.array_equal(m.params(), p)
    m.close()


@pytest.mark.parametrize("rows", [1, 16, 301, 4096])
def test_gradient_matches_oracle(engine, rows):
    m, p = _random_model(engine, seed=rows)
    rng = np.random.default_rng(rows)
    x = rng.normal(0, 1, (rows, m.num_features)).astype(np.float32)
    t = rng.normal(0, 1, rows).astype(np.float32)
    g, loss = m.gradient(x, t)
    ref, ref_loss = jp.gradient(p, x, t)
    tol = 1e-4 * np.max(np.abs(ref)) + 1e-3 * np.abs(ref)
    bad = np.nonzero(np.abs(g - ref) > tol)[0]
    assert bad.size == 0, (bad[:10], g[bad[:10]], ref[bad[:10]])
    assert abs(loss - ref_loss) <= 1e-5 * (1 + ref_loss)
    # a gradient call does not move the parameters
    assert np.array_equal(m.params(), p)
    m.close()


def test_training_fits_a_smooth_target(engine):
    from kushdb_b200.engine import JoinPriorModel
    from kushdb_b200.join_prior import train
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, (4096, 64)).astype(np.float32)
    y = (np.sin(2 * x[:, 0]) + x[:, 1] * x[:, 2] + 0.5 * np.abs(x[:, 3])).astype(np.float32)
    m = JoinPriorModel(engine, seed=1)
    losses = train(m, x, y, steps=600, batch=512, lr=2e-3)
    assert np.mean(losses[-20:]) < 0.1 * np.mean(losses[:5])
    m.close()


def _queries(seed0, count, max_rows=20_000):
    out = []
    for i in range(count):
        shape = "star" if i % 2 == 0 else "chain"
        n_tables = 5 + i % 3
        zipf = 1.5 if i % 4 >= 2 else 0.0
        tables, tokens = wl.skinner_tables(shape, n_tables, min_rows=1000, max_rows=max_rows, zipf_s=zipf,
                                           seed=seed0 + 31 * i, prefix=f"jp{seed0}_{i}_")
        out.append((tables, wl.skinner_plan(tables, tokens, shape)))
    return out


def test_policies_never_change_results(engine):
    from oracle import Oracle
    m, _ = _random_model(engine, seed=9)  # an untrained (arbitrary) prior
    for tables, plan in _queries(900, 3):
        o = Oracle()
        for t in tables:
            engine.register_table(t)
            o.register_table(t)
        ref = o.execute(plan)
        for policy in ("uct", "prior", "random"):
            engine.set_skinner_policy(policy, prior=m if policy == "prior" else None)
            engine.set_skinner(1500, seed=2)
            assert compare(engine.execute(plan), ref) == "", policy
    engine.set_skinner_policy("uct")
    engine.set_skinner()
    m.close()


def test_prior_needs_fewer_episodes_than_uct(engine):
    from kushdb_b200.join_prior import fit_prior
    budget = 1000
    train_q = _queries(100, 12)
    test_q = _queries(500, 8)
    for tables, _ in train_q + test_q:
        for t in tables:
            engine.register_table(t)
    model, info = fit_prior(engine, [p for _, p in train_q], budget, seeds=(0, 1), steps=1500)
    assert info["samples"] > 1000
    assert info["last_loss"] < info["first_loss"]
    totals = {"uct": [0, 0, 0, 0.0], "prior": [0, 0, 0, 0.0]}
    # one join order per episode batch: every decision is the policy's own
    # (with 16 orders per batch these small joins finish inside the first
    # batch whichever policy picks the orders)
    engine.set_option("KDB_SKINNER_BATCH", "1")
    for _, plan in test_q:  # compile every plan's kernels before timing
        engine.set_skinner_policy("uct")
        engine.set_skinner(budget, seed=0)
        engine.execute(plan, fetch=False)
    for _, plan in test_q:
        for seed in (0, 1, 2):
            for policy in ("uct", "prior"):
                engine.set_skinner_policy(policy, prior=model if policy == "prior" else None)
                engine.set_skinner(budget, seed=seed)
                engine.execute(plan, fetch=False)
                totals[policy][0] += engine.last_skinner_episodes()
                totals[policy][1] += engine.last_skinner_work()
                totals[policy][2] += engine.last_skinner_batches()
                totals[policy][3] += engine.last_device_ms()
    engine.set_skinner_policy("uct")
    engine.set_skinner()
    engine.set_option("KDB_SKINNER_BATCH", None)
    print("episodes / work / batches / device ms (uct, prior):", totals)
    # fewer episodes and tuples, and the gain reaches the clock: less device
    # time (the prior's values come from one forward pass per join)
    assert totals["prior"][0] < totals["uct"][0]
    assert totals["prior"][1] < totals["uct"][1]
    assert totals["prior"][3] < totals["uct"][3]
    model.close()
