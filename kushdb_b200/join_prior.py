"""Training of the learned join-order prior for the Skinner join.

Samples come from the engine itself: Skinner joins run with the "random"
policy (uniformly random connected join orders) and logging on record, for
every step of every episode, the features of (join-order prefix, next
table) and the episode's reward (0.5 * progress + 0.5 * results / budget,
the reward of runtime/skinner_join_executor.cc:252-274).  The model
regresses the reward; at query time UCT starts every action at the model's
prediction and lets observed rewards overrule it.  Forward, backward and the
Adam step run in the library's own CUDA kernels (kdb_mlp_*).
"""

from __future__ import annotations

from typing import Iterable, List, Tuple

import numpy as np

from .engine import Engine, JoinPriorModel


def collect_samples(engine: Engine, plans: Iterable, budget: int, seeds: Iterable[int] = (0, 1, 2)
                    ) -> Tuple[np.ndarray, np.ndarray]:
    """Runs every plan once per seed with random join orders and returns the
    logged (features, rewards)."""
    xs: List[np.ndarray] = []
    ys: List[np.ndarray] = []
    try:
        engine.set_skinner_policy("random", log=True)
        for plan in plans:
            for seed in seeds:
                engine.set_skinner(budget, seed)
                engine.execute(plan, fetch=False)
                x, r = engine.last_skinner_samples()
                xs.append(x)
                ys.append(r)
    finally:
        engine.set_skinner_policy("uct")
        engine.set_skinner()
    if not xs:
        return np.zeros((0, 64), np.float32), np.zeros(0, np.float32)
    return np.concatenate(xs), np.concatenate(ys)


def train(model: JoinPriorModel, x: np.ndarray, y: np.ndarray, steps: int = 2000, batch: int = 512,
          lr: float = 1e-3, seed: int = 0) -> List[float]:
    """Adam on minibatches drawn with replacement; returns the loss per step."""
    rng = np.random.default_rng(seed)
    n = len(y)
    losses = []
    for _ in range(steps):
        idx = rng.integers(0, n, min(batch, n))
        losses.append(model.train_step(x[idx], y[idx], lr))
    return losses


def fit_prior(engine: Engine, plans: Iterable, budget: int, seeds: Iterable[int] = (0, 1, 2),
              steps: int = 2000, model_seed: int = 0) -> Tuple[JoinPriorModel, dict]:
    """Collects samples on `plans` and trains a fresh model on them."""
    x, y = collect_samples(engine, plans, budget, seeds)
    model = JoinPriorModel(engine, seed=model_seed)
    losses = train(model, x, y, steps=steps)
    return model, {"samples": int(len(y)), "first_loss": losses[0] if losses else None,
                   "last_loss": float(np.mean(losses[-50:])) if losses else None}
