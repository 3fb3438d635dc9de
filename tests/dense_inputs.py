"""Seeded candidate-group rows (the arrays the dense group early-stop
binding reads) with uneven groups, ties, collisions and extreme values."""
from __future__ import annotations

import numpy as np


def make_rows(n: int, seed: int, *, n_groups: int | None = None, ties: bool = True, zero_cost: float = 0.05,
              big_group: int = 0) -> dict:
    rng = np.random.default_rng(seed)
    g = n_groups or max(1, n // 6)
    q = rng.integers(1, 4 * g + 1, n).astype(np.uint64)
    if big_group:
        q[:big_group] = 7
    rng.shuffle(q)
    trace = np.zeros((n, 8))
    trace[:, 0] = (rng.random(n) < 0.3).astype(np.float64)
    trace[:, 5] = rng.gamma(2.0, 3.0, n)
    trace[rng.random(n) < zero_cost, 5] = 0.0  # PositiveCost replaces it with 1
    trace[rng.random(n) < 0.02, 5] = -2.5
    c0 = rng.random(n)
    trace[:, 6] = c0
    trace[:, 7] = np.minimum(1.0, c0 + rng.random(n) * 0.2)
    scores = rng.normal(0.0, 1.0, (n, 8)).astype(np.float32)
    if ties:
        scores[::7, 3] = scores[::7, 1]
        scores[::11] = 0.0
    prio = rng.normal(0.0, 1.0, n).astype(np.float32)
    cost = rng.random(n).astype(np.float32)
    if ties:
        prio[::5] = 0.5
        prio[1::9] = -0.0
        prio[2::9] = 0.0
        cost[::4] = 0.25
    cost_target = rng.random(n).astype(np.float32)
    cost_target[::13] = 0.0
    cost_target[1::17] = np.float32(1e-20)  # narrow cost floored at 1e-12
    cost_target[2::19] = np.nan
    unc = rng.random(n).astype(np.float32)
    return {"query_id": q, "candidate_id": np.arange(1, n + 1, dtype=np.uint64), "cost_target": cost_target,
            "oracle_trace": trace, "interval_scores": scores, "priority_score": prio, "cost_score": cost,
            "uncertainty_score": unc}
