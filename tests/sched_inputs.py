"""Seeded inputs for the proposal-scheduling tests: the candidates of a proxy
scene, their runtime feature rows, and proposal outputs covering every branch
(missing, invalid, out-of-distribution, high uncertainty, family scores on
both sides of the threshold, tied priorities including -0.0 and +0.0)."""
from __future__ import annotations

import numpy as np


def make_inputs(seed: int = 3, n_objects: int = 5, patches: int = 30):
    import oracle
    from p2cccd_b200 import scenes
    from p2cccd_b200.records import PROPOSAL_OUTPUT_DTYPE

    sc = scenes.proxy_scene(n_objects=n_objects, patches_per_object=patches, n_slabs=3, seed=seed, duplicates=0.3)
    raw, cand = oracle.proxy_candidates(sc)
    rows = oracle.runtime_feature_rows(cand, int(sc["n"]), len(raw), len(cand), {7: 1})
    g = np.random.default_rng(seed)
    n = len(cand)
    outs = np.zeros(n, PROPOSAL_OUTPUT_DTYPE)
    outs["candidate_id"] = cand["candidate_id"]
    outs["interval_scores"] = g.uniform(0, 1, (n, 8))
    outs["family_scores"] = g.choice([0.2, 0.5, 0.7], (n, 8))
    outs["priority_score"] = g.choice([0.0, -0.0, 0.25, 0.5, 1.0, 3.0, -1.0], n)
    outs["cost_score"] = g.uniform(0, 2, n)
    outs["uncertainty_score"] = g.choice([0.1, 0.5, 0.95, 0.99], n, p=[0.5, 0.3, 0.1, 0.1])
    k = g.permutation(n)
    outs["cost_score"][k[:3]] = -1.0                     # invalid: negative cost
    outs["interval_scores"][k[3:5], 2] = np.nan           # invalid: non-finite score
    rows["features"][k[5:8], 10] = 2.0e5                  # out of distribution
    keep = np.ones(n, bool)
    keep[k[8:14]] = False                                 # missing proposals
    return cand, rows, outs[keep], outs
