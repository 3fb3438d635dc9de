"""A seeded exact work queue for the audit-row tests: work items with random
ids, sub-intervals, depths, priorities and family masks over plain-workload
primitives (CSR lists, only of each item's requested families), one item
holding a primitive with a NaN coordinate (an invalid-input certificate)."""
from __future__ import annotations

import numpy as np


def make_queue(n_items: int = 120, seed: int = 5):
    from p2cccd_b200 import workloads
    from p2cccd_b200.records import AUDIT_ITEM_DTYPE

    w = workloads.plain_queries(workloads.PlainSpec(n_vf=6 * n_items, n_ee=6 * n_items, seed=seed))
    g = np.random.default_rng(seed)
    mask = g.integers(1, 4, n_items)
    # an item lists only primitives of its requested families (the device queue's contract)
    k_pt = np.where(mask & 1, g.integers(0, 7, n_items), 0)
    k_ee = np.where(mask & 2, g.integers(0, 7, n_items), 0)
    pt_off = np.concatenate([[0], np.cumsum(k_pt)]).astype(np.int64)
    ee_off = np.concatenate([[0], np.cumsum(k_ee)]).astype(np.int64)
    pts = w["vf"][:pt_off[-1]].copy()
    ees = w["ee"][:ee_off[-1]].copy()
    bad = int(np.argmax(k_pt > 0))
    name = pts.dtype.names[2]
    pts[pt_off[bad]][name]["position_t1"][1] = np.nan
    items = np.zeros(n_items, AUDIT_ITEM_DTYPE)
    t0 = g.uniform(0.0, 0.5, n_items)
    items["query_id"] = g.integers(1, 9, n_items)
    items["candidate_id"] = g.integers(1, 1000, n_items)
    items["work_item_id"] = np.arange(1, n_items + 1) * 3
    items["interval_t0"] = t0
    items["interval_t1"] = t0 + g.uniform(0.05, 0.5, n_items)
    items["priority_score"] = g.normal(0, 2, n_items).astype(np.float32)
    items["feature_family_mask"] = mask
    items["depth"] = g.integers(0, 6, n_items)
    return items, pts, pt_off, ees, ee_off
