"""Seeded external query batches (vertex-face and edge-edge queries with
four vertices at t0 and t1) for the batched candidate tests."""
from __future__ import annotations

import numpy as np


def make_batch(n: int, seed: int, *, miss: float = 0.3, zero_id: bool = True, box_pairs: bool = True,
               touching: bool = False, ids: str = "sparse") -> dict:
    """``miss`` of the queries have their right features moved away so that
    no candidate forms; one query has source id 0 and the id its index + 1
    would take is used by an earlier query (the runtime id is bumped);
    ``touching`` puts some right boxes exactly on the left box's face."""
    from p2cccd_b200.external import batch_arrays

    rng = np.random.default_rng(seed)
    fam = rng.integers(0, 2, n).astype(np.uint8)
    base = rng.normal(0.0, 3.0, (n, 1, 3))
    v0 = base + rng.normal(0.0, 0.5, (n, 4, 3))
    v1 = v0 + rng.normal(0.0, 0.3, (n, 4, 3))
    far = rng.random(n) < miss
    shift = np.where(far, 50.0 + rng.random(n) * 10.0, 0.0)
    for side in (1, 2):  # move the right features (vertex 1.. for VF, 2.. for EE) along y
        sel = far & ((fam == 0) | (side == 2))
        for i in range(side, 4):
            v0[sel, i, 1] += shift[sel]
            v1[sel, i, 1] += shift[sel]
    if touching:
        t = np.nonzero(~far)[0][::5]
        for k in t:  # right box's min y onto the left box's max y
            lo = [0] if fam[k] == 0 else [0, 1]
            ri = [1, 2, 3] if fam[k] == 0 else [2, 3]
            top = max(v0[k, lo, 1].max(), v1[k, lo, 1].max())
            bot = min(v0[k, ri, 1].min(), v1[k, ri, 1].min())
            v0[k, ri, 1] += top - bot
            v1[k, ri, 1] += top - bot
        v0[t[:3], 0, 2] = -0.0
    if ids == "sparse":
        qid = rng.choice(np.arange(n + 10, 11 * n + 10), n, replace=False).astype(np.uint64)  # above n + 2
    else:
        qid = np.arange(1, n + 1, dtype=np.uint64)
    if zero_id and n >= 4:
        z = n // 2
        qid[z] = 0
        if ids == "sparse":
            qid[1] = z + 1  # taken before the zero-id query asks for it
            qid[2] = z + 2  # the bump lands on an id in use again
    sidx = rng.permutation(n).astype(np.uint32)
    gt = rng.integers(-1, 2, n).astype(np.int8)
    pairs = rng.integers(1, 40, (n, 2)).astype(np.uint32)
    has = (rng.random(n) < 0.5).astype(np.uint8) if box_pairs else np.zeros(n, np.uint8)
    return batch_arrays(qid, sidx, fam, v0, v1, gt, pairs, has)
