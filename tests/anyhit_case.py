"""Shared cases of the candidate-group any-hit tests.

A case is a small scene run through the reference scene tool (compiled
unchanged, oracle/ref_tool.cpp): its own object ids, unique edges, candidate
lists in emission order and random-policy scores.  The expected per-group
outcome comes from the C restatement (oracle_group_anyhit) with the proposal
lists ordered by (score desc, index asc).
"""
from __future__ import annotations

import numpy as np

from p2cccd_b200 import records, scenes

CFG = dict(eps_time=1e-6, eps_space=1e-6, max_depth=32)


def two_spheres_small(seed: int = 20261203) -> dict:
    return scenes.two_spheres(n_lon=24, n_rings=16, seed=seed)


def cloth_small(seed: int = 20261203) -> dict:
    return scenes.cloth_on_sphere(n=17, sphere_lon=24, sphere_rings=16, seed=seed, gap=1e-3, drop=0.05)


def sphere_cluster(k: int = 7, seed: int = 5) -> dict:
    """k small spheres (radius 0.2-0.35) in a unit box, each translating by
    up to 0.6 with vertex jitter: many object pairs, some of them meeting."""
    rng = np.random.default_rng(seed)
    objs = []
    for i in range(k):
        v, f = scenes.uv_sphere(8 + i % 3, 5 + i % 2, radius=float(rng.uniform(0.2, 0.35)))
        c = rng.uniform(-0.6, 0.6, 3)
        d = rng.normal(0.0, 0.3, 3)
        v0 = v + c + rng.normal(0, 1e-3, v.shape)
        v1 = v + c + d + rng.normal(0, 1e-3, v.shape)
        objs.append((v0, v1, f, scenes.unique_edges(f)))
    return scenes.combine(objs)


def primitives(s: dict, edges: np.ndarray, cands: np.ndarray, kind: str) -> np.ndarray:
    """Reference primitive records of candidate pairs (ids = scene indices)."""
    v0, v1 = s["v_t0"], s["v_t1"]
    a, b = cands[:, 0].astype(np.int64), cands[:, 1].astype(np.int64)
    if kind == "vf":
        idx = np.stack([a, s["faces"][b, 0], s["faces"][b, 1], s["faces"][b, 2]], 1)
        fam = records.FAMILY_POINT_TRIANGLE
    else:
        idx = np.stack([edges[a, 0], edges[a, 1], edges[b, 0], edges[b, 1]], 1).astype(np.int64)
        fam = records.FAMILY_EDGE_EDGE
    return records.pack_primitives(v0[idx], v1[idx], a, b, idx, family=fam)


def hits(oracle_mod, s, edges, cands, kind) -> np.ndarray:
    """Conservative decision of every candidate: certificate is not a separation."""
    if len(cands) == 0:
        return np.zeros(0, dtype=np.uint8)
    res, st, _ = oracle_mod.eval_batch(primitives(s, edges, cands, kind), 0.0, 1.0, CFG["eps_time"],
                                       CFG["eps_space"], CFG["max_depth"])
    return ((res["status"] != records.STATUS_SEPARATION) | (st != 0)).astype(np.uint8)


def groups_of(tool, cands: np.ndarray, kind: str) -> np.ndarray:
    if kind == "vf":
        oa, ob = tool.v_obj[cands[:, 0]], tool.f_obj[cands[:, 1]]
    else:
        oa, ob = tool.e_obj[cands[:, 0]], tool.e_obj[cands[:, 1]]
    lo, hi = np.minimum(oa, ob), np.maximum(oa, ob)
    return (lo * tool.n_obj + hi).astype(np.int32)


def top_lists(groups: np.ndarray, scores: np.ndarray, n_groups: int, top_k: int):
    """Per group the top_k candidate indices by (score desc, index asc), CSR."""
    order = np.lexsort((np.arange(len(groups)), -scores, groups))
    offs = np.zeros(n_groups + 1, dtype=np.int64)
    idx = []
    sorted_groups = groups[order]
    for g in range(n_groups):
        members = order[sorted_groups == g][:top_k]
        idx.append(members)
        offs[g + 1] = offs[g] + len(members)
    return offs, (np.concatenate(idx) if idx else np.zeros(0, dtype=np.int64)).astype(np.int64)


def expected(oracle_mod, groups, hit, scores, n_groups, top_k) -> dict:
    """Oracle per-group outcome plus the tool row's aggregate fields."""
    offs, tidx = top_lists(groups, scores, n_groups, top_k)
    det, pc, fc, ev = oracle_mod.group_anyhit(groups, hit, n_groups, offs, tidx)
    present = np.bincount(groups, minlength=n_groups) > 0 if len(groups) else np.zeros(n_groups, bool)
    prop_hit = np.zeros(n_groups, dtype=bool)
    for g in range(n_groups):
        if pc[g] > 0:
            prop_hit[g] = bool(hit[tidx[offs[g] + pc[g] - 1]])
    return {
        "detected": det, "proposal_calls": pc, "fallback_calls": fc, "evaluated": ev,
        "row": {
            "exact_calls": int(pc.sum() + fc.sum()),
            "proposal_exact_calls": int(pc.sum()),
            "fallback_exact_calls": int(fc.sum()),
            "hit_count": int(det.sum()),
            "group_count": int(present.sum()),
            "fallback_groups": int((present & ~prop_hit).sum()),
            "positive_first_hit_rank_sum": int((pc + fc)[det.astype(bool)].sum()),
        },
    }


def tool_case(oracle_mod, s: dict, kind: str, thickness: float = 0.0, exclude_self: bool = False):
    """(tool scene, candidates, scores, groups, hits) for one family."""
    tool = oracle_mod.RefToolScene(s["v_t0"], s["v_t1"], s["faces"], thickness, exclude_self)
    cands = tool.candidates(kind)
    scores = tool.random_scores(kind, len(cands))
    groups = groups_of(tool, cands, kind)
    hit = hits(oracle_mod, s, tool.edges, cands, kind)
    return tool, cands, scores, groups, hit
