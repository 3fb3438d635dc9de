"""Candidates for a batch of independent primitive queries (one proxy scene).

The reference packs N external vertex-face / edge-edge queries into ONE
proxy scene and generates their candidates in one broad-phase pass
(rt_candidate/external_batch_candidate.cpp:125-339):

* query k gets time slab k = [2k, 2k+1] (kBatchSlabStride 2.0) and two swept
  AABB proxies: object 1 / patch 2k+1 bounds its left features (the vertex
  of a VF query, the first edge of an EE query) over t0 and t1, object 2 /
  patch 2k+2 its right features (:62-98, :166-220);
* the queries are tiled along x: query k is shifted by ``x_cursor - min_x``,
  and the cursor advances by the query's x extent plus 1e-2 (kBatchXMargin),
  in query order (:162-166, :220);
* each proxy's motion bound is the conservative radius half its largest
  extent (:102-119);
* every candidate is translated back to its query: query id = the runtime id
  (the source id, or index + 1 when the source id is 0, bumped past ids in
  use, :154-159), objects = the query's box pair (default 1, 2), patch a = 0
  (VF) or 1 (EE), patch b = source index + 1, both proxies swept AABBs; the
  list is ordered by (query id, patch a, patch b) and candidate k gets id
  ``runtime_id * 1000003 + k + 1`` (:255-303).

Here the encoding is a few vectorised host passes over the query arrays (the
x cursor is a left-to-right ``np.add.accumulate``, the same additions in the
same order as the reference's running sum, so every bound is bit-identical),
the broad phase is the device proxy path (``ProxyCandidates``: sort, sweep,
pair sort, compaction), and the translation is a gather over the compact
records.
"""
from __future__ import annotations

import time

import numpy as np

from p2cccd_b200.records import CANDIDATE_RECORD_DTYPE

BATCH_SCENE_QUERY_ID = 1  # kBatchedSceneQueryId
BATCH_SLAB_STRIDE = 2.0  # kBatchSlabStride
BATCH_X_MARGIN = 1.0e-2  # kBatchXMargin
CANDIDATE_ID_STRIDE = 1_000_003  # kCandidateIdStride

_LHS = {0: (0,), 1: (0, 1)}  # LhsFeatureIndices (:62-67): VF vertex 0, EE edge (0, 1)
_RHS = {0: (1, 2, 3), 1: (2, 3)}  # RhsFeatureIndices (:69-74)


class ExternalBatchError(ValueError):
    pass


def batch_arrays(query_id, source_query_index, family, vertices_t0, vertices_t1, ground_truth=None,
                 box_pair=None, has_box=None) -> dict:
    """A batch as column arrays: ``family`` 0 = vf, 1 = ee; ``ground_truth``
    -1 unknown / 0 / 1; ``box_pair`` (n, 2) object ids, used where
    ``has_box`` is set (all rows when ``box_pair`` is given without it)."""
    n = len(query_id)
    gt = np.full(n, -1, np.int8) if ground_truth is None else np.asarray(ground_truth, np.int8)
    if box_pair is None:
        has, pairs = np.zeros(n, np.uint8), np.zeros((n, 2), np.uint32)
    else:
        pairs = np.asarray(box_pair, np.uint32).reshape(n, 2)
        has = np.ones(n, np.uint8) if has_box is None else np.asarray(has_box, np.uint8)
    return {"query_id": np.asarray(query_id, np.uint64), "source_query_index": np.asarray(source_query_index, np.uint32),
            "family": np.asarray(family, np.uint8), "vertices_t0": np.asarray(vertices_t0, np.float64).reshape(n, 4, 3),
            "vertices_t1": np.asarray(vertices_t1, np.float64).reshape(n, 4, 3), "ground_truth": gt,
            "has_box": has, "box_pair": pairs}


def _first_error(b: dict) -> None:
    """ValidateExternalBatchQuery (:48-60) and the source id uniqueness check
    (:150-152), applied in query order: the first failing query decides, and
    within one query t0 before t1 before uniqueness."""
    v0 = b["vertices_t0"].reshape(len(b["query_id"]), 12)
    v1 = b["vertices_t1"].reshape(len(b["query_id"]), 12)
    bad0 = ~np.isfinite(v0).all(1)
    bad1 = ~np.isfinite(v1).all(1)
    _, first = np.unique(b["query_id"], return_index=True)
    dup = np.ones(len(b["query_id"]), bool)
    dup[first] = False
    bad = bad0 | bad1 | dup
    if not bad.any():
        return
    k = int(np.argmax(bad))
    if bad0[k]:
        raise ExternalBatchError("external batch query vertices_t0 must be finite")
    if bad1[k]:
        raise ExternalBatchError("external batch query vertices_t1 must be finite")
    raise ExternalBatchError("external batch source_query_id values must be unique")


def runtime_query_ids(source_ids: np.ndarray) -> np.ndarray:
    """Runtime query ids (:154-159): the source id, or index + 1 for a source
    id of 0, then bumped while an earlier query already took it.  With unique
    source ids at most one query has id 0, so a bump can only start there; a
    collision-free tentative assignment is therefore final, and otherwise the
    reference's sequential walk runs."""
    src = np.asarray(source_ids, np.uint64)
    tentative = np.where(src > 0, src, np.arange(1, len(src) + 1, dtype=np.uint64))
    if len(np.unique(tentative)) == len(tentative):
        return tentative
    used, out = set(), np.empty(len(src), np.uint64)
    for k, t in enumerate(tentative.tolist()):
        while t in used:
            t = (t + 1) & 0xFFFFFFFFFFFFFFFF
        used.add(t)
        out[k] = t
    return out


def _feature_bounds(v0: np.ndarray, v1: np.ndarray, family: np.ndarray, side: dict) -> np.ndarray:
    """AabbFromFeatureIndices (:76-91): min / max over the listed vertices,
    t0 then t1 point of each, folded in that order from +-inf with the
    comparisons of std::min / std::max (the first of equal values stays)."""
    n = len(family)
    lo = np.full((n, 3), np.inf)
    hi = np.full((n, 3), -np.inf)
    for fam, idx in side.items():
        rows = np.nonzero(family == fam)[0]
        if len(rows) == 0:
            continue
        l, h = lo[rows], hi[rows]
        for i in idx:
            for p in (v0[rows, i], v1[rows, i]):
                l = np.where(p < l, p, l)
                h = np.where(h < p, p, h)
        lo[rows], hi[rows] = l, h
    return np.concatenate([lo, hi], 1)


def encode_scene(b: dict) -> dict:
    """BuildBatchedProxyScene (:125-227) as the proxy column arrays the device
    proxy path reads: proxies 2k (left) and 2k+1 (right) for query k."""
    n = len(b["query_id"])
    fam = b["family"]
    v0, v1 = b["vertices_t0"], b["vertices_t1"]
    lhs = _feature_bounds(v0, v1, fam, _LHS)
    rhs = _feature_bounds(v0, v1, fam, _RHS)
    qmin = np.where(rhs[:, 0] < lhs[:, 0], rhs[:, 0], lhs[:, 0])  # std::min(lhs, rhs)
    qmax = np.where(lhs[:, 3] < rhs[:, 3], rhs[:, 3], lhs[:, 3])  # std::max(lhs, rhs)
    step = (qmax - qmin) + BATCH_X_MARGIN
    cursor = np.zeros(n)
    if n > 1:
        cursor[1:] = np.add.accumulate(step[:-1])  # x_cursor += ..., left to right
    off = cursor - qmin
    bounds = np.empty((2 * n, 6))
    bounds[0::2], bounds[1::2] = lhs, rhs
    bounds[:, 0] += np.repeat(off, 2)  # TranslateAabbX (:93-98)
    bounds[:, 3] += np.repeat(off, 2)
    ext = bounds[:, 3:] - bounds[:, :3]
    mb = np.zeros((2 * n, 4))
    mb[:, 3] = 0.5 * np.maximum(np.maximum(ext[:, 0], ext[:, 1]), ext[:, 2])  # MotionBoundForAabb
    k = np.arange(n, dtype=np.uint64)
    t0 = k.astype(np.float64) * BATCH_SLAB_STRIDE
    patch = np.empty(2 * n, np.uint32)
    patch[0::2] = (2 * k + 1).astype(np.uint32)
    patch[1::2] = (2 * k + 2).astype(np.uint32)
    obj = np.empty(2 * n, np.uint32)
    obj[0::2], obj[1::2] = 1, 2
    return {"query_id": BATCH_SCENE_QUERY_ID, "n": 2 * n, "object_id": obj, "patch_id": patch,
            "slab_id": np.repeat(k.astype(np.uint32), 2), "proxy_type": np.ones(2 * n, np.uint8),
            "t0": np.repeat(t0, 2), "t1": np.repeat(t0 + 1.0, 2), "bounds": bounds, "motion_bound": mb}


def _validate_bounds(scene: dict) -> None:
    """ValidateProxyScene's bound check (proxy_scene.cpp:143-151) for the
    encoded scene; ids, types and the slab partition are valid by
    construction (one slab per query, [2k, 2k+1])."""
    b = scene["bounds"]
    if not np.all(np.isfinite(b)):
        raise ExternalBatchError("proxy bounds contain a non-finite value")


def translate(cand: np.ndarray, b: dict, rid: np.ndarray) -> tuple:
    """Candidates of the batched scene back in their queries' terms (:255-303)
    and the set of queries with at least one candidate."""
    q = (cand["patch_a_id"].astype(np.int64) - 1) // 2
    qb = (cand["patch_b_id"].astype(np.int64) - 1) // 2
    if np.any(q != qb):
        raise ExternalBatchError("external batch candidate crossed query boundaries")
    out = cand.copy()
    out["query_id"] = rid[q]
    has = b["has_box"][q] != 0
    out["object_a_id"] = np.where(has, b["box_pair"][q, 0], 1)
    out["object_b_id"] = np.where(has, b["box_pair"][q, 1], 2)
    out["patch_a_id"] = np.where(b["family"][q] == 0, 0, 1)
    out["patch_b_id"] = b["source_query_index"][q].astype(np.uint64) + 1 & 0xFFFFFFFF
    out["proxy_type_a"] = 1
    out["proxy_type_b"] = 1
    order = np.lexsort((out["patch_b_id"], out["patch_a_id"], out["query_id"]))
    sorted_out = np.zeros(len(out), CANDIDATE_RECORD_DTYPE)  # zero padding, field by field
    for f in CANDIDATE_RECORD_DTYPE.names:
        sorted_out[f] = out[f][order]
    out = sorted_out
    with np.errstate(over="ignore"):
        out["candidate_id"] = (out["query_id"] * np.uint64(CANDIDATE_ID_STRIDE) +
                               np.arange(len(out), dtype=np.uint64) + np.uint64(1))
    if np.any(out["candidate_id"] == 0):
        raise ExternalBatchError("CandidateRecord.candidate_id is required")
    return out, np.unique(q)


def candidate_recall(b: dict, active: np.ndarray) -> float:
    """Covered ground-truth positives over positives, 1 with none (:305-317)."""
    pos = b["ground_truth"] > 0
    total = int(pos.sum())
    if total == 0:
        return 1.0
    covered = np.zeros(len(pos), bool)
    covered[active] = True
    return float((pos & covered).sum()) / float(total)


def generate(b: dict, device=None) -> dict:
    """GenerateCandidatesForExternalBatch (:231-339) with the broad phase on
    the GPU.  Returns the translated candidates (CANDIDATE_RECORD_DTYPE), the
    runtime id per query, the counts, the recall and per-stage host timings."""
    from p2cccd_b200.proxy import ProxyCandidates

    n = len(b["query_id"])
    if n == 0:
        raise ExternalBatchError("external batch candidate generation requires at least one query")
    start = time.perf_counter()
    _first_error(b)
    rid = runtime_query_ids(b["query_id"])
    scene = encode_scene(b)
    _validate_bounds(scene)
    t_enc = time.perf_counter()
    raw, cand = ProxyCandidates(scene, device=device or "cuda").run_checked()
    t_gen = time.perf_counter()
    out, active = translate(cand, b, rid)
    t_end = time.perf_counter()
    return {"candidates": out, "runtime_query_ids": rid, "primitive_count": 2 * n, "raw_hit_count": len(raw),
            "compact_candidate_count": len(out), "candidate_recall": candidate_recall(b, active),
            "encode_ms": (t_enc - start) * 1e3, "generate_ms": (t_gen - t_enc) * 1e3,
            "compact_ms": (t_end - t_gen) * 1e3}
