"""numpy record dtypes of the C ABI (include/p2c_b200.h).

They are byte-identical to the reference's host structs
(``cpp/certificate/certificate_engine.h:32-81``): a packed array of these
records is what ``std::vector<PointTriangleIntervalPrimitive>`` holds.
"""
from __future__ import annotations

import numpy as np

TRAJECTORY_DTYPE = np.dtype([
    ("feature_id", "<i8"),
    ("position_t0", "<f8", (3,)),
    ("position_t1", "<f8", (3,)),
])

POINT_TRIANGLE_DTYPE = np.dtype([
    ("point_id", "<i8"),
    ("triangle_id", "<i8"),
    ("point", TRAJECTORY_DTYPE),
    ("triangle_v0", TRAJECTORY_DTYPE),
    ("triangle_v1", TRAJECTORY_DTYPE),
    ("triangle_v2", TRAJECTORY_DTYPE),
])

EDGE_EDGE_DTYPE = np.dtype([
    ("edge_a_id", "<i8"),
    ("edge_b_id", "<i8"),
    ("edge_a0", TRAJECTORY_DTYPE),
    ("edge_a1", TRAJECTORY_DTYPE),
    ("edge_b0", TRAJECTORY_DTYPE),
    ("edge_b1", TRAJECTORY_DTYPE),
])

INTERVAL_RESULT_DTYPE = np.dtype({
    "names": ["status", "covered_feature_mask", "interval_t0", "interval_t1", "toi_upper",
              "safe_margin_lb", "witness_family", "witness_id_a", "witness_id_b", "reason_code",
              "next_refinement_mode"],
    "formats": ["u1", "<u4", "<f8", "<f8", "<f8", "<f8", "u1", "<i8", "<i8", "<u2", "u1"],
    "offsets": [0, 4, 8, 16, 24, 32, 40, 48, 56, 64, 66],
    "itemsize": 72,
})

QUERY_CERTIFICATE_DTYPE = np.dtype({
    "names": ["status", "witness_family", "reason_code", "covered_feature_mask", "toi_upper",
              "safe_margin_lb", "witness_id_a", "witness_id_b", "witness_index", "next_refinement_mode"],
    "formats": ["u1", "u1", "<u2", "<u4", "<f8", "<f8", "<i8", "<i8", "<i8", "u1"],
    "offsets": [0, 1, 2, 4, 8, 16, 24, 32, 40, 48],
    "itemsize": 56,
})

CERTIFY_STATS_DTYPE = np.dtype([
    ("nodes_evaluated", "<u8"),
    ("distance_evals", "<u8"),
    ("fp64_ops", "<u8"),
    ("donations", "<u8"),
    ("queries", "<u8"),
    ("error_word", "<u8"),
    ("max_warp_iterations", "<u8"),
    ("busy_lane_iterations", "<u8"),
])

# RawCandidateHit (rt_candidate/candidate_buffer.h:19-31) and CandidateRecord
# (common/runtime_contracts.h:41-56), the broad-phase output contracts.
RAW_HIT_DTYPE = np.dtype({
    "names": ["query_id", "pair_key", "proxy_a_index", "proxy_b_index", "slab_id", "rt_hit_count", "flags",
              "reserved0", "motion_bound", "reserved1", "reserved2"],
    "formats": ["<u8", "<u8", "<u4", "<u4", "<u4", "<u4", "<u4", "<u4", ("<f4", (4,)), "<u4", "<u4"],
    "offsets": [0, 8, 16, 20, 24, 28, 32, 36, 40, 56, 60],
    "itemsize": 64,
})
CANDIDATE_RECORD_DTYPE = np.dtype({
    "names": ["schema_version", "candidate_id", "query_id", "slab_id", "object_a_id", "patch_a_id", "object_b_id",
              "patch_b_id", "proxy_type_a", "proxy_type_b", "rt_hit_count", "motion_bound",
              "proxy_features_offset", "flags"],
    "formats": ["<u4", "<u8", "<u8", "<u4", "<u4", "<u4", "<u4", "<u4", "u1", "u1", "<u4", ("<f4", (4,)), "<u4",
                "<u4"],
    "offsets": [0, 8, 16, 24, 28, 32, 36, 40, 44, 45, 48, 52, 68, 72],
    "itemsize": 80,
})

assert POINT_TRIANGLE_DTYPE.itemsize == 240
assert EDGE_EDGE_DTYPE.itemsize == 240
assert INTERVAL_RESULT_DTYPE.itemsize == 72

# CertificateStatus / reason / refinement constants (runtime_contracts.h:20-31,
# certificate_engine.h:12-22)
STATUS_COLLISION = 0
STATUS_SEPARATION = 1
STATUS_UNDECIDED = 2
FAMILY_POINT_TRIANGLE = 1
FAMILY_EDGE_EDGE = 2
REASON_NONE = 0
REASON_MISSING_GEOMETRY = 1
REASON_MAX_SUBDIVISION_DEPTH = 2
REASON_INVALID_INPUT = 3
REFINE_NONE = 0
REFINE_BISECT_INTERVAL = 1
REFINE_REQUEST_GEOMETRY = 2
REFINE_ESCALATE_PRECISION = 3

RESULT_FIELDS = INTERVAL_RESULT_DTYPE.names


def pack_primitives(p0: np.ndarray, p1: np.ndarray, ids_a: np.ndarray, ids_b: np.ndarray,
                    feature_ids: np.ndarray | None = None, family: int = FAMILY_POINT_TRIANGLE) -> np.ndarray:
    """Pack (n, 4, 3) t0/t1 positions plus ids into 240-byte records.

    Vertex order is (point, v0, v1, v2) for point-triangle and (a0, a1, b0, b1)
    for edge-edge.
    """
    n = p0.shape[0]
    dt = POINT_TRIANGLE_DTYPE if family == FAMILY_POINT_TRIANGLE else EDGE_EDGE_DTYPE
    rec = np.zeros(n, dtype=dt)
    names = dt.names
    rec[names[0]] = ids_a
    rec[names[1]] = ids_b
    for k in range(4):
        rec[names[2 + k]]["position_t0"] = p0[:, k, :]
        rec[names[2 + k]]["position_t1"] = p1[:, k, :]
        rec[names[2 + k]]["feature_id"] = -1 if feature_ids is None else feature_ids[:, k]
    return rec


def unpack_positions(rec: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Inverse of pack_primitives for the geometry: (n, 4, 3) t0 and t1 arrays."""
    names = rec.dtype.names
    p0 = np.stack([rec[names[2 + k]]["position_t0"] for k in range(4)], axis=1)
    p1 = np.stack([rec[names[2 + k]]["position_t1"] for k in range(4)], axis=1)
    return p0, p1


# CandidateDensityStats without timing / backend name (p2c_candidate_density, 96 bytes)
DENSITY_DTYPE = np.dtype({
    "names": ["query_id", "proxy_count", "object_count", "slab_count", "cross_object_same_slab_pair_count",
              "raw_hit_count", "compact_candidate_count", "raw_hits_per_proxy", "candidates_per_proxy",
              "candidates_per_slab", "aabb_overlap_ratio", "avg_rt_hits_per_candidate"],
    "formats": ["<u8"] * 7 + ["<f8"] * 5,
    "offsets": [8 * k for k in range(12)],
    "itemsize": 96,
})

# ProposalFeatureRow (proposal/proposal_features.h:27-43), 256 bytes
FEATURE_ROW_DTYPE = np.dtype({
    "names": ["schema_version", "query_id", "candidate_id", "slab_id", "object_a_id", "patch_a_id", "object_b_id",
              "patch_b_id", "features", "interval_targets", "family_targets", "priority_target", "cost_target",
              "uncertainty_target", "target_mask"],
    "formats": ["<u4", "<u8", "<u8", "<u4", "<u4", "<u4", "<u4", "<u4", ("<f4", (32,)), ("<f4", (8,)),
                ("<f4", (8,)), "<f4", "<f4", "<f4", "<u4"],
    "offsets": [0, 8, 16, 24, 28, 32, 36, 40, 44, 172, 204, 236, 240, 244, 248],
    "itemsize": 256,
})


# the ExactWorkItem fields an audit row reads (p2c_audit_item, 56 bytes)
AUDIT_ITEM_DTYPE = np.dtype({
    "names": ["query_id", "candidate_id", "work_item_id", "interval_t0", "interval_t1", "priority_score",
              "feature_family_mask", "depth"],
    "formats": ["<u8", "<u8", "<u8", "<f8", "<f8", "<f4", "<u4", "<u2"],
    "offsets": [0, 8, 16, 24, 32, 40, 44, 48],
    "itemsize": 56,
})

# AuditLogRow (common/runtime_contracts.h:101-114), 80 bytes
AUDIT_ROW_DTYPE = np.dtype({
    "names": ["event_id", "query_id", "candidate_id", "work_item_id", "stage", "action", "depth", "interval_t0",
              "interval_t1", "timestamp_us", "aux_value0", "aux_value1"],
    "formats": ["<u8", "<u8", "<u8", "<u8", "u1", "<u2", "<u2", "<f8", "<f8", "<u8", "<f8", "<f8"],
    "offsets": [0, 8, 16, 24, 32, 34, 36, 40, 48, 56, 64, 72],
    "itemsize": 80,
})


# ProposalOutput (common/runtime_contracts.h:58-65), 88 bytes
PROPOSAL_OUTPUT_DTYPE = np.dtype({
    "names": ["candidate_id", "interval_scores", "family_scores", "priority_score", "cost_score",
              "uncertainty_score"],
    "formats": ["<u8", ("<f4", (8,)), ("<f4", (8,)), "<f4", "<f4", "<f4"],
    "offsets": [0, 8, 40, 72, 76, 80],
    "itemsize": 88,
})

# ExactWorkItem (common/runtime_contracts.h:67-81), 80 bytes
EXACT_WORK_ITEM_DTYPE = np.dtype({
    "names": ["work_item_id", "parent_candidate_id", "query_id", "slab_id", "patch_a_id", "patch_b_id",
              "interval_t0", "interval_t1", "feature_family_mask", "topk_feature_ids_offset", "depth",
              "priority_score", "source"],
    "formats": ["<u8", "<u8", "<u8", "<u4", "<u4", "<u4", "<f8", "<f8", "<u4", "<u4", "<u2", "<f4", "u1"],
    "offsets": [0, 8, 16, 24, 28, 32, 40, 48, 56, 60, 64, 68, 72],
    "itemsize": 80,
})

SCHEDULE_STATS_FIELDS = ("raw_candidate_count", "proposal_output_count", "work_item_count", "fallback_count",
                         "missing_proposal_fallback_count", "invalid_proposal_fallback_count", "ood_fallback_count",
                         "high_uncertainty_fallback_count", "reordered_count", "monotonic_safe")
SCHEDULE_STATS_DTYPE = np.dtype([(k, "<u8") for k in SCHEDULE_STATS_FIELDS])

# p2c_dense_group_stats (DenseGroupEarlyStopStats without host timings, plus
# the first invalid row)
DENSE_GROUP_STATS_DTYPE = np.dtype([
    ("candidate_count", "<u8"), ("group_count", "<u8"), ("positive_group_count", "<u8"),
    ("no_proposal_exact_calls", "<u8"), ("no_proposal_exact_work", "<f8"), ("learned_exact_calls", "<u8"),
    ("learned_fallback_calls", "<u8"), ("learned_interval_hit_count", "<u8"),
    ("learned_interval_miss_count", "<u8"), ("learned_exact_work", "<f8"), ("first_positive_rank_sum", "<f8"),
    ("cost_before_first_positive_sum", "<f8"), ("tp", "<u8"), ("tn", "<u8"), ("fp", "<u8"), ("fn", "<u8"),
    ("reordered_count", "<u8"), ("high_uncertainty_group_count", "<u8"), ("error_row", "<i8"),
    ("error_kind", "<i4"), ("pad", "<i4")])
assert DENSE_GROUP_STATS_DTYPE.itemsize == 160
