"""``p2cccd_cpp`` — the reference's compiled module surface for the
certification hot path, backed by the B200 library.

The reference builds ``p2cccd_cpp`` with pybind11
(cpp/bindings/py_module.cpp:1803-2015); its Python host API
(``p2cccd.cuda_bindings``, ``p2cccd.bench.rt_exact``) imports it by that name.
This module keeps the names, argument meanings, return types and error
convention (``ValueError`` for every reference ``Status`` error,
py_module.cpp:38-42) of the entry points on this path, so those callers switch
by putting this directory first on ``sys.path``.  Every certificate is computed
by ``libp2c_b200.so`` on the GPU; there is no CPU certifier here (names ending
in ``_cpu`` keep the reference's name; they run on the GPU too).

Beyond the reference surface, ``*_tensor`` entry points take and return CUDA
tensors of 240-byte / 72-byte records (``device_pointer_abi`` is True).
"""
from __future__ import annotations

import enum
import math
from typing import Any, Sequence

import numpy as np

from p2cccd_b200 import _lib, records as _rec
from p2cccd_b200.certify import CertConfig as _CertConfig

# ---------------------------------------------------------------------------
# enums (py_module.cpp:1326-1357)


class ProxyType(enum.IntEnum):
    UNKNOWN = 0
    SWEPT_AABB = 1
    CAPSULE = 2


class ProposalSource(enum.IntEnum):
    RAW = 0
    REFINED = 1
    FALLBACK = 2


class CertificateStatus(enum.IntEnum):
    COLLISION = 0
    SEPARATION = 1
    UNDECIDED = 2
    Collision = 0
    Separation = 1
    Undecided = 2


class CertificateRefinementMode(enum.IntEnum):
    NONE = 0
    BISECT_INTERVAL = 1
    REQUEST_GEOMETRY = 2
    ESCALATE_PRECISION = 3


class AuditStage(enum.IntEnum):
    RT = 0
    PROPOSAL = 1
    EXACT = 2
    REFINE = 3
    CERTIFY = 4


FEATURE_FAMILY_POINT_TRIANGLE = 1
FEATURE_FAMILY_EDGE_EDGE = 2
CERTIFICATE_REASON_NONE = 0
CERTIFICATE_REASON_MISSING_GEOMETRY = 1
CERTIFICATE_REASON_MAX_SUBDIVISION_DEPTH = 2
CERTIFICATE_REASON_INVALID_INPUT = 3
EXACT_AUDIT_DEQUEUED = 1
EXACT_AUDIT_COLLISION = 2
EXACT_AUDIT_SEPARATION = 3
EXACT_AUDIT_UNDECIDED = 4
EXACT_AUDIT_INVALID_INPUT = 5
CUDA_DEVICE_POINTER_ABI_ENABLED = True


# ---------------------------------------------------------------------------
# plain structs with the reference's fields and defaults


class _Struct:
    _fields: tuple = ()

    def __init__(self):
        for name, default in self._fields:
            object.__setattr__(self, name, default() if callable(default) else default)

    def __repr__(self):
        inner = ", ".join(f"{n}={getattr(self, n)!r}" for n, _ in self._fields)
        return f"{type(self).__name__}({inner})"

    def __eq__(self, other):
        return type(self) is type(other) and all(getattr(self, n) == getattr(other, n) for n, _ in self._fields)


def _vec3(v) -> list:
    out = [float(x) for x in v]
    if len(out) != 3:
        raise TypeError("expected a sequence of 3 floats")
    return out


class LinearVertexTrajectory(_Struct):
    _fields = (("feature_id", -1), ("position_t0", lambda: [0.0, 0.0, 0.0]),
               ("position_t1", lambda: [0.0, 0.0, 0.0]))

    def __setattr__(self, name, value):
        if name in ("position_t0", "position_t1"):
            value = _vec3(value)
        elif name == "feature_id":
            value = int(value)
        object.__setattr__(self, name, value)


class PointTriangleIntervalPrimitive(_Struct):
    _fields = (("point_id", -1), ("triangle_id", -1), ("point", LinearVertexTrajectory),
               ("triangle_v0", LinearVertexTrajectory), ("triangle_v1", LinearVertexTrajectory),
               ("triangle_v2", LinearVertexTrajectory))


class EdgeEdgeIntervalPrimitive(_Struct):
    _fields = (("edge_a_id", -1), ("edge_b_id", -1), ("edge_a0", LinearVertexTrajectory),
               ("edge_a1", LinearVertexTrajectory), ("edge_b0", LinearVertexTrajectory),
               ("edge_b1", LinearVertexTrajectory))


class CertificateEngineConfig(_Struct):
    _fields = (("eps_time", 1.0e-4), ("eps_space", 1.0e-6), ("max_subdivision_depth", 32))

    def __setattr__(self, name, value):
        if name == "max_subdivision_depth":
            value = int(value)
            if not 0 <= value <= 0xFFFF:
                raise TypeError("max_subdivision_depth must fit in uint16")
        else:
            value = float(value)
        object.__setattr__(self, name, value)


class PrimitiveIntervalResult(_Struct):
    _fields = (("status", CertificateStatus.UNDECIDED), ("covered_feature_mask", 0), ("interval_t0", 0.0),
               ("interval_t1", 1.0), ("toi_upper", 1.0), ("safe_margin_lb", 0.0), ("witness_family", 0),
               ("witness_id_a", -1), ("witness_id_b", -1), ("reason_code", 0),
               ("next_refinement_mode", CertificateRefinementMode.NONE))


class ExactWorkItem(_Struct):
    _fields = (("work_item_id", 0), ("parent_candidate_id", 0), ("query_id", 0), ("slab_id", 0), ("patch_a_id", 0),
               ("patch_b_id", 0), ("interval_t0", 0.0), ("interval_t1", 1.0), ("feature_family_mask", 0),
               ("topk_feature_ids_offset", 0), ("depth", 0), ("priority_score", 0.0),
               ("source", ProposalSource.RAW))


class CertificateResult(_Struct):
    _fields = (("work_item_id", 0), ("query_id", 0), ("status", CertificateStatus.UNDECIDED), ("interval_t0", 0.0),
               ("interval_t1", 1.0), ("toi_upper", 1.0), ("safe_margin_lb", 0.0), ("witness_family", 0),
               ("witness_id_a", -1), ("witness_id_b", -1), ("covered_feature_mask", 0), ("eps_time", 1.0e-4),
               ("eps_space", 1.0e-6), ("reason_code", 0), ("next_refinement_mode", CertificateRefinementMode.NONE))


class AuditLogRow(_Struct):
    _fields = (("event_id", 0), ("query_id", 0), ("candidate_id", 0), ("work_item_id", 0), ("stage", AuditStage.RT),
               ("action", 0), ("depth", 0), ("interval_t0", 0.0), ("interval_t1", 1.0), ("timestamp_us", 0),
               ("aux_value0", 0.0), ("aux_value1", 0.0))


class ExactCertificateQuery(_Struct):
    _fields = (("work_item", ExactWorkItem), ("config", CertificateEngineConfig),
               ("point_triangle_primitives", list), ("edge_edge_primitives", list))


class ExactWorkQueueConfig(_Struct):
    _fields = (("first_event_id", 1), ("first_timestamp_us", 1), ("emit_dequeue_events", True))


class ExactWorkQueueResult(_Struct):
    _fields = (("certificates", list), ("audit_log", list), ("processed_count", 0))


class ExactRefinementConfig(_Struct):
    _fields = (("first_child_work_item_id", 1), ("max_child_depth", 64), ("min_interval_width", 1.0e-4))


class Mesh(_Struct):
    _fields = (("vertices_ref", list), ("triangles", list), ("patch_ids", list))


class MeshExactBuildConfig(_Struct):
    _fields = (("prune_by_swept_aabb", True), ("max_point_triangle_primitives", 0), ("max_edge_edge_primitives", 0))


class MeshExactBuildStats(_Struct):
    _fields = tuple((n, 0) for n in (
        "vertex_count_a", "vertex_count_b", "triangle_count_a", "triangle_count_b", "edge_count_a", "edge_count_b",
        "point_triangle_total_pairs", "point_triangle_kept_pairs", "point_triangle_pruned_pairs",
        "edge_edge_total_pairs", "edge_edge_kept_pairs", "edge_edge_pruned_pairs"))


class MeshExactBuildResult(_Struct):
    _fields = (("query", ExactCertificateQuery), ("stats", MeshExactBuildStats))


# ---------------------------------------------------------------------------
# conversions between these structs and the ABI records

_PT_NAMES = ("point", "triangle_v0", "triangle_v1", "triangle_v2")
_EE_NAMES = ("edge_a0", "edge_a1", "edge_b0", "edge_b1")


def _to_records(prims: Sequence[Any], family: int) -> np.ndarray:
    dt = _rec.POINT_TRIANGLE_DTYPE if family == 1 else _rec.EDGE_EDGE_DTYPE
    names = _PT_NAMES if family == 1 else _EE_NAMES
    ids = ("point_id", "triangle_id") if family == 1 else ("edge_a_id", "edge_b_id")
    n = len(prims)
    flat = np.zeros((n, 30), dtype=np.float64)
    iv = flat.view(np.int64)
    for i, p in enumerate(prims):
        iv[i, 0] = int(getattr(p, ids[0]))
        iv[i, 1] = int(getattr(p, ids[1]))
        for k, nm in enumerate(names):
            t = getattr(p, nm)
            iv[i, 2 + 7 * k] = int(t.feature_id)
            flat[i, 3 + 7 * k:6 + 7 * k] = t.position_t0
            flat[i, 6 + 7 * k:9 + 7 * k] = t.position_t1
    return flat.view(np.uint8).reshape(n, 240).view(dt).reshape(-1) if n else np.zeros(0, dtype=dt)


def _from_records(rec: np.ndarray, family: int) -> list:
    names = _PT_NAMES if family == 1 else _EE_NAMES
    cls = PointTriangleIntervalPrimitive if family == 1 else EdgeEdgeIntervalPrimitive
    ids = ("point_id", "triangle_id") if family == 1 else ("edge_a_id", "edge_b_id")
    out = []
    for r in rec:
        p = cls()
        setattr(p, ids[0], int(r[ids[0]]))
        setattr(p, ids[1], int(r[ids[1]]))
        for nm in names:
            t = LinearVertexTrajectory()
            t.feature_id = int(r[nm]["feature_id"])
            t.position_t0 = r[nm]["position_t0"].tolist()
            t.position_t1 = r[nm]["position_t1"].tolist()
            setattr(p, nm, t)
        out.append(p)
    return out


def _result_objects(res: np.ndarray) -> list:
    out = []
    for r in res:
        o = PrimitiveIntervalResult()
        o.status = CertificateStatus(int(r["status"]))
        o.covered_feature_mask = int(r["covered_feature_mask"])
        o.interval_t0 = float(r["interval_t0"])
        o.interval_t1 = float(r["interval_t1"])
        o.toi_upper = float(r["toi_upper"])
        o.safe_margin_lb = float(r["safe_margin_lb"])
        o.witness_family = int(r["witness_family"])
        o.witness_id_a = int(r["witness_id_a"])
        o.witness_id_b = int(r["witness_id_b"])
        o.reason_code = int(r["reason_code"])
        o.next_refinement_mode = CertificateRefinementMode(int(r["next_refinement_mode"]))
        out.append(o)
    return out


def _config(c: CertificateEngineConfig) -> _CertConfig:
    return _CertConfig(float(c.eps_time), float(c.eps_space), int(c.max_subdivision_depth))


# ---------------------------------------------------------------------------
# restated validators (cpp/common/validators.cpp)


def _require_nonzero(v, name):
    if int(v) == 0:
        raise ValueError(f"{name} is required")


def _require_finite(v, name):
    if not math.isfinite(float(v)):
        raise ValueError(f"{name} must be finite")


def _validate_unit_interval(t0, t1):  # :60-72
    _require_finite(t0, "interval_t0")
    _require_finite(t1, "interval_t1")
    if t0 < 0.0 or t1 > 1.0 or t0 > t1:
        raise ValueError("interval must satisfy 0 <= interval_t0 <= interval_t1 <= 1")


def validate_exact_work_item(item: ExactWorkItem) -> bool:  # validators.cpp:207-230
    _require_nonzero(item.work_item_id, "ExactWorkItem.work_item_id")
    _require_nonzero(item.parent_candidate_id, "ExactWorkItem.parent_candidate_id")
    _require_nonzero(item.query_id, "ExactWorkItem.query_id")
    _validate_unit_interval(item.interval_t0, item.interval_t1)
    if int(item.feature_family_mask) == 0:
        raise ValueError("ExactWorkItem.feature_family_mask is required")
    _require_finite(item.priority_score, "ExactWorkItem.priority_score")
    if int(item.source) not in (0, 1, 2):
        raise ValueError("ExactWorkItem.source is invalid")
    return True


def validate_certificate_result(result: CertificateResult) -> bool:  # validators.cpp:232-293
    _require_nonzero(result.work_item_id, "CertificateResult.work_item_id")
    _require_nonzero(result.query_id, "CertificateResult.query_id")
    if int(result.status) not in (0, 1, 2):
        raise ValueError("CertificateResult.status is invalid")
    _validate_unit_interval(result.interval_t0, result.interval_t1)
    _require_finite(result.toi_upper, "CertificateResult.toi_upper")
    _require_finite(result.safe_margin_lb, "CertificateResult.safe_margin_lb")
    for v, n in ((result.eps_time, "CertificateResult.eps_time"), (result.eps_space, "CertificateResult.eps_space")):
        _require_finite(v, n)
        if not v > 0.0:
            raise ValueError(f"{n} must be positive")
    if int(result.next_refinement_mode) not in (0, 1, 2, 3):
        raise ValueError("CertificateResult.next_refinement_mode is invalid")
    st, mode = int(result.status), int(result.next_refinement_mode)
    if st == 0:
        if result.toi_upper < result.interval_t0 or result.toi_upper > result.interval_t1:
            raise ValueError("CertificateResult.toi_upper must lie inside the certified interval")
        if result.witness_id_a < 0 or result.witness_id_b < 0:
            raise ValueError("CertificateResult collision witnesses are required")
        if mode != 0:
            raise ValueError("CertificateResult collision cannot request refinement")
    if st == 1:
        if result.safe_margin_lb < 0.0:
            raise ValueError("CertificateResult.safe_margin_lb must be non-negative")
        if result.covered_feature_mask == 0:
            raise ValueError("CertificateResult.covered_feature_mask is required for separation")
        if mode != 0:
            raise ValueError("CertificateResult separation cannot request refinement")
    if st == 2 and int(result.reason_code) == 0:
        raise ValueError("CertificateResult.reason_code is required for undecided results")
    if st == 2 and mode == 0:
        raise ValueError("CertificateResult.next_refinement_mode is required for undecided results")
    return True


def validate_audit_log_row(row: AuditLogRow) -> bool:  # validators.cpp ValidateAuditLogRow
    _require_nonzero(row.event_id, "AuditLogRow.event_id")
    _require_nonzero(row.query_id, "AuditLogRow.query_id")
    if int(row.stage) not in (0, 1, 2, 3, 4):
        raise ValueError("AuditLogRow.stage is invalid")
    _validate_unit_interval(row.interval_t0, row.interval_t1)
    if int(row.timestamp_us) == 0:
        raise ValueError("AuditLogRow.timestamp_us is required")
    _require_finite(row.aux_value0, "AuditLogRow.aux_value0")
    _require_finite(row.aux_value1, "AuditLogRow.aux_value1")
    return True


def validate_audit_log_rows(rows: Sequence[AuditLogRow]) -> bool:  # py_module.cpp:470-475
    for r in rows:
        validate_audit_log_row(r)
    return True


def audit_log_rows_for_query(rows: Sequence[AuditLogRow], query_id: int) -> list:  # py_module.cpp:477-487
    return [r for r in rows if r.query_id == query_id]


def _validate_config(c: CertificateEngineConfig) -> None:  # certificate_engine.cpp:224-232
    if not math.isfinite(c.eps_time) or c.eps_time <= 0.0:
        raise ValueError("CertificateEngineConfig.eps_time must be finite and positive")
    if not math.isfinite(c.eps_space) or c.eps_space <= 0.0:
        raise ValueError("CertificateEngineConfig.eps_space must be finite and positive")


# ---------------------------------------------------------------------------
# CUDA batch entry points (cuda_bindings.py:8-14; py_module.cpp:1966-1991)


def is_cuda_exact_built() -> bool:
    return bool(_lib.load().p2c_is_cuda_exact_built())


def cuda_binding_status() -> dict:
    built = is_cuda_exact_built()
    return {
        "cuda_exact_built": built,
        "host_batch_exact_api": True,
        "device_pointer_abi": True,
        "backend_name": "b200_sm100a" if built else "unavailable",
        "safety_policy": ("host-owned batch entry points copy in and out on the library's stream; "
                          "*_tensor entry points take caller-owned CUDA tensors and never free them."),
    }


def _batch(primitives, family, interval_t0, interval_t1, config):
    from p2cccd_b200 import certify

    rec = _to_records(list(primitives), family)
    res = certify.certify_batch_host(rec, float(interval_t0), float(interval_t1), _config(config))
    return _result_objects(res)


def evaluate_point_triangle_batch_cuda(primitives, interval_t0, interval_t1, config) -> list:
    return _batch(primitives, 1, interval_t0, interval_t1, config)


def evaluate_edge_edge_batch_cuda(primitives, interval_t0, interval_t1, config) -> list:
    return _batch(primitives, 2, interval_t0, interval_t1, config)


def evaluate_point_triangle_interval(primitive, interval_t0, interval_t1, config) -> PrimitiveIntervalResult:
    return _batch([primitive], 1, interval_t0, interval_t1, config)[0]


def evaluate_edge_edge_interval(primitive, interval_t0, interval_t1, config) -> PrimitiveIntervalResult:
    return _batch([primitive], 2, interval_t0, interval_t1, config)[0]


def evaluate_point_triangle_batch_cuda_tensor(records, interval_t0, interval_t1, config):
    """CUDA uint8 (n, 240) records -> CUDA uint8 (n, 72) results (caller's stream, asynchronous)."""
    from p2cccd_b200 import certify

    return certify.certify_batch(records, 1, interval_t0, interval_t1, _config(config))


def evaluate_edge_edge_batch_cuda_tensor(records, interval_t0, interval_t1, config):
    from p2cccd_b200 import certify

    return certify.certify_batch(records, 2, interval_t0, interval_t1, _config(config))


def _compare(a: np.ndarray, b: np.ndarray, eps_cert: float, label: str) -> None:
    """ComparePrimitiveResults (certificate_cuda.cu:554-583)."""
    for x, y in zip(a, b):
        if x["status"] != y["status"]:
            raise ValueError(f"{label} status mismatch")
        if x["covered_feature_mask"] != y["covered_feature_mask"]:
            raise ValueError(f"{label} covered feature mask mismatch")
        if x["status"] == 0:
            if abs(x["toi_upper"] - y["toi_upper"]) > eps_cert:
                raise ValueError(f"{label} TOI mismatch")
            if (x["witness_family"], x["witness_id_a"], x["witness_id_b"]) != (
                    y["witness_family"], y["witness_id_a"], y["witness_id_b"]):
                raise ValueError(f"{label} witness mismatch")
        if x["status"] == 1 and abs(x["safe_margin_lb"] - y["safe_margin_lb"]) > eps_cert:
            raise ValueError(f"{label} safe margin mismatch")
        if x["status"] == 2 and (x["reason_code"], x["next_refinement_mode"]) != (
                y["reason_code"], y["next_refinement_mode"]):
            raise ValueError(f"{label} undecided refinement mismatch")


def cross_check_cpu_cuda_exact(point_triangles, edge_edges, interval_t0, interval_t1, config, eps_cert) -> bool:
    """CrossCheckCpuCudaExact (certificate_cuda.cu:616-679): the GPU engine's
    certificates (the production launch, as evaluate_*_batch_cuda returns
    them) against the library's CPU certifier (p2c_certify_*_batch_cpu, an
    independent host evaluation of the recursion), with the reference's
    comparison rules; raises ValueError with the reference's message on the
    first mismatch, returns True otherwise."""
    from p2cccd_b200 import certify

    if not math.isfinite(float(eps_cert)) or float(eps_cert) < 0.0:
        raise ValueError("eps_cert must be finite and non-negative")
    cfg = _config(config)
    pt = _to_records(list(point_triangles), 1)
    ee = _to_records(list(edge_edges), 2)
    gpu_pt = certify.certify_batch_host(pt, interval_t0, interval_t1, cfg)
    cpu_pt = certify.certify_batch_cpu(pt, interval_t0, interval_t1, cfg)
    _compare(cpu_pt, gpu_pt, float(eps_cert), "point-triangle CPU/CUDA cross-check")
    gpu_ee = certify.certify_batch_host(ee, interval_t0, interval_t1, cfg)
    cpu_ee = certify.certify_batch_cpu(ee, interval_t0, interval_t1, cfg)
    _compare(cpu_ee, gpu_ee, float(eps_cert), "edge-edge CPU/CUDA cross-check")
    return True


# ---------------------------------------------------------------------------
# certificate engine and work queue (certificate_engine.cpp:593-824)


def _base_certificate(item: ExactWorkItem, cfg: CertificateEngineConfig) -> CertificateResult:  # :388-402
    r = CertificateResult()
    r.work_item_id = item.work_item_id
    r.query_id = item.query_id
    r.interval_t0 = item.interval_t0
    r.interval_t1 = item.interval_t1
    r.toi_upper = item.interval_t1
    r.eps_time = cfg.eps_time
    r.eps_space = cfg.eps_space
    r.status = CertificateStatus.UNDECIDED
    r.reason_code = CERTIFICATE_REASON_MISSING_GEOMETRY
    r.next_refinement_mode = CertificateRefinementMode.REQUEST_GEOMETRY
    return r


def _certify_queries(queries: Sequence[ExactCertificateQuery]) -> list:
    """One GPU launch per distinct config; returns per query a CertificateResult
    or a ValueError (the Status Evaluate would return)."""
    from p2cccd_b200 import queue

    out: list = [None] * len(queries)
    groups: dict = {}
    for i, q in enumerate(queries):
        try:
            _validate_config(q.config)
        except ValueError as exc:
            out[i] = exc
            continue
        key = (float(q.config.eps_time), float(q.config.eps_space), int(q.config.max_subdivision_depth))
        groups.setdefault(key, []).append(i)
    for key, idx in groups.items():
        pts, ees, pto, eeo, t0, t1, mask = [], [], [0], [0], [], [], []
        for i in idx:
            q = queries[i]
            m = int(q.work_item.feature_family_mask)
            p = list(q.point_triangle_primitives) if m & 1 else []
            e = list(q.edge_edge_primitives) if m & 2 else []
            pts += p
            ees += e
            pto.append(pto[-1] + len(p))
            eeo.append(eeo[-1] + len(e))
            t0.append(float(q.work_item.interval_t0))
            t1.append(float(q.work_item.interval_t1))
            mask.append(m)
        res = queue.certify_work_items(_to_records(pts, 1), np.array(pto), _to_records(ees, 2), np.array(eeo),
                                       np.array(t0), np.array(t1), np.array(mask, np.uint32), _CertConfig(*key))
        invalid_msg = _first_invalid_messages(pts, ees, pto, eeo, res)
        for j, i in enumerate(idx):
            c = res["certs"][j]
            if c["status"] == 2 and c["reason_code"] == CERTIFICATE_REASON_INVALID_INPUT:
                out[i] = ValueError(invalid_msg.get(j, "primitive failed validation"))
                continue
            q = queries[i]
            r = _base_certificate(q.work_item, q.config)
            r.status = CertificateStatus(int(c["status"]))
            r.toi_upper = float(c["toi_upper"])
            r.safe_margin_lb = float(c["safe_margin_lb"])
            r.witness_family = int(c["witness_family"])
            r.witness_id_a = int(c["witness_id_a"])
            r.witness_id_b = int(c["witness_id_b"])
            r.covered_feature_mask = int(c["covered_feature_mask"])
            r.reason_code = int(c["reason_code"])
            r.next_refinement_mode = CertificateRefinementMode(int(c["next_refinement_mode"]))
            out[i] = r
    return out


def _first_invalid_messages(pts, ees, pto, eeo, res) -> dict:
    """Reference message of the first invalid primitive of each failed query."""
    msgs = {}
    for j in range(len(pto) - 1):
        for fam, lst, off, results in ((1, pts, pto, res["pt_results"]), (2, ees, eeo, res["ee_results"])):
            if j in msgs:
                break
            for k in range(off[j], off[j + 1]):
                if results[k]["reason_code"] == CERTIFICATE_REASON_INVALID_INPUT:
                    p = lst[k]
                    a, b = (p.point_id, p.triangle_id) if fam == 1 else (p.edge_a_id, p.edge_b_id)
                    kind = "point-triangle" if fam == 1 else "edge-edge"
                    msgs[j] = (f"{kind} primitive ids are required" if a < 0 or b < 0
                               else f"{kind} primitive trajectories must be finite")
                    break
    return msgs


def evaluate_certificate_query_cpu(query: ExactCertificateQuery) -> CertificateResult:
    _validate_config(query.config)
    validate_exact_work_item(query.work_item)
    r = _certify_queries([query])[0]
    if isinstance(r, Exception):
        raise r
    return r


class CertificateEngine:
    def evaluate_work_item(self, work_item: ExactWorkItem) -> CertificateResult:  # :722-727
        return _base_certificate(work_item, CertificateEngineConfig())

    def evaluate_query(self, query: ExactCertificateQuery) -> CertificateResult:
        return evaluate_certificate_query_cpu(query)


def process_exact_work_queue_cpu(work_queue: Sequence[ExactCertificateQuery],
                                 config: ExactWorkQueueConfig) -> ExactWorkQueueResult:
    """ProcessExactWorkQueueCpu (:593-661): every work item certified in one
    GPU launch per config; the audit log written on the GPU (p2c_audit_rows);
    work item / certificate validation and the coverage guard on the host."""
    from p2cccd_b200 import queue as _queue
    from p2cccd_b200.records import AUDIT_ITEM_DTYPE, QUERY_CERTIFICATE_DTYPE

    if int(config.first_event_id) == 0:
        raise ValueError("ExactWorkQueueConfig.first_event_id must be non-zero")
    if int(config.first_timestamp_us) == 0:
        raise ValueError("ExactWorkQueueConfig.first_timestamp_us must be non-zero")
    queue_list = list(work_queue)
    for q in queue_list:
        validate_exact_work_item(q.work_item)
    certs = _certify_queries(queue_list)
    result = ExactWorkQueueResult()
    items = np.zeros(len(queue_list), AUDIT_ITEM_DTYPE)
    crec = np.zeros(len(queue_list), QUERY_CERTIFICATE_DTYPE)
    for k, (q, c) in enumerate(zip(queue_list, certs)):
        if isinstance(c, Exception):  # MakeInvalidInputCertificate, :426-431
            c = _base_certificate(q.work_item, q.config)
            c.reason_code = CERTIFICATE_REASON_INVALID_INPUT
            c.next_refinement_mode = CertificateRefinementMode.REQUEST_GEOMETRY
            c.safe_margin_lb = 0.0
            c.covered_feature_mask = 0
        validate_certificate_result(c)
        w = q.work_item
        items[k] = (w.query_id, w.parent_candidate_id, w.work_item_id, w.interval_t0, w.interval_t1,
                    w.priority_score, w.feature_family_mask, w.depth)
        r = crec[k]
        r["status"], r["reason_code"] = int(c.status), int(c.reason_code)
        r["toi_upper"], r["safe_margin_lb"] = float(c.toi_upper), float(c.safe_margin_lb)
        r["next_refinement_mode"] = int(c.next_refinement_mode)
        result.certificates.append(c)
    try:
        rows = _queue.audit_rows(items, crec, int(config.first_event_id), int(config.first_timestamp_us),
                                 bool(config.emit_dequeue_events))
    except _queue.AuditRowError as exc:  # the reference's message for the first failing row
        validate_audit_log_row(_audit_row_object(exc.rows[exc.row]))
        raise
    result.audit_log = [_audit_row_object(r) for r in rows]
    result.processed_count = len(queue_list)
    validate_exact_work_queue_coverage(queue_list, result)
    return result


def _audit_row_object(r) -> AuditLogRow:
    row = AuditLogRow()
    for k in ("event_id", "query_id", "candidate_id", "work_item_id", "action", "depth", "timestamp_us"):
        setattr(row, k, int(r[k]))
    row.stage = AuditStage(int(r["stage"]))
    for k in ("interval_t0", "interval_t1", "aux_value0", "aux_value1"):
        setattr(row, k, float(r[k]))
    return row


def validate_exact_work_queue_coverage(work_queue, result) -> bool:  # :553-591
    if result.processed_count != len(work_queue):
        raise ValueError("exact work queue processed_count must match input size")
    if len(result.certificates) != len(work_queue):
        raise ValueError("each exact work item must produce exactly one certificate")
    expected = set()
    for q in work_queue:
        validate_exact_work_item(q.work_item)
        key = (q.work_item.query_id, q.work_item.work_item_id)
        if key in expected:
            raise ValueError("exact work queue contains duplicate work_item_id for a query")
        expected.add(key)
    covered = set()
    for c in result.certificates:
        validate_certificate_result(c)
        key = (c.query_id, c.work_item_id)
        if key not in expected:
            raise ValueError("certificate references a work item that was not queued")
        if key in covered:
            raise ValueError("exact work item produced more than one certificate")
        covered.add(key)
    if len(covered) != len(expected):
        raise ValueError("at least one exact work item disappeared without certificate coverage")
    return True


def generate_conservative_refinement_work_items(parent: ExactWorkItem, certificate: CertificateResult,
                                                config: ExactRefinementConfig) -> list:  # :663-720
    validate_exact_work_item(parent)
    validate_certificate_result(certificate)
    if certificate.work_item_id != parent.work_item_id or certificate.query_id != parent.query_id:
        raise ValueError("certificate must correspond to the parent exact work item")
    if int(config.first_child_work_item_id) == 0:
        raise ValueError("ExactRefinementConfig.first_child_work_item_id must be non-zero")
    if not math.isfinite(config.min_interval_width) or config.min_interval_width <= 0.0:
        raise ValueError("ExactRefinementConfig.min_interval_width must be finite and positive")
    if parent.depth >= config.max_child_depth:
        return []

    def child(wid, t0, t1):
        c = ExactWorkItem()
        for n, _ in ExactWorkItem._fields:
            setattr(c, n, getattr(parent, n))
        c.work_item_id, c.interval_t0, c.interval_t1 = wid, t0, t1
        c.depth = (parent.depth + 1) & 0xFFFF
        c.source = ProposalSource.REFINED
        return c

    if certificate.status == CertificateStatus.COLLISION:
        t0 = parent.interval_t0
        toi = certificate.toi_upper
        t1 = parent.interval_t0 if toi < parent.interval_t0 else (parent.interval_t1 if parent.interval_t1 < toi
                                                                  else toi)
        return [child(config.first_child_work_item_id, t0, t1)] if t1 - t0 > config.min_interval_width else []
    if (certificate.status == CertificateStatus.UNDECIDED
            and certificate.next_refinement_mode == CertificateRefinementMode.BISECT_INTERVAL):
        if parent.interval_t1 - parent.interval_t0 > config.min_interval_width:
            mid = 0.5 * (parent.interval_t0 + parent.interval_t1)
            return [child(config.first_child_work_item_id, parent.interval_t0, mid),
                    child(config.first_child_work_item_id + 1, mid, parent.interval_t1)]
    return []


# ---------------------------------------------------------------------------
# mesh-pair query (cpp/certificate/mesh_exact_query.cpp:143-327)


class BenchmarkRow(_Struct):  # common/runtime_contracts.h (BenchmarkRow), py_module.cpp:1433-1447
    _fields = (("query_count", 0), ("fn_count", 0), ("fp_count", 0), ("candidate_recall", 0.0),
               ("avg_candidates", 0.0), ("avg_exact_evals", 0.0), ("avg_subdivision_depth", 0.0),
               ("fallback_ratio", 0.0), ("rt_ms", 0.0), ("proposal_ms", 0.0), ("exact_ms", 0.0), ("total_ms", 0.0),
               ("qps", 0.0))


def validate_benchmark_row(row) -> bool:  # validators.cpp:317-357
    if int(row.query_count) == 0:
        raise ValueError("BenchmarkRow.query_count is required")
    if int(row.fn_count) > int(row.query_count):
        raise ValueError("BenchmarkRow.fn_count cannot exceed query_count")
    for k in ("candidate_recall", "fallback_ratio"):  # ValidateRatio
        v = float(getattr(row, k))
        if not math.isfinite(v):
            raise ValueError(f"BenchmarkRow.{k} must be finite")
        if not (0.0 <= v <= 1.0):
            raise ValueError(f"BenchmarkRow.{k} must be in [0, 1]")
    for k in ("avg_candidates", "avg_exact_evals", "avg_subdivision_depth", "rt_ms", "proposal_ms", "exact_ms",
              "total_ms", "qps"):  # RequireNonNegative
        v = float(getattr(row, k))
        if not math.isfinite(v):
            raise ValueError(f"BenchmarkRow.{k} must be finite")
        if not v >= 0.0:
            raise ValueError(f"BenchmarkRow.{k} must be non-negative")
    return True


def validate_candidate_record(record) -> bool:  # validators.cpp:160-181, py_module.cpp:488-491
    from p2cccd_b200.schedule import candidate_record_error

    msg = candidate_record_error(_candidate_array([record])[0])
    if msg:
        raise ValueError(msg)
    return True


# ---- triangle meshes (geometry/mesh_io.cpp) --------------------------------

def _area2(v, t) -> float:  # TriangleAreaSquared (:113-119): 0.25 * |e0 x e1|^2, the reference's op order
    a, b, c = v[t[0]], v[t[1]], v[t[2]]
    e0 = (b[0] - a[0], b[1] - a[1], b[2] - a[2])
    e1 = (c[0] - a[0], c[1] - a[1], c[2] - a[2])
    x = (e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0])
    return 0.25 * (x[0] * x[0] + x[1] * x[1] + x[2] * x[2])


def validate_triangle_mesh(mesh) -> bool:  # ValidateTriangleMesh, mesh_io.cpp:306-340
    v, t, p = list(mesh.vertices_ref), list(mesh.triangles), list(mesh.patch_ids)
    if not v:
        raise ValueError("mesh has no vertices")
    if not t:
        raise ValueError("mesh has no triangles")
    if p and len(p) != len(t):
        raise ValueError("mesh patch_ids must be empty or match triangle count")
    for vert in v:
        if not all(math.isfinite(float(x)) for x in vert):
            raise ValueError("mesh vertex contains a non-finite coordinate")
    vf = [tuple(float(x) for x in vert) for vert in v]
    for tri in t:
        i = [int(x) for x in tri]
        if i[0] == i[1] or i[0] == i[2] or i[1] == i[2]:
            raise ValueError("mesh triangle contains duplicate vertex indices")
        if any(x >= len(v) for x in i):
            raise ValueError("mesh triangle references a vertex outside the vertex array")
        if _area2(vf, i) <= 0.0:
            raise ValueError("mesh triangle has zero area")
    return True


def center_mesh_at_aabb_center(mesh) -> tuple:  # CenterMeshAtAabbCenter, mesh_io.cpp:423-456
    validate_triangle_mesh(mesh)
    v = [tuple(float(x) for x in vert) for vert in mesh.vertices_ref]
    lo, hi = list(v[0]), list(v[0])
    for vert in v:
        for a in range(3):
            lo[a] = vert[a] if vert[a] < lo[a] else lo[a]  # std::min
            hi[a] = vert[a] if hi[a] < vert[a] else hi[a]  # std::max
    center = [0.5 * (lo[a] + hi[a]) for a in range(3)]
    out = Mesh()
    out.vertices_ref = [[vert[0] - center[0], vert[1] - center[1], vert[2] - center[2]] for vert in v]
    out.triangles = [list(t) for t in mesh.triangles]
    out.patch_ids = list(mesh.patch_ids)
    return out, center


def _obj_index(token: str, count: int) -> int:  # ParseObjVertexIndex, :52-91
    text = token.split("/", 1)[0]
    if not text:
        raise ValueError("OBJ face token has empty vertex index")
    body = text[1:] if text[:1] in "+-" else text
    if not body or not body.isdigit():
        if not body or not body[:1].isdigit():
            raise ValueError("OBJ face token has invalid vertex index")
        raise ValueError("OBJ vertex index must be a non-zero integer")
    k = int(text)
    if abs(k) > (1 << 63) - 1:  # std::stoll's range
        raise ValueError("OBJ face token has invalid vertex index")
    if k == 0:
        raise ValueError("OBJ vertex index must be a non-zero integer")
    z = k - 1 if k > 0 else count + k
    if z < 0 or z >= count:
        raise ValueError("OBJ face references a vertex outside the loaded vertex range")
    return z


def _load_obj(path: str) -> Mesh:  # LoadTriangleMeshObj, :342-409 (default options: triangulate, one patch)
    import re

    num = re.compile(r"^[+-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?")  # what operator>> reads as a double
    m = Mesh()
    try:
        text = open(path, encoding="utf-8", errors="replace").read().splitlines()
    except OSError:
        raise ValueError("failed to open OBJ file: " + str(path)) from None
    for ln, line in enumerate(text, 1):
        toks = line.split("#", 1)[0].split()
        if not toks:
            continue
        if toks[0] == "v":
            vals = []
            for tok in toks[1:4]:  # operator>> reads the leading number of each token
                mm = num.match(tok)
                if not mm:
                    break
                vals.append(float(mm.group(0)))
                if mm.end() != len(tok):
                    break
            if len(vals) < 3:
                raise ValueError(f"invalid OBJ vertex at line {ln}")
            m.vertices_ref.append(vals)
        elif toks[0] == "f":
            try:
                face = [_obj_index(tok, len(m.vertices_ref)) for tok in toks[1:]]
                if len(face) < 3:
                    raise ValueError("OBJ face must have at least 3 vertices")
                for i in range(1, len(face) - 1):  # AddFaceTriangles (:121-140): a fan from the first vertex
                    if face[0] == face[i] or face[0] == face[i + 1] or face[i] == face[i + 1]:
                        raise ValueError("OBJ face creates a degenerate triangle with duplicate indices")
                    m.triangles.append([face[0], face[i], face[i + 1]])
                    m.patch_ids.append(0)
            except ValueError as e:
                raise ValueError(f"{e} at line {ln}") from None
    validate_triangle_mesh(m)
    return m


def _dedup_vertices(xyz: np.ndarray) -> tuple:
    """AddOrGetVertexIndex (:164-188): float vertices numbered in first-seen
    order, equal floats (+0 and -0 alike) sharing one index."""
    key = np.where(xyz == 0, np.float32(0.0), xyz).view(np.uint32)  # +0 and -0 compare equal
    flat = key.reshape(-1, 3)
    _, first, inv = np.unique(flat, axis=0, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")
    rank = np.empty(len(order), np.int64)
    rank[order] = np.arange(len(order))
    idx = rank[inv.reshape(-1)]
    verts = xyz.reshape(-1, 3)[np.sort(first)].astype(np.float64)
    return verts, idx


def _stl_mesh(xyz: np.ndarray) -> Mesh:
    verts, idx = _dedup_vertices(xyz.astype(np.float32))
    tri = idx.reshape(-1, 3)
    keep = (tri[:, 0] != tri[:, 1]) & (tri[:, 0] != tri[:, 2]) & (tri[:, 1] != tri[:, 2])
    m = Mesh()
    m.vertices_ref = verts.tolist()
    m.triangles = tri[keep].tolist()
    validate_triangle_mesh(m)
    return m


def _load_stl(path: str) -> Mesh:  # LooksLikeBinaryStl + the binary / ASCII loaders, :142-300
    import os

    try:
        size = os.path.getsize(path)
        raw = open(path, "rb").read()
    except OSError:
        raise ValueError("failed to open STL file: " + str(path)) from None
    if size >= 84 and 84 + int(np.frombuffer(raw[80:84], "<u4")[0]) * 50 == size:
        n = int(np.frombuffer(raw[80:84], "<u4")[0])
        rec = np.frombuffer(raw[84:], dtype=np.dtype([("f", "<f4", (12,)), ("a", "<u2")]), count=n)
        return _stl_mesh(rec["f"][:, 3:12].reshape(-1, 3))
    rows = []
    for line in raw.decode("utf-8", errors="replace").splitlines():
        toks = line.split()
        if not toks or toks[0] not in ("vertex", "VERTEX"):
            continue
        try:
            rows.append([np.float32(t) for t in toks[1:4]])
        except ValueError:
            raise ValueError("invalid ASCII STL vertex row in " + str(path)) from None
        if len(rows[-1]) < 3:
            raise ValueError("invalid ASCII STL vertex row in " + str(path))
    if len(rows) % 3:
        raise ValueError("ASCII STL ended with a partial triangle")
    return _stl_mesh(np.array(rows, np.float32).reshape(-1, 3))


def load_triangle_mesh(path) -> Mesh:  # LoadTriangleMesh, mesh_io.cpp:411-421
    """OBJ (fan-triangulated polygons, one patch) or STL (binary or ASCII,
    float vertices merged by value) into a Mesh, validated."""
    import os

    ext = os.path.splitext(str(path))[1]
    if ext in (".obj", ".OBJ"):
        return _load_obj(str(path))
    if ext in (".stl", ".STL"):
        return _load_stl(str(path))
    raise ValueError("unsupported triangle mesh format: " + ext)


def _mesh_arrays(mesh: Mesh):
    v = np.asarray(mesh.vertices_ref, dtype=np.float64).reshape(-1, 3)
    f = np.asarray(mesh.triangles, dtype=np.int64).reshape(-1, 3)
    if not np.isfinite(v).all():
        raise ValueError("mesh vertices must be finite")
    if len(f) and (f.min() < 0 or f.max() >= len(v)):
        raise ValueError("mesh triangle index out of range")
    return v, f


def build_mesh_exact_certificate_query(mesh_a, translation_a_t0, translation_a_t1, mesh_b, translation_b_t0,
                                       translation_b_t1, work_item, config, build_config) -> MeshExactBuildResult:
    """Candidate primitives of a translating mesh pair, found by the GPU
    sweep-and-prune instead of the reference's O(V*F + E^2) loops; the list,
    ids, order and statistics equal BuildMeshExactCertificateQuery's."""
    import torch

    from p2cccd_b200 import scenes
    from p2cccd_b200.scene import ScenePipeline

    va, fa = _mesh_arrays(mesh_a)
    vb, fb = _mesh_arrays(mesh_b)
    validate_exact_work_item(work_item)
    if int(build_config.max_point_triangle_primitives) >= 2 ** 64 - 1:
        raise ValueError("max_point_triangle_primitives must be smaller than uint64 max")
    if int(build_config.max_edge_edge_primitives) >= 2 ** 64 - 1:
        raise ValueError("max_edge_edge_primitives must be smaller than uint64 max")
    ta0, ta1, tb0, tb1 = (np.asarray(_vec3(t)) for t in (translation_a_t0, translation_a_t1, translation_b_t0,
                                                         translation_b_t1))
    ea, eb = scenes.unique_edges(fa.astype(np.int32)), scenes.unique_edges(fb.astype(np.int32))
    scene = scenes.combine([(va + ta0, va + ta1, fa.astype(np.int32), ea), (vb + tb0, vb + tb1,
                                                                            fb.astype(np.int32), eb)])
    mask = int(work_item.feature_family_mask)
    st = MeshExactBuildStats()
    st.vertex_count_a, st.vertex_count_b = len(va), len(vb)
    st.triangle_count_a, st.triangle_count_b = len(fa), len(fb)
    st.edge_count_a, st.edge_count_b = len(ea), len(eb)
    if build_config.prune_by_swept_aabb:
        dev = torch.device("cuda", torch.cuda.current_device())
        pipe = ScenePipeline(scene, dev, exclude_self=True, config=_config(config), family_mask=3)
        pipe.step_checked()
        vf_rec, ee_rec = pipe.materialize()
    else:  # every pair, no box test
        nva, nfa, nea = len(va), len(fa), len(ea)
        ab = np.stack(np.meshgrid(np.arange(nva), np.arange(len(fb)) + nfa, indexing="ij"), -1).reshape(-1, 2)
        ba = np.stack(np.meshgrid(np.arange(len(vb)) + nva, np.arange(nfa), indexing="ij"), -1).reshape(-1, 2)
        vf_pairs = np.concatenate([ab, ba])
        ee_pairs = np.stack(np.meshgrid(np.arange(nea), np.arange(len(eb)) + nea, indexing="ij"), -1).reshape(-1, 2)
        vf_rec = _materialize_host(scene, vf_pairs, 1)
        ee_rec = _materialize_host(scene, ee_pairs, 2)
    # the reference's trajectory feature ids (mesh_exact_query.cpp:244-258,
    # 282-289, 302-313): B-triangle vertices carry triangle_offset_b + the B
    # vertex index, A-side ids are plain A indices, B points and B edge
    # vertices carry vertex_offset_b + index
    nva, nfa = len(va), len(fa)
    if len(vf_rec):
        a_side = vf_rec["point_id"] < nva
        for k in ("triangle_v0", "triangle_v1", "triangle_v2"):
            fid = vf_rec[k]["feature_id"]
            vf_rec[k]["feature_id"] = np.where(a_side, fid - nva + nfa, fid)
    result = MeshExactBuildResult()
    result.query.work_item = work_item
    result.query.config = config
    if mask & 1:
        st.point_triangle_total_pairs = len(va) * len(fb) + len(vb) * len(fa)
        st.point_triangle_kept_pairs = len(vf_rec)
        st.point_triangle_pruned_pairs = st.point_triangle_total_pairs - len(vf_rec)
        if build_config.max_point_triangle_primitives > 0 and len(vf_rec) > build_config.max_point_triangle_primitives:
            raise ValueError("point-triangle primitive budget exceeded")
        result.query.point_triangle_primitives = _from_records(vf_rec, 1)
    if mask & 2:
        st.edge_edge_total_pairs = len(ea) * len(eb)
        st.edge_edge_kept_pairs = len(ee_rec)
        st.edge_edge_pruned_pairs = st.edge_edge_total_pairs - len(ee_rec)
        if build_config.max_edge_edge_primitives > 0 and len(ee_rec) > build_config.max_edge_edge_primitives:
            raise ValueError("edge-edge primitive budget exceeded")
        result.query.edge_edge_primitives = _from_records(ee_rec, 2)
    result.stats = st
    return result


def _materialize_host(scene: dict, pairs: np.ndarray, family: int) -> np.ndarray:
    n = len(pairs)
    dt = _rec.POINT_TRIANGLE_DTYPE if family == 1 else _rec.EDGE_EDGE_DTYPE
    rec = np.zeros(n, dtype=dt)
    if n == 0:
        return rec
    a, b = pairs[:, 0], pairs[:, 1]
    if family == 1:
        verts = np.stack([a, *scene["faces"][b].T], 1)
    else:
        verts = np.concatenate([scene["edges"][a], scene["edges"][b]], 1)
    names = dt.names
    rec[names[0]], rec[names[1]] = a, b
    for k in range(4):
        rec[names[2 + k]]["feature_id"] = verts[:, k]
        rec[names[2 + k]]["position_t0"] = scene["v_t0"][verts[:, k]]
        rec[names[2 + k]]["position_t1"] = scene["v_t1"][verts[:, k]]
    return rec


# ---------------------------------------------------------------------------
# proxy scenes: patch-level candidates (rt_candidate/, py_module.cpp:1541-1650,
# 1863-1882).  Raw hits and compaction run on the GPU (p2c_proxy_candidates).


class Aabb(_Struct):
    _fields = (("min", lambda: [0.0, 0.0, 0.0]), ("max", lambda: [0.0, 0.0, 0.0]))


class PatchMotionBound(_Struct):
    _fields = (("patch_id", 0), ("t0", 0.0), ("t1", 1.0), ("center_t0", lambda: [0.0, 0.0, 0.0]),
               ("center_t1", lambda: [0.0, 0.0, 0.0]), ("translation_bound", 0.0), ("rotation_angle", 0.0),
               ("center_rotation_bound", 0.0), ("surface_rotation_bound", 0.0), ("radial_motion_bound", 0.0),
               ("conservative_radius", 0.0))


class CapsuleProxy(_Struct):
    _fields = (("patch_id", 0), ("endpoint0", lambda: [0.0, 0.0, 0.0]), ("endpoint1", lambda: [0.0, 0.0, 0.0]),
               ("radius", 0.0), ("motion_bound", PatchMotionBound))


class ProxyPrimitive(_Struct):  # rt_candidate/proxy_scene.h:29-41
    _fields = (("proxy_id", 0), ("object_id", 0), ("patch_id", 0), ("slab_id", 0), ("motion_segment_id", 0),
               ("proxy_type", ProxyType.UNKNOWN), ("t0", 0.0), ("t1", 1.0), ("bounds", Aabb),
               ("capsule", CapsuleProxy), ("motion_bound", PatchMotionBound))


class ProxyScene(_Struct):  # :43-46
    _fields = (("query_id", 0), ("primitives", list))


class RawCandidateHit(_Struct):  # rt_candidate/candidate_buffer.h
    _fields = (("query_id", 0), ("pair_key", 0), ("proxy_a_index", 0), ("proxy_b_index", 0), ("slab_id", 0),
               ("rt_hit_count", 0), ("flags", 0), ("motion_bound", lambda: [0.0, 0.0, 0.0, 0.0]))


class RawCandidateBuffer(_Struct):
    _fields = (("hits", list),)


class CandidateRecord(_Struct):  # common/runtime_contracts.h:41-56
    _fields = (("schema_version", 1), ("candidate_id", 0), ("query_id", 0), ("slab_id", 0), ("object_a_id", 0),
               ("patch_a_id", 0), ("object_b_id", 0), ("patch_b_id", 0), ("proxy_type_a", ProxyType.UNKNOWN),
               ("proxy_type_b", ProxyType.UNKNOWN), ("rt_hit_count", 0),
               ("motion_bound", lambda: [0.0, 0.0, 0.0, 0.0]), ("proxy_features_offset", 0), ("flags", 0))


class RtCandidateTiming(_Struct):  # rt_candidate/candidate_generation_result.h:12-19
    _fields = (("build_ms", 0.0), ("update_ms", 0.0), ("trace_ms", 0.0), ("compact_ms", 0.0), ("stats_ms", 0.0),
               ("total_ms", 0.0))


class CandidateDensityStats(_Struct):  # :21-37
    _fields = (("schema_version", 1), ("query_id", 0), ("proxy_count", 0), ("object_count", 0), ("slab_count", 0),
               ("cross_object_same_slab_pair_count", 0), ("raw_hit_count", 0), ("compact_candidate_count", 0),
               ("raw_hits_per_proxy", 0.0), ("candidates_per_proxy", 0.0), ("candidates_per_slab", 0.0),
               ("aabb_overlap_ratio", 0.0), ("avg_rt_hits_per_candidate", 0.0), ("timing", RtCandidateTiming),
               ("backend_name", ""))


class CandidateGenerationResult(_Struct):  # :39-45
    _fields = (("backend_name", ""), ("raw_buffer", RawCandidateBuffer), ("candidates", list),
               ("timing", RtCandidateTiming), ("density", CandidateDensityStats))


def _time_tolerance(t0: float, t1: float) -> float:  # proxy_scene.cpp:41-43
    return 1.0e-12 * max(1.0, abs(t0), abs(t1), abs(t1 - t0))


def _proxy_arrays(scene) -> dict:
    """The primitive list of a ProxyScene (or the equivalent dict of arrays)
    as the column arrays p2c_proxy_candidates reads."""
    if isinstance(scene, dict):
        return scene
    prims = scene.primitives
    n = len(prims)
    out = {"query_id": int(scene.query_id), "n": n,
           "object_id": np.fromiter((p.object_id for p in prims), np.uint32, n),
           "patch_id": np.fromiter((p.patch_id for p in prims), np.uint32, n),
           "slab_id": np.fromiter((p.slab_id for p in prims), np.uint32, n),
           "proxy_type": np.fromiter((int(p.proxy_type) for p in prims), np.uint8, n),
           "t0": np.fromiter((p.t0 for p in prims), np.float64, n),
           "t1": np.fromiter((p.t1 for p in prims), np.float64, n),
           "bounds": np.array([[*p.bounds.min, *p.bounds.max] for p in prims], np.float64).reshape(n, 6),
           "motion_bound": np.array([[p.motion_bound.translation_bound, p.motion_bound.rotation_angle,
                                      p.motion_bound.radial_motion_bound, p.motion_bound.conservative_radius]
                                     for p in prims], np.float64).reshape(n, 4)}
    ids = np.fromiter((p.proxy_id for p in prims), np.int64, n)
    if np.any(ids != np.arange(n)):  # proxy_scene.cpp:140-142
        raise ValueError("proxy_id must match primitive array index")
    return out


def _validate_slab_partition(a: dict) -> None:
    """ValidateGlobalSlabPartition (proxy_scene.cpp:58-85): one time interval
    per slab id (within TimeTolerance of the first proxy's), and the slab
    intervals, ordered by start then id, do not overlap."""
    slab, t0, t1 = np.asarray(a["slab_id"]), np.asarray(a["t0"]), np.asarray(a["t1"])
    if len(slab) == 0:
        return
    ids, first = np.unique(slab, return_index=True)
    ft0, ft1 = t0[first], t1[first]
    k = np.searchsorted(ids, slab)
    tol = 1.0e-12 * np.maximum.reduce([np.ones_like(ft0), np.abs(ft0), np.abs(ft1), np.abs(ft1 - ft0)])
    if np.any(np.abs(ft0[k] - t0) > tol[k]) or np.any(np.abs(ft1[k] - t1) > tol[k]):
        raise ValueError("proxy scene slab_id must map to one global time interval")
    order = np.lexsort((ids, ft0))
    s0, s1, st = ft0[order], ft1[order], tol[order]
    for i in range(1, len(order)):
        t = max(st[i - 1], st[i])
        if s0[i - 1] < s1[i] - t and s0[i] < s1[i - 1] - t:
            raise ValueError("proxy scene global slab intervals must not overlap")


def _validate_proxies(a: dict) -> None:
    """ValidateProxyScene's per-proxy checks (proxy_scene.cpp:143-151) for the
    host-side validator; the device repeats them while generating."""
    if int(a["query_id"]) == 0:
        raise ValueError("ProxyScene.query_id is required")
    typ, t0, t1, b = (np.asarray(a[k]) for k in ("proxy_type", "t0", "t1", "bounds"))
    if np.any((typ != 1) & (typ != 2)):
        raise ValueError("proxy primitive has an unsupported proxy type")
    if not (np.all(np.isfinite(t0)) and np.all(np.isfinite(t1)) and np.all(t0 < t1)):
        raise ValueError("proxy primitive must satisfy finite t0 < t1")
    b = b.reshape(-1, 6)
    if not np.all(np.isfinite(b)):
        raise ValueError("proxy bounds contain a non-finite value")
    if np.any(b[:, :3] > b[:, 3:]):
        raise ValueError("proxy bounds min cannot exceed max")


def validate_proxy_scene(scene) -> bool:  # py_module.cpp:1314-1317
    a = _proxy_arrays(scene)
    _validate_proxies(a)
    _validate_slab_partition(a)
    return True


def _run_proxy(scene, query_id: int, raw_only: bool):
    from p2cccd_b200.proxy import ProxyCandidates

    a = _proxy_arrays(scene)
    if query_id == 0:
        raise ValueError("query_id is required")
    _validate_slab_partition(a)
    if int(a["query_id"]) == 0:
        raise ValueError("ProxyScene.query_id is required")
    if query_id != int(a["query_id"]):
        raise ValueError("query_id must match ProxyScene.query_id")
    return a, ProxyCandidates(a).run_checked(raw_only=raw_only)


def _raw_objects(raw: np.ndarray) -> RawCandidateBuffer:
    buf = RawCandidateBuffer()
    for r in raw:
        h = RawCandidateHit()
        h.query_id, h.pair_key = int(r["query_id"]), int(r["pair_key"])
        h.proxy_a_index, h.proxy_b_index = int(r["proxy_a_index"]), int(r["proxy_b_index"])
        h.slab_id, h.rt_hit_count, h.flags = int(r["slab_id"]), int(r["rt_hit_count"]), int(r["flags"])
        h.motion_bound = [float(x) for x in r["motion_bound"]]
        buf.hits.append(h)
    return buf


def _candidate_objects(cand: np.ndarray) -> list:
    out = []
    for r in cand:
        c = CandidateRecord()
        for k in ("schema_version", "candidate_id", "query_id", "slab_id", "object_a_id", "patch_a_id",
                  "object_b_id", "patch_b_id", "rt_hit_count", "proxy_features_offset", "flags"):
            setattr(c, k, int(r[k]))
        c.proxy_type_a, c.proxy_type_b = ProxyType(int(r["proxy_type_a"])), ProxyType(int(r["proxy_type_b"]))
        c.motion_bound = [float(x) for x in r["motion_bound"]]
        out.append(c)
    return out


def _density(a: dict, raw: np.ndarray, cand: np.ndarray, timing: RtCandidateTiming,
             backend: str) -> CandidateDensityStats:
    """ComputeCandidateDensityStats (candidate_stats.cpp:128-170); the pair
    count of CountCrossObjectSameSlabPairs (:31-43) in closed form: pairs in
    one slab minus pairs in one (slab, object)."""
    def ratio(x, y):
        return float(x) / float(y) if y else 0.0

    slab, obj = np.asarray(a["slab_id"], np.int64), np.asarray(a["object_id"], np.int64)
    _, per_slab = np.unique(slab, return_counts=True)
    _, per_so = np.unique(np.stack([slab, obj], 1), axis=0, return_counts=True) if len(slab) else (None, per_slab)
    d = CandidateDensityStats()
    d.query_id, d.proxy_count = int(a["query_id"]), int(a["n"])
    d.object_count, d.slab_count = len(np.unique(obj)), len(per_slab)
    d.cross_object_same_slab_pair_count = int((per_slab * (per_slab - 1) // 2).sum() -
                                              (per_so * (per_so - 1) // 2).sum())
    d.raw_hit_count, d.compact_candidate_count = len(raw), len(cand)
    d.raw_hits_per_proxy = ratio(d.raw_hit_count, d.proxy_count)
    d.candidates_per_proxy = ratio(d.compact_candidate_count, d.proxy_count)
    d.candidates_per_slab = ratio(d.compact_candidate_count, d.slab_count)
    d.aabb_overlap_ratio = ratio(d.raw_hit_count, d.cross_object_same_slab_pair_count)
    d.avg_rt_hits_per_candidate = ratio(int(cand["rt_hit_count"].sum()) if len(cand) else 0,
                                        d.compact_candidate_count)
    d.timing, d.backend_name = timing, backend
    return d


def generate_raw_candidates_cpu(scene, query_id: int = 0) -> RawCandidateBuffer:  # py_module.cpp:366-371
    query_id = int(query_id) or int(_proxy_arrays(scene)["query_id"])
    _, (raw, _cand) = _run_proxy(scene, query_id, raw_only=True)
    return _raw_objects(raw)


RAW_CANDIDATE_VALID = 1  # RawCandidateFlags (rt_candidate/candidate_buffer.h:14-17)
RAW_CANDIDATE_AABB_OVERLAP = 2


class CandidateBackend(enum.IntEnum):  # rt_candidate/candidate_generator.h:13-16
    CPU_REFERENCE = 0
    OPTIX = 1


class CandidateGeneratorConfig(_Struct):  # :18-21
    _fields = (("backend", CandidateBackend.CPU_REFERENCE), ("allow_optix_cpu_fallback", False))


class CandidateGenerator:  # :23-38, py_module.cpp:1821-1829
    """The candidate generator of a backend config; both backends run the
    device proxy path (OptiX as the reference built without it)."""

    def __init__(self, config: CandidateGeneratorConfig | None = None):
        self.config = config if config is not None else CandidateGeneratorConfig()

    def trace_candidates_for_proxy_scene(self, scene, query_id: int = 0) -> list:
        """TraceCandidates (candidate_generator.cpp:40-47): the candidates, or
        an empty list where generation fails."""
        name = "optix" if CandidateBackend(self.config.backend) == CandidateBackend.OPTIX else "cpu_reference"
        try:
            return generate_candidates_for_proxy_scene(scene, query_id, name,
                                                       bool(self.config.allow_optix_cpu_fallback)).candidates
        except ValueError:
            return []


class ObjLoadOptions(_Struct):  # geometry/mesh_io.h:10-13
    _fields = (("triangulate_polygon_faces", True), ("use_object_groups_as_patch_ids", False))


def _raw_array(raw_buffer) -> np.ndarray:
    """RawCandidateBuffer (or its hits, or RAW_HIT_DTYPE records) as records."""
    from p2cccd_b200.records import RAW_HIT_DTYPE

    if isinstance(raw_buffer, np.ndarray):
        return np.ascontiguousarray(raw_buffer, dtype=RAW_HIT_DTYPE)
    hits = raw_buffer.hits if hasattr(raw_buffer, "hits") else raw_buffer
    out = np.zeros(len(hits), RAW_HIT_DTYPE)
    for r, h in zip(out, hits):
        for k in ("query_id", "pair_key", "proxy_a_index", "proxy_b_index", "slab_id", "rt_hit_count", "flags"):
            r[k] = int(getattr(h, k))
        mb = list(h.motion_bound)
        if len(mb) != 4:
            raise ValueError("RawCandidateHit.motion_bound must have length 4")
        r["motion_bound"] = mb
    return out


def compact_raw_candidates(scene, raw_buffer) -> list:  # py_module.cpp:373-379, 1873-1876
    """CompactRawCandidates (rt_candidate/candidate_buffer.cpp:181-227) on the
    GPU for any raw hits of the scene (from generate_raw_candidates_cpu or
    another tracer): ValidateProxyScene, ValidateRawHit on every hit, then the
    compacted CandidateRecords in key order with ids 1, 2, ..."""
    from p2cccd_b200.proxy import ProxyCandidates

    a = _proxy_arrays(scene)
    validate_proxy_scene(a)
    return _candidate_objects(ProxyCandidates(a, raw_capacity=0).compact(_raw_array(raw_buffer)))


def generate_candidates_for_proxy_scene(scene, query_id: int = 0, backend_name: str = "cpu_reference",
                                        allow_optix_cpu_fallback: bool = False) -> CandidateGenerationResult:
    """GenerateCandidatesForProxyScene (py_module.cpp:103-116) through
    CandidateGenerator::GenerateCandidates (candidate_generator.cpp:13-33).
    The cpu_reference backends run the device path under their own name; the
    OptiX backends behave as the reference built without OptiX
    (optix_candidate_tracer.cpp:882-888): an error, or with
    allow_optix_cpu_fallback the same generation named "optix_cpu_fallback"."""
    import time

    name = _backend(backend_name)
    start = time.perf_counter()
    a = _proxy_arrays(scene)
    qid = int(query_id) or int(a["query_id"])
    if qid == 0:
        raise ValueError("query_id is required")
    if qid != int(a["query_id"]):
        raise ValueError("query_id must match ProxyScene.query_id")
    if name == "optix_cpu_fallback" and not allow_optix_cpu_fallback:
        validate_proxy_scene(a)
        raise ValueError("P2CCCD was built without OptiX support; configure with -DP2CCCD_ENABLE_OPTIX=ON")
    timing = RtCandidateTiming()
    t = time.perf_counter()
    a, (raw, cand) = _run_proxy(a, qid, raw_only=False)
    timing.trace_ms = (time.perf_counter() - t) * 1e3  # hits and compaction are one device call
    timing.build_ms = (t - start) * 1e3
    t = time.perf_counter()
    res = CandidateGenerationResult()
    res.backend_name = name
    res.raw_buffer, res.candidates = _raw_objects(raw), _candidate_objects(cand)
    res.density = _density(a, raw, cand, timing, name)
    timing.stats_ms = (time.perf_counter() - t) * 1e3
    timing.total_ms = (time.perf_counter() - start) * 1e3
    res.timing = timing
    return res


class RuntimeQueryIdMapping(_Struct):  # rt_candidate/external_batch_candidate.h
    _fields = (("source_query_id", 0), ("runtime_query_id", 0))


class ExternalBatchCandidateResult(_Struct):  # py_module.cpp:1657-1667
    _fields = (("backend_name", ""), ("timing", RtCandidateTiming), ("primitive_count", 0), ("raw_hit_count", 0),
               ("compact_candidate_count", 0), ("candidate_recall", 0.0), ("candidates", list),
               ("runtime_query_ids", list))


def _vertex_array(v, field: str) -> list:  # ParseVertexArray, py_module.cpp:129-146
    if len(v) != 4:
        raise ValueError(field + " must contain four vertices")
    out = []
    for p in v:
        if len(p) != 3:
            raise ValueError(field + " vertices must be 3D")
        out.append([float(x) for x in p])
    return out


def _external_batch(batch) -> dict:
    """ParseExternalBatchQueries (py_module.cpp:148-181): ``batch.queries``
    items with query_id, source_query_index, family ("vf" / "ee"),
    vertices_t0 / vertices_t1 (4 x 3), ground_truth_collides (None or bool)
    and box_pair (None or two ids).  A dict of column arrays
    (``p2cccd_b200.external.batch_arrays``) passes through."""
    from p2cccd_b200.external import batch_arrays

    if isinstance(batch, dict):
        return batch
    qid, sidx, fam, v0, v1, gt, has, pairs = [], [], [], [], [], [], [], []
    for item in batch.queries:
        qid.append(int(item.query_id))
        sidx.append(int(item.source_query_index))
        f = str(item.family)
        if f not in ("vf", "ee"):
            raise ValueError("unsupported external CCD query family: " + f)
        fam.append(0 if f == "vf" else 1)
        v0.append(_vertex_array(item.vertices_t0, "vertices_t0"))
        v1.append(_vertex_array(item.vertices_t1, "vertices_t1"))
        g = item.ground_truth_collides
        gt.append(-1 if g is None else int(bool(g)))
        bp = item.box_pair
        if bp is None:
            has.append(0)
            pairs.append((0, 0))
        else:
            if len(bp) != 2:
                raise ValueError("box_pair must contain exactly two object ids")
            has.append(1)
            pairs.append((int(bp[0]), int(bp[1])))
    n = len(qid)
    return batch_arrays(np.array(qid, np.uint64), sidx, fam, np.array(v0, np.float64).reshape(n, 4, 3),
                        np.array(v1, np.float64).reshape(n, 4, 3), gt, np.array(pairs, np.uint32).reshape(n, 2), has)


def _backend(backend_name: str) -> str:  # ParseCandidateBackend
    if backend_name in ("cpu_reference", "cpu_reference_rt"):
        return "cpu_reference"
    if backend_name in ("optix", "optix_compatible", "optix_rt"):
        return "optix_cpu_fallback"
    raise ValueError("unsupported candidate backend: " + str(backend_name))


def generate_candidates_for_external_batch(batch, backend_name: str = "cpu_reference",
                                           allow_optix_cpu_fallback: bool = False) -> ExternalBatchCandidateResult:
    """GenerateCandidatesForExternalBatch (external_batch_candidate.cpp:231-339,
    py_module.cpp:183-200): the queries packed into one x-tiled proxy scene,
    its candidates from the device proxy path, translated back to the
    queries.  OptiX backends behave as in a reference built without OptiX."""
    from p2cccd_b200 import external

    name = _backend(backend_name)
    b = _external_batch(batch)
    if name == "optix_cpu_fallback" and not allow_optix_cpu_fallback:
        n = len(b["query_id"])
        if n == 0:
            raise ValueError("external batch candidate generation requires at least one query")
        external._first_error(b)
        raise ValueError("P2CCCD was built without OptiX support; configure with -DP2CCCD_ENABLE_OPTIX=ON")
    return _external_result(b, external.generate(b), name)


def _external_result(b: dict, r: dict, name: str) -> ExternalBatchCandidateResult:
    res = ExternalBatchCandidateResult()
    res.backend_name = name
    res.primitive_count, res.raw_hit_count = r["primitive_count"], r["raw_hit_count"]
    res.compact_candidate_count, res.candidate_recall = r["compact_candidate_count"], r["candidate_recall"]
    res.candidates = _candidate_objects(r["candidates"])
    for s, t in zip(b["query_id"].tolist(), r["runtime_query_ids"].tolist()):
        m = RuntimeQueryIdMapping()
        m.source_query_id, m.runtime_query_id = int(s), int(t)
        res.runtime_query_ids.append(m)
    t = res.timing
    t.build_ms, t.trace_ms, t.compact_ms = r["encode_ms"], r["generate_ms"], r["compact_ms"]
    t.total_ms = t.build_ms + t.update_ms + t.trace_ms + t.compact_ms
    return res


class PoseSample(_Struct):  # geometry/motion.h:9-12
    _fields = (("translation", lambda: [0.0, 0.0, 0.0]), ("rotation_xyzw", lambda: [0.0, 0.0, 0.0, 1.0]))


class MotionSegment(_Struct):  # :14-19
    _fields = (("t0", 0.0), ("t1", 1.0), ("pose_t0", PoseSample), ("pose_t1", PoseSample))


class Patch(_Struct):  # geometry/patch.h:9-16
    _fields = (("patch_id", 0), ("triangle_ids", list), ("triangle_count", 0), ("area", 0.0),
               ("local_center", lambda: [0.0, 0.0, 0.0]), ("radius", 0.0))


class ProxyObjectBuildInput(_Struct):  # rt_candidate/proxy_scene.h:15-22
    _fields = (("object_id", 0), ("proxy_type", ProxyType.SWEPT_AABB), ("patches", list), ("motion_segments", list),
               ("slabs_per_motion_segment", 1), ("eps_proxy", 0.0))


class ProxySceneBuildInput(_Struct):  # :24-27
    _fields = (("query_id", 0), ("objects", list))


def _build_input_arrays(inp) -> dict:
    """A ProxySceneBuildInput as the arrays p2c_proxy_scene_build reads."""
    if isinstance(inp, dict):
        return inp
    objs = []
    for o in inp.objects:
        segs = np.array([[s.t0, s.t1, *s.pose_t0.translation, *s.pose_t0.rotation_xyzw, *s.pose_t1.translation,
                          *s.pose_t1.rotation_xyzw] for s in o.motion_segments], np.float64).reshape(-1, 16)
        objs.append({"object_id": int(o.object_id), "proxy_type": int(o.proxy_type),
                     "slabs_per_motion_segment": int(o.slabs_per_motion_segment), "eps_proxy": float(o.eps_proxy),
                     "patch_id": np.array([p.patch_id for p in o.patches], np.uint32),
                     "local_center": np.array([list(p.local_center) for p in o.patches], np.float64).reshape(-1, 3),
                     "radius": np.array([p.radius for p in o.patches], np.float64), "segments": segs})
    return {"query_id": int(inp.query_id), "objects": objs}


def build_proxy_scene(input) -> ProxyScene:  # py_module.cpp:1868, proxy_scene.cpp:156-213
    """BuildProxyScene on the device (p2c_proxy_scene_build): one proxy per
    object, motion segment, slab and patch, with its motion bound, bounds and
    (capsules) capsule; ValueError with the reference's message on an invalid
    input."""
    from p2cccd_b200.proxy import ProxySceneBuild

    a = _build_input_arrays(input)
    if int(a["query_id"]) == 0:
        raise ValueError("ProxySceneBuildInput.query_id is required")
    if not a["objects"]:
        raise ValueError("ProxySceneBuildInput.objects is empty")
    b = ProxySceneBuild(a)
    b.run_checked()
    h = b.to_host()
    scene = ProxyScene()
    scene.query_id = int(a["query_id"])
    for i in range(h["n"]):
        p = ProxyPrimitive()
        p.proxy_id, p.object_id, p.patch_id = i, int(h["object_id"][i]), int(h["patch_id"][i])
        p.slab_id, p.motion_segment_id = int(h["slab_id"][i]), int(h["motion_segment_id"][i])
        p.proxy_type, p.t0, p.t1 = ProxyType(int(h["proxy_type"][i])), float(h["t0"][i]), float(h["t1"][i])
        p.bounds.min, p.bounds.max = h["bounds"][i, :3].tolist(), h["bounds"][i, 3:].tolist()
        m, det = p.motion_bound, h["motion_detail"][i].tolist()
        m.patch_id, m.t0, m.t1 = p.patch_id, p.t0, p.t1
        m.center_t0, m.center_t1 = det[0:3], det[3:6]
        m.translation_bound, m.rotation_angle, m.radial_motion_bound, m.conservative_radius = \
            h["motion_bound"][i].tolist()
        m.center_rotation_bound, m.surface_rotation_bound = det[6], det[7]
        if p.proxy_type == ProxyType.CAPSULE:
            c = p.capsule
            c.patch_id, c.endpoint0, c.endpoint1 = p.patch_id, list(m.center_t0), list(m.center_t1)
            c.radius = float(h["capsule_radius"][i])
            c.motion_bound = m
        scene.primitives.append(p)
    return scene


# ---------------------------------------------------------------------------
# proposal feature rows (proposal/proposal_features.h:27-43, py_module.cpp:639-753, 1895-1908)


class ProposalFeatureRow(_Struct):
    _fields = (("schema_version", 1), ("query_id", 0), ("candidate_id", 0), ("slab_id", 0), ("object_a_id", 0),
               ("patch_a_id", 0), ("object_b_id", 0), ("patch_b_id", 0), ("features", lambda: [0.0] * 32),
               ("interval_targets", lambda: [0.0] * 8), ("family_targets", lambda: [0.0] * 8),
               ("priority_target", 0.0), ("cost_target", 0.0), ("uncertainty_target", 0.0), ("target_mask", 0))


def _candidate_array(candidates) -> np.ndarray:
    """CandidateRecord objects (or records) as CANDIDATE_RECORD_DTYPE records."""
    from p2cccd_b200.records import CANDIDATE_RECORD_DTYPE

    if isinstance(candidates, np.ndarray):
        return np.ascontiguousarray(candidates, dtype=CANDIDATE_RECORD_DTYPE)
    out = np.zeros(len(candidates), CANDIDATE_RECORD_DTYPE)
    for r, c in zip(out, candidates):
        for k in ("schema_version", "candidate_id", "query_id", "slab_id", "object_a_id", "patch_a_id", "object_b_id",
                  "patch_b_id", "rt_hit_count", "proxy_features_offset", "flags"):
            r[k] = int(getattr(c, k))
        r["proxy_type_a"], r["proxy_type_b"] = int(c.proxy_type_a), int(c.proxy_type_b)
        mb = list(c.motion_bound)
        if len(mb) != 4:
            raise ValueError("CandidateRecord.motion_bound must have length 4")
        r["motion_bound"] = mb
    return out


def _row_objects(rows: np.ndarray) -> list:
    out = []
    for r in rows:
        o = ProposalFeatureRow()
        for k in ("schema_version", "query_id", "candidate_id", "slab_id", "object_a_id", "patch_a_id", "object_b_id",
                  "patch_b_id", "target_mask"):
            setattr(o, k, int(r[k]))
        for k in ("features", "interval_targets", "family_targets"):
            setattr(o, k, [float(x) for x in r[k]])
        o.priority_target, o.cost_target = float(r["priority_target"]), float(r["cost_target"])
        o.uncertainty_target = float(r["uncertainty_target"])
        out.append(o)
    return out


def _runtime_rows(candidates, primitive_count, raw_hit_count, compact_candidate_count, masks) -> np.ndarray:
    from p2cccd_b200.proxy import runtime_feature_rows

    return runtime_feature_rows(_candidate_array(candidates), primitive_count, raw_hit_count,
                                compact_candidate_count, dict(masks or {}))


def build_runtime_proposal_feature_rows(candidates, primitive_count: int, raw_hit_count: int,
                                        compact_candidate_count: int,
                                        conservative_family_masks_by_query_id) -> list:  # py_module.cpp:639-652
    """BuildProposalFeatureRowsFromRuntimeCandidates (proposal_policy.cpp:568-592)
    on the GPU: one ProposalFeatureRow per candidate."""
    return _row_objects(_runtime_rows(candidates, primitive_count, raw_hit_count, compact_candidate_count,
                                      conservative_family_masks_by_query_id))


def build_runtime_proposal_feature_arrays(candidates, primitive_count: int, raw_hit_count: int,
                                          compact_candidate_count: int,
                                          conservative_family_masks_by_query_id) -> dict:  # py_module.cpp:654-753
    """The same rows as a dict of numpy arrays (the reference's keys)."""
    rows = _runtime_rows(candidates, primitive_count, raw_hit_count, compact_candidate_count,
                         conservative_family_masks_by_query_id)
    out = {"schema_version": int(rows["schema_version"][0]) if len(rows) else 1}
    for k in ("query_id", "candidate_id", "slab_id", "object_a_id", "patch_a_id", "object_b_id", "patch_b_id",
              "features", "interval_targets", "family_targets", "priority_target", "cost_target",
              "uncertainty_target", "target_mask"):
        out[k] = np.ascontiguousarray(rows[k])
    return out


def extract_proposal_feature_rows(scene, generation_result) -> list:
    """ExtractProposalFeatureRows (proposal_features.cpp:236-259) on the GPU for a
    ProxyScene and the CandidateGenerationResult of generate_candidates_for_proxy_scene:
    candidates regenerated on the device for the scene (identical to the
    result's; checked), density stats and rows from p2c_proposal_feature_rows."""
    from p2cccd_b200.proxy import ProxyCandidates

    a = _proxy_arrays(scene)
    validate_proxy_scene(a)
    if int(generation_result.density.query_id) != int(a["query_id"]):
        raise ValueError("candidate density query_id must match proxy scene query_id")
    pc = ProxyCandidates(a)
    _, cand = pc.run_checked()
    given = _candidate_array(generation_result.candidates)
    if cand.tobytes() != given.tobytes():
        raise ValueError("generation_result candidates do not belong to this scene")
    _, rows = pc.feature_rows()
    return _row_objects(rows)


# ---------------------------------------------------------------------------
# the runtime exact work queue from proposals (proposal_policy.cpp:595-742, py_module.cpp:1035-1174, 1918-1937)


class ProposalOutput(_Struct):  # runtime_contracts.h:58-65
    _fields = (("candidate_id", 0), ("interval_scores", lambda: [0.0] * 8), ("family_scores", lambda: [0.0] * 8),
               ("priority_score", 0.0), ("cost_score", 0.0), ("uncertainty_score", 0.0))


class ProposalSchedulingConfig(_Struct):  # proposal_policy.h:13-23
    _fields = (("first_work_item_id", 1), ("conservative_feature_family_mask", 3), ("fallback_interval_t0", 0.0),
               ("fallback_interval_t1", 1.0), ("family_score_threshold", 0.5),
               ("uncertainty_fallback_threshold", 0.95), ("ood_abs_feature_threshold", 1.0e5),
               ("preserve_candidate_order", False))


class ProposalScheduleStats(_Struct):  # proposal_policy.h:25-36
    _fields = (("raw_candidate_count", 0), ("proposal_output_count", 0), ("work_item_count", 0),
               ("fallback_count", 0), ("missing_proposal_fallback_count", 0), ("invalid_proposal_fallback_count", 0),
               ("ood_fallback_count", 0), ("high_uncertainty_fallback_count", 0), ("reordered_count", 0),
               ("monotonic_safe", False))


def _row_array(rows) -> np.ndarray:
    from p2cccd_b200.records import FEATURE_ROW_DTYPE

    if isinstance(rows, np.ndarray):
        return np.ascontiguousarray(rows, dtype=FEATURE_ROW_DTYPE)
    out = np.zeros(len(rows), FEATURE_ROW_DTYPE)
    for r, o in zip(out, rows):
        for k in ("schema_version", "query_id", "candidate_id", "slab_id", "object_a_id", "patch_a_id",
                  "object_b_id", "patch_b_id", "priority_target", "cost_target", "uncertainty_target",
                  "target_mask"):
            r[k] = getattr(o, k)
        for k, m in (("features", 32), ("interval_targets", 8), ("family_targets", 8)):
            v = list(getattr(o, k))
            if len(v) != m:
                raise ValueError(f"ProposalFeatureRow.{k} must have length {m}")
            r[k] = v
    return out


def _output_array(outputs) -> np.ndarray:
    from p2cccd_b200.records import PROPOSAL_OUTPUT_DTYPE

    out = np.zeros(len(outputs), PROPOSAL_OUTPUT_DTYPE)
    for r, o in zip(out, outputs):
        r["candidate_id"] = int(o.candidate_id)
        for k in ("interval_scores", "family_scores"):
            v = list(getattr(o, k))
            if len(v) != 8:
                raise ValueError(f"ProposalOutput.{k} must have length 8")
            r[k] = v
        r["priority_score"], r["cost_score"], r["uncertainty_score"] = o.priority_score, o.cost_score, \
            o.uncertainty_score
    return out


def _require(arrays: dict, key: str, shape: tuple, dtype) -> np.ndarray:  # py_module.cpp:756-790
    if key not in arrays:
        raise ValueError(f"missing or invalid array field: {key}")
    a = np.ascontiguousarray(arrays[key], dtype=dtype)
    if a.shape != shape:
        raise ValueError(f"{key} must have shape [{', '.join(str(x) for x in shape)}]")
    return a


def _rows_from_arrays(fa: dict) -> np.ndarray:  # ParseProposalFeatureRowsFromArrays, :792-852
    from p2cccd_b200.records import FEATURE_ROW_DTYPE

    n = len(fa["query_id"])
    out = np.zeros(n, FEATURE_ROW_DTYPE)
    out["schema_version"] = int(fa["schema_version"])
    for k, dt in (("candidate_id", np.uint64), ("query_id", np.uint64), ("slab_id", np.uint32),
                  ("object_a_id", np.uint32), ("patch_a_id", np.uint32), ("object_b_id", np.uint32),
                  ("patch_b_id", np.uint32), ("priority_target", np.float32), ("cost_target", np.float32),
                  ("uncertainty_target", np.float32), ("target_mask", np.uint32)):
        out[k] = _require(fa, k, (n,), dt)
    for k, m in (("features", 32), ("interval_targets", 8), ("family_targets", 8)):
        out[k] = _require(fa, k, (n, m), np.float32)
    return out


def _outputs_from_arrays(fa: dict, pa: dict) -> np.ndarray:  # ParseProposalOutputsFromArrays, :853-890
    from p2cccd_b200.records import PROPOSAL_OUTPUT_DTYPE

    n = len(fa["query_id"])
    out = np.zeros(n, PROPOSAL_OUTPUT_DTYPE)
    out["candidate_id"] = _require(fa, "candidate_id", (n,), np.uint64)
    for k in ("interval_scores", "family_scores"):
        out[k] = _require(pa, k, (n, 8), np.float32)
    for k in ("priority_score", "cost_score", "uncertainty_score"):
        out[k] = _require(pa, k, (n,), np.float32)
    return out


def _schedule(cand, rows, outs, masks, config, mode) -> tuple:
    from p2cccd_b200.schedule import schedule_work_items

    cfg = {k: getattr(config, k) for k, _ in ProposalSchedulingConfig._fields}
    items, stats = schedule_work_items(cand, rows, outs, dict(masks or {}), mode, **cfg)
    return _queue_objects(items), _stats_object(stats)


def _queue_objects(items: np.ndarray) -> list:
    queue = []
    for r in items:
        w = ExactWorkItem()
        for k in ("work_item_id", "parent_candidate_id", "query_id", "slab_id", "patch_a_id", "patch_b_id",
                  "feature_family_mask", "topk_feature_ids_offset", "depth"):
            setattr(w, k, int(r[k]))
        w.interval_t0, w.interval_t1 = float(r["interval_t0"]), float(r["interval_t1"])
        w.priority_score = float(r["priority_score"])
        w.source = ProposalSource(int(r["source"]))
        queue.append(w)
    return queue


def _stats_object(stats) -> ProposalScheduleStats:
    st = ProposalScheduleStats()
    for k, _ in ProposalScheduleStats._fields:
        setattr(st, k, bool(stats[k]) if k == "monotonic_safe" else int(stats[k]))
    return st


def _output_objects(outs: np.ndarray) -> list:
    res = []
    for r in outs:
        o = ProposalOutput()
        o.candidate_id = int(r["candidate_id"])
        o.interval_scores = [float(x) for x in r["interval_scores"]]
        o.family_scores = [float(x) for x in r["family_scores"]]
        o.priority_score, o.cost_score = float(r["priority_score"]), float(r["cost_score"])
        o.uncertainty_score = float(r["uncertainty_score"])
        res.append(o)
    return res


class ProposalRuntimeScheduleResult(_Struct):  # proposal_policy.h:38-43
    _fields = (("feature_rows", list), ("proposal_outputs", list), ("work_queue", list),
               ("stats", ProposalScheduleStats))


class ExternalBatchDummyProposalScheduleResult(_Struct):  # py_module.cpp:202-209
    _fields = (("candidate_result", ExternalBatchCandidateResult), ("feature_rows", list),
               ("proposal_outputs", list), ("work_queue", list), ("stats", ProposalScheduleStats),
               ("proposal_elapsed_ms", 0.0))


def _config_dict(config) -> dict:
    config = config if config is not None else ProposalSchedulingConfig()
    return {k: getattr(config, k) for k, _ in ProposalSchedulingConfig._fields}


def run_dummy_runtime_proposal_schedule(candidates, primitive_count: int, raw_hit_count: int,
                                        compact_candidate_count: int, conservative_family_masks_by_query_id,
                                        config=None, materialize_artifacts: bool = True
                                        ) -> ProposalRuntimeScheduleResult:  # py_module.cpp:1009-1033
    """RunDummyProposalScheduleFromRuntimeCandidates on the GPU: the runtime
    feature rows, density-derived dummy proposals and the ordered queue."""
    from p2cccd_b200.schedule import dummy_schedule

    items, stats, rows, outs = dummy_schedule(_candidate_array(candidates), primitive_count, raw_hit_count,
                                              compact_candidate_count, dict(conservative_family_masks_by_query_id or {}),
                                              materialize_artifacts, **_config_dict(config))
    res = ProposalRuntimeScheduleResult()
    res.feature_rows, res.proposal_outputs = _row_objects(rows), _output_objects(outs)
    res.work_queue, res.stats = _queue_objects(items), _stats_object(stats)
    return res


def external_batch_dummy_schedule(b: dict, r: dict, config=None, materialize_artifacts: bool = False) -> tuple:
    """The schedule half of GenerateExternalBatchDummyProposalScheduleOrThrow
    (py_module.cpp:284-360) on the device, for a batch (column arrays) and its
    candidates from ``external.generate``: a mask per runtime query id from
    its query's family (:213-246), then the raw bypass when every candidate
    has its own query and a single-family mask (:248-318), else the dummy
    schedule with the batch's counts (:320-349).  Returns (items, stats,
    rows, outputs)."""
    from p2cccd_b200.schedule import dummy_schedule

    cand = r["candidates"]
    masks = dict(zip(r["runtime_query_ids"].tolist(), np.where(b["family"] == 0, 1, 2).tolist()))
    q = cand["query_id"]
    fam = np.array([masks.get(int(x), 3) for x in q], np.int64) if len(q) else np.zeros(0, np.int64)
    bypass = len(np.unique(q)) == len(q) and bool(np.all((fam != 0) & ((fam & (fam - 1)) == 0)))
    return dummy_schedule(cand, r["primitive_count"], r["raw_hit_count"], r["compact_candidate_count"], masks,
                          materialize_artifacts, bypass=bypass, **_config_dict(config))


def generate_external_batch_dummy_proposal_schedule(batch, backend_name: str = "cpu_reference",
                                                    allow_optix_cpu_fallback: bool = False, config=None,
                                                    materialize_artifacts: bool = False
                                                    ) -> ExternalBatchDummyProposalScheduleResult:
    """GenerateExternalBatchDummyProposalScheduleOrThrow (py_module.cpp:269-361):
    the batch's candidates, then its exact work queue, on the GPU."""
    import time

    from p2cccd_b200 import external

    name = _backend(backend_name)
    b = _external_batch(batch)
    if name == "optix_cpu_fallback" and not allow_optix_cpu_fallback:
        generate_candidates_for_external_batch(b, backend_name, allow_optix_cpu_fallback)  # raises its error
    r = external.generate(b)
    res = ExternalBatchDummyProposalScheduleResult()
    res.candidate_result = _external_result(b, r, name)
    start = time.perf_counter()
    items, stats, rows, outs = external_batch_dummy_schedule(b, r, config, materialize_artifacts)
    res.proposal_elapsed_ms = (time.perf_counter() - start) * 1e3
    res.feature_rows, res.proposal_outputs = _row_objects(rows), _output_objects(outs)
    res.work_queue, res.stats = _queue_objects(items), _stats_object(stats)
    return res


def schedule_runtime_exact_work_items(candidates, rows, proposal_outputs, conservative_family_masks_by_query_id,
                                      config: ProposalSchedulingConfig) -> tuple:  # py_module.cpp:1035-1059
    """ScheduleRuntimeExactWorkItemsFromProposals on the GPU: (work queue, stats)."""
    return _schedule(_candidate_array(candidates), _row_array(rows), _output_array(proposal_outputs),
                     conservative_family_masks_by_query_id, config, 0)


def schedule_runtime_exact_work_items_from_arrays(candidates, feature_arrays, prediction_arrays,
                                                  conservative_family_masks_by_query_id,
                                                  config: ProposalSchedulingConfig) -> tuple:  # :1061-1086
    return _schedule(_candidate_array(candidates), _rows_from_arrays(feature_arrays),
                     _outputs_from_arrays(feature_arrays, prediction_arrays), conservative_family_masks_by_query_id,
                     config, 0)


def schedule_runtime_exact_work_items_from_proposal_arrays(feature_arrays, prediction_arrays,
                                                           conservative_family_masks_by_query_id,
                                                           config: ProposalSchedulingConfig) -> tuple:  # :1088-1174
    rows = _rows_from_arrays(feature_arrays)
    outs = _outputs_from_arrays(feature_arrays, prediction_arrays)
    if len(rows) != len(outs):
        raise ValueError("feature row and proposal output array lengths must match")
    return _schedule(None, rows, outs, conservative_family_masks_by_query_id, config, 1)


# ---------------------------------------------------------------------------
# the candidate-group interface (common/group_scheduler.cpp, py_module.cpp:1179-1311, 1938-1945)

def run_native_dense_group_exact_early_stop(feature_arrays: dict, prediction_arrays: dict,
                                            uncertainty_fallback_threshold: float = 0.75,
                                            representative_attempt_limit: int = 3,
                                            interval_miss_penalty_scale: float = 0.22,
                                            preserve_input_order: bool = False) -> dict:
    """RunNativeDenseGroupExactEarlyStopOrThrow: the label replay of a learned
    group schedule (first hit per query group, uncertainty fallback, interval
    miss penalties) on the GPU; the counts and work totals equal the
    reference's bit for bit."""
    from p2cccd_b200 import dense_groups

    return dense_groups.early_stop(feature_arrays, prediction_arrays, uncertainty_fallback_threshold,
                                   representative_attempt_limit, interval_miss_penalty_scale, preserve_input_order)
