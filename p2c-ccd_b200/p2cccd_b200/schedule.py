"""The runtime exact work queue from proposals on the device
(p2c_schedule_work_items): the learned scheduler's outputs turned into the
ordered ExactWorkItem queue the certifier consumes, with the reference's
fallback rules (ScheduleRuntimeExactWorkItemsFromProposals,
proposal/proposal_policy.cpp:595-742, and the binding's aligned-array form,
bindings/py_module.cpp:1088-1174)."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .certify import _stream_ptr
from .records import (CANDIDATE_RECORD_DTYPE, EXACT_WORK_ITEM_DTYPE, FEATURE_ROW_DTYPE, PROPOSAL_OUTPUT_DTYPE,
                      SCHEDULE_STATS_DTYPE)

DEFAULTS = dict(first_work_item_id=1, conservative_feature_family_mask=3, fallback_interval_t0=0.0,
                fallback_interval_t1=1.0, family_score_threshold=0.5, uncertainty_fallback_threshold=0.95,
                ood_abs_feature_threshold=1.0e5, preserve_candidate_order=False)

# error word bits in the order the reference meets the failures
_ERRORS = ((2, "proposal runtime feature rows contain a zero or duplicate candidate_id"),
           (4, "proposal runtime outputs contain a zero or duplicate candidate_id"),
           (128, "proposal arrays must preserve candidate_id order"),
           (1, "a CandidateRecord fails validation"),
           (16, "a scheduled ExactWorkItem fails validation"),
           (8, "runtime candidates contain duplicate candidate_id"),
           (32, "runtime scheduled work item has no exact feature family enabled"),
           (64, "runtime scheduled work item has unknown exact feature-family bits"))


class SchedulingConfigStruct(ctypes.Structure):
    _fields_ = [("first_work_item_id", ctypes.c_uint64), ("conservative_feature_family_mask", ctypes.c_uint32),
                ("preserve_candidate_order", ctypes.c_uint32), ("fallback_interval_t0", ctypes.c_double),
                ("fallback_interval_t1", ctypes.c_double), ("family_score_threshold", ctypes.c_float),
                ("uncertainty_fallback_threshold", ctypes.c_float), ("ood_abs_feature_threshold", ctypes.c_float),
                ("pad0", ctypes.c_uint32)]


def _dev(a, dtype, d):
    a = np.ascontiguousarray(a, dtype=dtype)
    return torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).to(d) if len(a) else None


def schedule_work_items(candidates, rows, outputs, masks: dict | None = None, mode: int = 0,
                        device: str | torch.device = "cuda", **config) -> tuple[np.ndarray, np.void]:
    """Work items (EXACT_WORK_ITEM_DTYPE) and stats (SCHEDULE_STATS_DTYPE).
    mode 0: candidates with rows / outputs found by candidate id; mode 1: rows
    and outputs paired by position (candidates unused).  ValueError with the
    reference's message on an invalid config or input."""
    lib = _lib.load()
    d = torch.device(device)
    c = dict(DEFAULTS, **config)
    cfg = SchedulingConfigStruct()
    for k, v in c.items():
        setattr(cfg, k, int(v) if k in ("first_work_item_id", "conservative_feature_family_mask",
                                         "preserve_candidate_order") else float(v))
    cand = np.zeros(0, CANDIDATE_RECORD_DTYPE) if candidates is None else np.ascontiguousarray(candidates)
    rows, outputs = np.ascontiguousarray(rows), np.ascontiguousarray(outputs)
    n = len(cand) if mode == 0 else len(rows)
    keys = sorted(int(k) for k in (masks or {}))
    mq = _dev(np.array(keys, np.uint64), np.uint64, d) if keys else None
    mv = _dev(np.array([int(masks[k]) for k in keys], np.uint32), np.uint32, d) if keys else None
    dc, dr, do = _dev(cand, CANDIDATE_RECORD_DTYPE, d), _dev(rows, FEATURE_ROW_DTYPE, d), \
        _dev(outputs, PROPOSAL_OUTPUT_DTYPE, d)
    items = torch.empty((max(n, 1), EXACT_WORK_ITEM_DTYPE.itemsize), dtype=torch.uint8, device=d)
    stats = torch.zeros(SCHEDULE_STATS_DTYPE.itemsize, dtype=torch.uint8, device=d)
    err = torch.zeros(3, dtype=torch.int64, device=d)
    ws = torch.empty(int(lib.p2c_schedule_work_items_workspace_bytes(n, len(rows), len(outputs))),
                     dtype=torch.uint8, device=d)
    ptr = lambda t: t.data_ptr() if t is not None else None
    _lib.check(lib.p2c_schedule_work_items(int(mode), ptr(dc), len(cand), ptr(dr), len(rows), ptr(do), len(outputs),
                                           ptr(mq), ptr(mv), len(keys), ctypes.byref(cfg), items.data_ptr(),
                                           stats.data_ptr(), err.data_ptr(), ws.data_ptr(), ws.numel(),
                                           _stream_ptr(d)))
    e, first_none, first_unknown = (int(x) for x in err.cpu().numpy().view(np.uint64))
    if e & (32 | 64) and not e & (2 | 4 | 128 | 1 | 16 | 8):  # the earlier item decides
        e &= ~(64 if first_none < first_unknown else 32)
    for bit, msg in _ERRORS:
        if e & bit:
            raise ValueError(msg)
    return (items[:n].cpu().numpy().view(EXACT_WORK_ITEM_DTYPE).reshape(-1),
            stats.cpu().numpy().view(SCHEDULE_STATS_DTYPE)[0])


def candidate_record_error(r) -> str | None:
    """ValidateCandidateRecord's message (common/validators.cpp:160-181) for
    one CANDIDATE_RECORD_DTYPE record, None when valid."""
    if int(r["schema_version"]) != 1:
        return "CandidateRecord.schema_version is unsupported"
    if int(r["candidate_id"]) == 0:
        return "CandidateRecord.candidate_id is required"
    if int(r["query_id"]) == 0:
        return "CandidateRecord.query_id is required"
    if int(r["proxy_type_a"]) not in (1, 2):
        return "CandidateRecord.proxy_type_a must be a concrete proxy type"
    if int(r["proxy_type_b"]) not in (1, 2):
        return "CandidateRecord.proxy_type_b must be a concrete proxy type"
    if int(r["rt_hit_count"]) == 0:
        return "CandidateRecord.rt_hit_count is required"
    mb = np.asarray(r["motion_bound"], np.float32)
    if not np.all(np.isfinite(mb)) or np.any(mb < 0):
        return "CandidateRecord.motion_bound must contain finite non-negative values"
    return None


def work_item_error(it) -> str | None:
    """ValidateExactWorkItem's message (common/validators.cpp:207-230)."""
    for k in ("work_item_id", "parent_candidate_id", "query_id"):
        if int(it[k]) == 0:
            return f"ExactWorkItem.{k} is required"
    t0, t1 = float(it["interval_t0"]), float(it["interval_t1"])
    if not np.isfinite(t0):
        return "interval_t0 must be finite"
    if not np.isfinite(t1):
        return "interval_t1 must be finite"
    if t0 < 0.0 or t1 > 1.0 or t0 > t1:
        return "interval must satisfy 0 <= interval_t0 <= interval_t1 <= 1"
    if int(it["feature_family_mask"]) == 0:
        return "ExactWorkItem.feature_family_mask is required"
    if not np.isfinite(np.float32(it["priority_score"])):
        return "ExactWorkItem.priority_score must be finite"
    if int(it["source"]) not in (0, 1, 2):
        return "ExactWorkItem.source is invalid"
    return None


def _first_message(records, check) -> str:
    for r in records:
        m = check(r)
        if m:
            return m
    return "validation failed"


def dummy_schedule(candidates: np.ndarray, primitive_count: int, raw_hit_count: int, compact_candidate_count: int,
                   masks: dict | None = None, materialize: bool = True, bypass: bool = False,
                   device: str | torch.device = "cuda", **config) -> tuple:
    """p2c_dummy_schedule: (work items, stats, feature rows, proposal outputs);
    rows and outputs are empty unless ``materialize`` (and never in the
    bypass).  ValueError with the reference's message on an invalid config,
    candidate or work item."""
    lib = _lib.load()
    d = torch.device(device)
    c = dict(DEFAULTS, **config)
    cfg = SchedulingConfigStruct()
    for k, v in c.items():
        setattr(cfg, k, int(v) if k in ("first_work_item_id", "conservative_feature_family_mask",
                                         "preserve_candidate_order") else float(v))
    cand = np.ascontiguousarray(candidates, CANDIDATE_RECORD_DTYPE)
    n = len(cand)
    keys = sorted(int(k) for k in (masks or {}))
    mq = _dev(np.array(keys, np.uint64), np.uint64, d) if keys else None
    mv = _dev(np.array([int(masks[k]) for k in keys], np.uint32), np.uint32, d) if keys else None
    dc = _dev(cand, CANDIDATE_RECORD_DTYPE, d)
    items = torch.empty((max(n, 1), EXACT_WORK_ITEM_DTYPE.itemsize), dtype=torch.uint8, device=d)
    art = materialize and not bypass
    rows = torch.zeros((max(n, 1), FEATURE_ROW_DTYPE.itemsize), dtype=torch.uint8, device=d) if art else None
    outs = torch.zeros((max(n, 1), PROPOSAL_OUTPUT_DTYPE.itemsize), dtype=torch.uint8, device=d) if art else None
    stats = torch.zeros(SCHEDULE_STATS_DTYPE.itemsize, dtype=torch.uint8, device=d)
    err = torch.zeros(3, dtype=torch.int64, device=d)
    ws = torch.empty(int(lib.p2c_schedule_work_items_workspace_bytes(n, 0, 0)), dtype=torch.uint8, device=d)
    ptr = lambda t: t.data_ptr() if t is not None else None
    _lib.check(lib.p2c_dummy_schedule(int(bool(bypass)), ptr(dc), n, int(primitive_count), int(raw_hit_count),
                                      int(compact_candidate_count), ptr(mq), ptr(mv), len(keys), ctypes.byref(cfg),
                                      ptr(rows), ptr(outs), items.data_ptr(), stats.data_ptr(), err.data_ptr(),
                                      ws.data_ptr(), ws.numel(), _stream_ptr(d)))
    e = int(err[0].item())
    host_items = items[:n].cpu().numpy().view(EXACT_WORK_ITEM_DTYPE).reshape(-1)
    if e & 1:
        raise ValueError(_first_message(cand, candidate_record_error))
    if e & 16:
        raise ValueError(_first_message(host_items, work_item_error))
    r = rows[:n].cpu().numpy().view(FEATURE_ROW_DTYPE).reshape(-1) if art else np.zeros(0, FEATURE_ROW_DTYPE)
    o = outs[:n].cpu().numpy().view(PROPOSAL_OUTPUT_DTYPE).reshape(-1) if art else np.zeros(0, PROPOSAL_OUTPUT_DTYPE)
    return host_items, stats.cpu().numpy().view(SCHEDULE_STATS_DTYPE)[0], r, o
